// CUDA runtime API used by the host side of r3dgpu. The product build uses the
// real runtime; the test-only emulator build (R3DGPU_SIMT_EMULATION) maps the
// same calls onto host memory (tests/simt/fake_cuda_runtime.h).
#pragma once

#ifndef R3DGPU_SIMT_EMULATION
#include <cuda_runtime.h>
#else
#include "../../tests/simt/fake_cuda_runtime.h"
#endif

#include "simt.cuh"
