// The C ABI's error contract for the entry points outside the matcher: run
// the body, map r3dgpu::Error to its status, host allocation failures to
// R3DGPU_ENOMEM and other exceptions to R3DGPU_EDEVICE, and leave the
// message for r3dgpu_last_error on this thread ("" after success).
#pragma once

#include <new>

#include "common.cuh"
#include "matcher_internal.h"

namespace r3dgpu {

template <class F>
r3dgpu_status guard(F&& f) {
  try {
    set_thread_error("");
    f();
    return R3DGPU_OK;
  } catch (const Error& e) {
    set_thread_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_thread_error("r3dgpu: out of host memory");
    return R3DGPU_ENOMEM;
  } catch (const std::exception& e) {
    set_thread_error(e.what());
    return R3DGPU_EDEVICE;
  }
}

}  // namespace r3dgpu
