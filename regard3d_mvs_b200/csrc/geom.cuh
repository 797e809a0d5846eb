// Double-precision 3-vector products of the multi-view kernels, in the
// left-to-right order ((a0 x + a1 y) + a2 z) that the reference's Eigen
// expressions evaluate for a fixed 3x3 matrix times a vector (and the
// library is built without contraction).
#pragma once

#include "simt.cuh"

namespace r3dgpu {

// Row i of a row-major 3x3 matrix times (x, y, z).
R3D_DEVICE double row3(const double* m, int i, double x, double y, double z) {
  return (m[3 * i] * x + m[3 * i + 1] * y) + m[3 * i + 2] * z;
}

// Row i of the transpose (column i) times (x, y, z).
R3D_DEVICE double col3(const double* m, int i, double x, double y, double z) {
  return (m[i] * x + m[3 + i] * y) + m[6 + i] * z;
}

}  // namespace r3dgpu
