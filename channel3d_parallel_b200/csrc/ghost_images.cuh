#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace c3d {

// Ghost entries written by the thread that owns their source point
// (apply_boundary_conditions, src/boundary_conditions.f90:20-55): every
// ghost entry of a field of extents n1 x n2 x n3 is sign * F(fold(i), mapy(j),
// fold(k)) of one interior point, with the periodic folds 1 <- N+1,
// N+2 <- 2, N+3 <- 3 in x and z, and in y the odd reflections j = 1 <- -F(2),
// j = n2 <- -F(n2-1) (cell-centred y) or zero wall values (y faces, V).
// x images of interior index i in a field of x extent n1 (0: none)
struct XImages {
  int a, b;
};
__device__ __forceinline__ XImages x_images(int i, int Nx, int n1) {
  return XImages{i == Nx + 1 ? 1 : 0, i + Nx <= n1 ? i + Nx : 0};
}
// row1: the entry x = 1 of the row
__device__ __forceinline__ void put_row(double* __restrict__ row1, int i, XImages xi, double v) {
  row1[i - 1] = v;
  if (xi.a) row1[0] = v;
  if (xi.b) row1[xi.b - 1] = v;
}
// v at interior point (i, j, k) and every ghost entry whose source it is
static __device__ __noinline__ void put_images_all(double* __restrict__ F, int n1, int n2, int n3, int Nx, int Nz,
                                            bool yface, int i, int j, int k, double v) {
  const XImages xi = x_images(i, Nx, n1);
  const int za = k == Nz + 1 ? 1 : 0, zb = k + Nz <= n3 ? k + Nz : 0;
  const int ja = yface ? 0 : (j == 2 ? 1 : (j == n2 - 1 ? n2 : 0));
  auto row = [&](int jj, int kk) { return F + (int64_t)n1 * ((jj - 1) + (int64_t)n2 * (kk - 1)); };
  put_row(row(j, k), i, xi, v);
  if (za) put_row(row(j, za), i, xi, v);
  if (zb) put_row(row(j, zb), i, xi, v);
  if (ja) {
    put_row(row(ja, k), i, xi, -v);
    if (za) put_row(row(ja, za), i, xi, -v);
    if (zb) put_row(row(ja, zb), i, xi, -v);
  }
}

}  // namespace c3d
