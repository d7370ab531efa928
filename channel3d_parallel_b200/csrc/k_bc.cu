// Boundary conditions: apply_boundary_conditions of src/boundary_conditions.f90:20-55
// for one z slab.
//
// The reference applies, in order, periodic copies in x (:67-86), periodic
// copies in z (:91-224) and the wall conditions in y (:237-252).  Every ghost
// entry therefore ends up as  sign_y * F(mapx(i), mapy(j), mapz(k))  of an
// interior entry, where mapx/mapz fold the periodic images
// (1 -> N+1, N+2 -> 2, N+3 -> 3) and mapy reflects the y ghosts (odd) or
// zeroes the wall faces of V.  This kernel writes exactly that value into
// every ghost entry in one pass, touching only the boundary shell.
#include "c3d_internal.cuh"

namespace c3d {

struct GhostField {
  double* F;
  int n1, n2, n3;     // array extents
  int yface;          // 1: y faces with zero wall values (V); 0: odd y ghosts
  int64_t cX, cZ, cY; // counts of the three disjoint ghost sets
};

__device__ __forceinline__ int fold(int i, int N) {
  return (i == 1) ? (N + 1) : ((i >= N + 2) ? (i - N) : i);
}

__global__ void k_fill_ghosts(GhostField f0, GhostField f1, GhostField f2, int Nx, int Nz) {
  GhostField f = (blockIdx.y == 0) ? f0 : ((blockIdx.y == 1) ? f1 : f2);
  if (f.F == nullptr) return;
  const int64_t total = f.cX + f.cZ + f.cY;
  const int gx = f.n1 - Nx;   // number of x ghost planes
  const int gz = f.n3 - Nz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    if (t < f.cX) {                          // x ghost planes, all j, all k
      int64_t r = t;
      int a = (int)(r % gx); r /= gx;
      j = 1 + (int)(r % f.n2); r /= f.n2;
      k = 1 + (int)r;
      i = (a == 0) ? 1 : (Nx + 1 + a);
    } else if (t < f.cX + f.cZ) {            // z ghost planes, interior i, all j
      int64_t r = t - f.cX;
      i = 2 + (int)(r % Nx); r /= Nx;
      j = 1 + (int)(r % f.n2); r /= f.n2;
      int a = (int)r;
      k = (a == 0) ? 1 : (Nz + 1 + a);
    } else {                                 // y ghost rows, interior i, interior k
      int64_t r = t - f.cX - f.cZ;
      i = 2 + (int)(r % Nx); r /= Nx;
      int a = (int)(r % 2); r /= 2;
      k = 2 + (int)r;
      j = a ? f.n2 : 1;
    }
    const int64_t dst = (int64_t)(i - 1) + (int64_t)f.n1 * ((j - 1) + (int64_t)f.n2 * (k - 1));
    double v;
    if (f.yface && (j == 1 || j == f.n2)) {
      v = 0.0;
    } else {
      int sj = j;
      double s = 1.0;
      if (!f.yface) {
        if (j == 1) { sj = 2; s = -1.0; }
        else if (j == f.n2) { sj = f.n2 - 1; s = -1.0; }
      }
      const int si = fold(i, Nx), sk = fold(k, Nz);
      const int64_t src = (int64_t)(si - 1) + (int64_t)f.n1 * ((sj - 1) + (int64_t)f.n2 * (sk - 1));
      v = s * f.F[src];
    }
    f.F[dst] = v;
  }
}

static GhostField make_ghost(const Dims& d, double* F, FieldKind kind) {
  GhostField g{};
  g.F = F;
  if (kind == KIND_U) { g.n1 = d.nx; g.n2 = d.nyg; g.n3 = d.nzg; g.yface = 0; }
  else if (kind == KIND_V) { g.n1 = d.nxg; g.n2 = d.ny; g.n3 = d.nzg; g.yface = 1; }
  else { g.n1 = d.nxg; g.n2 = d.nyg; g.n3 = d.nz; g.yface = 0; }
  const int gx = g.n1 - d.Nx, gz = g.n3 - d.Nz;
  g.cX = (int64_t)gx * g.n2 * g.n3;
  g.cZ = (int64_t)d.Nx * g.n2 * gz;
  g.cY = (int64_t)d.Nx * 2 * d.Nz;
  return g;
}

int launch_fill_ghosts3(Handle* h, double* U, double* V, double* W) {
  GhostField a = make_ghost(h->d, U, KIND_U);
  GhostField b = make_ghost(h->d, V, KIND_V);
  GhostField c = make_ghost(h->d, W, KIND_W);
  int64_t mx = a.cX + a.cZ + a.cY;
  int64_t bx = (mx + 255) / 256;
  if (bx > 148 * 16) bx = 148 * 16;
  dim3 grid((unsigned)bx, 3);
  k_fill_ghosts<<<grid, 256, 0, h->stream>>>(a, b, c, h->d.Nx, h->d.Nz);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

int launch_fill_ghosts(Handle* h, double* F, FieldKind kind) {
  GhostField a = make_ghost(h->d, F, kind);
  GhostField z{};
  z.F = nullptr;
  int64_t mx = a.cX + a.cZ + a.cY;
  int64_t bx = (mx + 255) / 256;
  if (bx > 148 * 16) bx = 148 * 16;
  dim3 grid((unsigned)bx, 1);
  k_fill_ghosts<<<grid, 256, 0, h->stream>>>(a, z, z, h->d.Nx, h->d.Nz);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

}  // namespace c3d
