// Actual pressure, compute_pressure of src/pressure.f90:21-341.
//
//   bc_1, bc_2 = d/dy(nu dV/dy) at the walls            (:270-341)
//   rhs_p      = div(rhs_u, rhs_v, rhs_w), rhs_u and rhs_w periodic, bc_1 and
//                bc_2 as the wall values of rhs_v        (:42-70, :237-247)
//   Laplacian(P) = rhs_p with dP/dy = bc at the walls: the projection's
//                Poisson solve with the inhomogeneous Neumann rows moved to
//                the right-hand side, rhs(2) += coef_bc_1*(yg(2)-yg(1))*bc_1,
//                rhs(nyg-1) -= coef_bc_2*(yg(nyg)-yg(nyg-1))*bc_2 (:135-137;
//                the reference adds them to the transformed rows, the DFT is
//                linear, so they are added before the transform here)
//   P(2:nxg-2, 2:nyg-1, 2:nzg-2) = solution, y ghosts from the wall
//                conditions, periodic copies (:147-165, :173-187).
// The reference's y-ghost assignment (:160-161) takes a whole (nxg, nzg)
// section of P from bc_1, which is allocated (2:nxg-1, 2:nzg-1)
// (src/initialization.f90:385): the shapes do not conform.  It is applied
// over bc_1's domain; the x and z ghost planes of P keep their values.
#include "c3d_internal.cuh"

namespace c3d {

struct WallMetric {
  double gb, g2b, gt, g2t;   // dy/dzeta and d2y/dzeta2 at the bottom and top walls (dzeta = 1)
};

__device__ __forceinline__ int64_t bcidx(const Dims& d, int i, int k) {
  return (int64_t)(i - 1) + (int64_t)d.nxg * (k - 1);
}

// bc_1(i,k), bc_2(i,k) for i = 2..nxg-1, k = 2..nzg-1 (src/pressure.f90:270-341)
__global__ void k_pressure_bc(Dims d, WallMetric w, double nu, const double* __restrict__ V,
                              double* __restrict__ bc1, double* __restrict__ bc2) {
  const int ni = d.nxg - 2, nk = d.nzg - 2;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ni * nk; t += gridDim.x * blockDim.x) {
    const int i = 2 + t % ni, k = 2 + t / ni;
    const double v1 = V[idxV(d, i, 1, k)], v2 = V[idxV(d, i, 2, k)];
    const double v3 = V[idxV(d, i, 3, k)], v4 = V[idxV(d, i, 4, k)];
    double dV = (-3.0 * v1 + 4.0 * v2 - v3) / 2.0 * 1.0 / w.gb;
    double ddV = 2.0 * v1 - 5.0 * v2 + 4.0 * v3 - 1.0 * v4;
    ddV = (ddV - dV * w.g2b) / (w.gb * w.gb);
    bc1[bcidx(d, i, k)] = 0.0 * dV + nu * ddV;
    const int ny = d.ny;
    const double t1 = V[idxV(d, i, ny, k)], t2 = V[idxV(d, i, ny - 1, k)];
    const double t3 = V[idxV(d, i, ny - 2, k)], t4 = V[idxV(d, i, ny - 3, k)];
    dV = (3.0 * t1 - 4.0 * t2 + t3) / 2.0 * 1.0 / w.gt;
    ddV = 2.0 * t1 - 5.0 * t2 + 4.0 * t3 - 1.0 * t4;
    ddV = (ddV - dV * w.g2t) / (w.gt * w.gt);
    bc2[bcidx(d, i, k)] = 0.0 * dV + nu * ddV;
  }
}

// rhs_p(i,j,k), i = 2..nxg-1, j = 2..nyg-1, k = 2..nzg-1, from the interior
// right-hand sides (layouts of C3D_FIELD_RHS_U/V/W), plus the wall rows of
// the Neumann conditions on the transformed region (i <= nxg-2, k <= nzg-2)
__global__ void k_pressure_div(Dims d, Metric m, const double* __restrict__ ru, const double* __restrict__ rv,
                               const double* __restrict__ rw, const double* __restrict__ bc1,
                               const double* __restrict__ bc2, double cb1, double cb2,
                               double* __restrict__ rhs) {
  const int64_t nu1 = d.nx - 2, nu2 = d.nyg - 2;            // rhs_u(2:nx-1, 2:nyg-1, 2:nzg-1)
  const int64_t nv1 = d.nxg - 2, nv2 = d.ny - 2;            // rhs_v(2:nxg-1, 2:ny-1, 2:nzg-1)
  const int64_t nw1 = d.nxg - 2, nw2 = d.nyg - 2;           // rhs_w(2:nxg-1, 2:nyg-1, 2:nz-1)
  auto RU = [&](int i, int j, int k) {                      // periodic in x (face copy)
    if (i == 1) i = d.nx - 1;
    else if (i == d.nx) i = 2;
    return ru[(i - 2) + nu1 * ((j - 2) + nu2 * (int64_t)(k - 2))];
  };
  auto RV = [&](int i, int j, int k) {                      // walls: bc_1, bc_2
    if (j == 1) return bc1[bcidx(d, i, k)];
    if (j == d.ny) return bc2[bcidx(d, i, k)];
    return rv[(i - 2) + nv1 * ((j - 2) + nv2 * (int64_t)(k - 2))];
  };
  auto RW = [&](int i, int j, int k) {                      // periodic in z (face copy)
    if (k == 1) k = d.nz - 1;
    else if (k == d.nz) k = 2;
    return rw[(i - 2) + nw1 * ((j - 2) + nw2 * (int64_t)(k - 2))];
  };
  const int ni = d.nxg - 2, nj = d.nyg - 2, nk = d.nzg - 2;
  const int64_t tot = (int64_t)ni * nj * nk;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 2 + (int)(t % ni);
    const int j = 2 + (int)((t / ni) % nj);
    const int k = 2 + (int)(t / ((int64_t)ni * nj));
    double v = (RU(i, j, k) - RU(i - 1, j, k)) * m.rdx[i] + (RV(i, j, k) - RV(i, j - 1, k)) * m.rdy[j] +
               (RW(i, j, k) - RW(i, j, k - 1)) * m.rdz[k];
    if (i <= d.nxg - 2 && k <= d.nzg - 2) {
      if (j == 2) v = v + cb1 * bc1[bcidx(d, i, k)];
      if (j == d.nyg - 1) v = v - cb2 * bc2[bcidx(d, i, k)];
    }
    rhs[idxR(d, i, j, k)] = v;
  }
}

// P(i, j, k) for i = 2..nxg-1, k = 2..nzg-1 and every j: the solution on
// j = 2..nyg-1, the y ghosts from the wall conditions; the periodic copies
// i = nxg-1 and k = nzg-1 take the values of i = 2 and k = 2
__global__ void k_pressure_store(Dims d, const double* __restrict__ phi, const double* __restrict__ bc1,
                                 const double* __restrict__ bc2, double dyb, double dyt, double* __restrict__ P) {
  const int ni = d.nxg - 2, nj = d.nyg, nk = d.nzg - 2;
  const int64_t tot = (int64_t)ni * nj * nk;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 2 + (int)(t % ni);
    const int j = 1 + (int)((t / ni) % nj);
    const int k = 2 + (int)(t / ((int64_t)ni * nj));
    const int is = (i == d.nxg - 1) ? 2 : i, ks = (k == d.nzg - 1) ? 2 : k;
    double v;
    if (j == 1) v = phi[idxR(d, is, 2, ks)] - dyb * bc1[bcidx(d, is, ks)];
    else if (j == d.nyg) v = phi[idxR(d, is, d.nyg - 1, ks)] + dyt * bc2[bcidx(d, is, ks)];
    else v = phi[idxR(d, is, j, ks)];
    P[idxP(d, i, j, k)] = v;
  }
}

int compute_pressure(Handle* h) {
  const Dims& d = h->d;
  int rc;
  if (d.ny < 4) {
    h->last_error = "compute_pressure needs ny_global >= 4 (one-sided wall differences)";
    return C3D_ERR_PARAM;
  }
  if (!h->pbc && (rc = dev_alloc(h, &h->pbc, 2 * (int64_t)d.nxg * d.nzg))) return rc;
  double* bc1 = h->pbc;
  double* bc2 = h->pbc + (int64_t)d.nxg * d.nzg;
  // P's x and z ghost planes keep their current values
  if ((rc = rebuild_pressure(h))) return rc;
  const std::vector<double>& y = h->y;
  const std::vector<double>& yg = h->yg;
  const int ny = d.ny, nyg = d.nyg;
  WallMetric w;
  w.gb = (-3.0 * y[1] + 4.0 * y[2] - y[3]) / 2.0;
  w.g2b = 2.0 * y[1] - 5.0 * y[2] + 4.0 * y[3] - 1.0 * y[4];
  w.gt = (3.0 * y[ny] - 4.0 * y[ny - 1] + y[ny - 2]) / 2.0;
  w.g2t = 2.0 * y[ny] - 5.0 * y[ny - 1] + 4.0 * y[ny - 2] - 1.0 * y[ny - 3];
  const int nbc = (d.nxg - 2) * (d.nzg - 2);
  k_pressure_bc<<<(nbc + 255) / 256, 256, 0, h->stream>>>(d, w, h->p.nu, h->V, bc1, bc2);
  C3D_LAUNCH_CHECK(h);
  for (int c = 1; c <= 3; ++c)
    if ((rc = launch_rhs_only(h, c))) return rc;
  // coef_bc_1 = c(2), coef_bc_2 = a(nyg-1) of the Dyy set-up, src/initialization.f90:366-383
  const double coef1 = 1.0 / (y[2] - y[1]) / (yg[2] - yg[1]);
  const double coef2 = 1.0 / (y[nyg - 1] - y[nyg - 2]) / (yg[nyg] - yg[nyg - 1]);
  const double dyb = yg[2] - yg[1], dyt = yg[nyg] - yg[nyg - 1];
  k_pressure_div<<<148 * 8, 256, 0, h->stream>>>(d, h->m, h->rhsU, h->rhsV, h->rhsW, bc1, bc2, coef1 * dyb,
                                                 coef2 * dyt, h->rhs_p);
  C3D_LAUNCH_CHECK(h);
  if ((rc = launch_poisson_solve(h, h->rhs_p, 0, 1.0))) return rc;
  k_pressure_store<<<148 * 8, 256, 0, h->stream>>>(d, h->rhs_p, bc1, bc2, dyb, dyt, h->P);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

}  // namespace c3d
