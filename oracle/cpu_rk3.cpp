// C++/OpenMP restatement of the reference's FP64 RK3 fractional-step time
// advance for body_type = 'none' on one domain -- TEST AND BASELINE
// INFRASTRUCTURE ONLY.  The CUDA library never links or calls it; it is the
// timed CPU baseline (the Intel/MPI/FFTW reference cannot be built here) and
// is checked against the NumPy restatement in oracle/channel_oracle.py.
//
// It follows the same reference code, operation for operation where the
// NumPy oracle fixes an order:
//   compute_time_step_RK3       src/time_integration.f90:86-213
//   compute_dt                  src/time_integration.f90:219-267
//   compute_rhs_u/v/w           src/equations.f90:24-423
//   divergence, gradient        src/differential_operators.f90:16-74
//   solve_poisson_equation      src/poisson.f90:33-156 (2-D complex DFT per
//                               y plane, zgtsv per mode, 00-mode pin)
//   compute_non_IB_projection   src/projection.f90:22-46
//   apply_boundary_conditions   src/boundary_conditions.f90:20-252
//   constant mass flow          src/mass_flow.f90:144-175
// Two third-party steps are restated from their published algorithms: the
// DFT (FFTW in the reference) as a mixed-radix 2/3/4/5 Stockham FFT, and
// LAPACK zgtsv as Gaussian elimination with partial pivoting on the
// tridiagonal matrix.
//
// Arrays are Fortran-indexed with an unused index 0 in every axis (the
// oracle's convention): A(i,j,k) of extents (n1, n2, n3) is stored at
// i + (n1+1)*(j + (n2+1)*k), x fastest.
#include <cmath>
#include <complex>
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

using cd = std::complex<double>;

// RK3 tableau, src/initialization.f90:406-418
const double kRkT[3] = {8.0 / 15.0, 2.0 / 3.0, 1.0};
const double kRkCoef[3][3] = {{8.0 / 15.0, 0.0, 0.0}, {1.0 / 4.0, 5.0 / 12.0, 0.0}, {1.0 / 4.0, 0.0, 3.0 / 4.0}};

struct Arr {
  int n1 = 0, n2 = 0, n3 = 0;
  int64_t s1 = 0, s2 = 0;
  std::vector<double> a;
  void init(int e1, int e2, int e3) {
    n1 = e1; n2 = e2; n3 = e3;
    s1 = n1 + 1; s2 = (int64_t)(n1 + 1) * (n2 + 1);
    a.assign((size_t)(n1 + 1) * (n2 + 1) * (n3 + 1), 0.0);
  }
  double& operator()(int i, int j, int k) { return a[(size_t)(i + s1 * j + s2 * k)]; }
  double operator()(int i, int j, int k) const { return a[(size_t)(i + s1 * j + s2 * k)]; }
};

// ---------------------------------------------------------------------------
// FFT: out-of-place Stockham passes of radix 4, 2, 3, 5 over one line
// ---------------------------------------------------------------------------
struct Fft {
  int n = 0;
  std::vector<int> radix;
  std::vector<cd> w;   // exp(-2 pi i m / n), m < n
  void init(int len) {
    n = len;
    radix.clear();
    int r = n;
    while (r % 4 == 0) { radix.push_back(4); r /= 4; }
    while (r % 2 == 0) { radix.push_back(2); r /= 2; }
    while (r % 3 == 0) { radix.push_back(3); r /= 3; }
    while (r % 5 == 0) { radix.push_back(5); r /= 5; }
    w.resize(n);
    for (int m = 0; m < n; ++m) {
      const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
      w[m] = cd((double)std::cos(ang), (double)std::sin(ang));
    }
  }
  bool ok() const {
    int p = 1;
    for (int r : radix) p *= r;
    return p == n;
  }
  // One Stockham autosort pass of radix R: butterfly j takes
  // src[j + r*n/R] * w^(r*(j mod Ns)), w = exp(-+2 pi i/(Ns*R)), and writes
  // DFT_R(...)[q] to dst[(j div Ns)*Ns*R + (j mod Ns) + q*Ns].  Butterflies
  // sharing j mod Ns share their twiddles.
  template <int R>
  void pass(const cd* src, cd* dst, int Ns, int sign) const {
    const int nb = n / R;
    const int tws = n / (Ns * R);
    const int nblk = nb / Ns;
    const double s3 = 0.86602540378443864676;   // sqrt(3)/2
    for (int kk = 0; kk < Ns; ++kk) {
      cd t[R];
      for (int r = 1; r < R; ++r) {
        t[r] = w[(size_t)r * kk * tws];
        if (sign > 0) t[r] = std::conj(t[r]);
      }
      for (int blk = 0; blk < nblk; ++blk) {
        const int j = blk * Ns + kk;
        cd v[R], o[R];
        v[0] = src[j];
        for (int r = 1; r < R; ++r) v[r] = kk > 0 ? src[j + r * nb] * t[r] : src[j + r * nb];
        if constexpr (R == 2) {
          o[0] = v[0] + v[1];
          o[1] = v[0] - v[1];
        } else if constexpr (R == 4) {
          const cd a0 = v[0] + v[2], a1 = v[0] - v[2], a2 = v[1] + v[3], d = v[1] - v[3];
          const cd a3 = (sign < 0) ? cd(d.imag(), -d.real()) : cd(-d.imag(), d.real());
          o[0] = a0 + a2;
          o[1] = a1 + a3;
          o[2] = a0 - a2;
          o[3] = a1 - a3;
        } else if constexpr (R == 3) {
          const cd sm = v[1] + v[2], df = v[1] - v[2];
          const cd m = v[0] - 0.5 * sm;
          const cd id = (sign < 0) ? cd(s3 * df.imag(), -s3 * df.real()) : cd(-s3 * df.imag(), s3 * df.real());
          o[0] = v[0] + sm;
          o[1] = m + id;
          o[2] = m - id;
        } else {
          for (int q = 0; q < R; ++q) {
            cd acc = v[0];
            for (int r = 1; r < R; ++r) {
              cd tw = w[(size_t)((r * q) % R) * (n / R)];
              if (sign > 0) tw = std::conj(tw);
              acc += v[r] * tw;
            }
            o[q] = acc;
          }
        }
        const int base = blk * Ns * R + kk;
        for (int q = 0; q < R; ++q) dst[base + q * Ns] = o[q];
      }
    }
  }
  // sign = -1 forward, +1 inverse (unnormalised); x and tmp hold n values;
  // natural order in and out
  void run(cd* x, cd* tmp, int sign) const {
    cd* src = x;
    cd* dst = tmp;
    int Ns = 1;
    for (int R : radix) {
      if (R == 4) pass<4>(src, dst, Ns, sign);
      else if (R == 2) pass<2>(src, dst, Ns, sign);
      else if (R == 3) pass<3>(src, dst, Ns, sign);
      else pass<5>(src, dst, Ns, sign);
      std::swap(src, dst);
      Ns *= R;
    }
    if (src != x) std::memcpy(x, src, sizeof(cd) * n);
  }
};

// LAPACK zgtsv algorithm (Gaussian elimination with partial pivoting on a
// tridiagonal matrix, the reference's call at src/poisson.f90:72); dl, d, du
// are overwritten; b (n values) becomes the solution.  Returns info.
int zgtsv(int n, cd* dl, cd* d, cd* du, cd* b) {
  auto cabs1 = [](cd z) { return std::fabs(z.real()) + std::fabs(z.imag()); };
  for (int k = 0; k < n - 1; ++k) {
    if (dl[k] == cd(0.0, 0.0)) {
      if (d[k] == cd(0.0, 0.0)) return k + 1;   // singular
    } else if (cabs1(d[k]) >= cabs1(dl[k])) {
      const cd mult = dl[k] / d[k];
      d[k + 1] -= mult * du[k];
      b[k + 1] -= mult * b[k];
      if (k < n - 2) dl[k] = 0.0;
    } else {
      const cd mult = d[k] / dl[k];
      d[k] = dl[k];
      const cd temp = d[k + 1];
      d[k + 1] = du[k] - mult * temp;
      if (k < n - 2) {
        dl[k] = du[k + 1];
        du[k + 1] = -mult * dl[k];
      }
      du[k] = temp;
      const cd tb = b[k];
      b[k] = b[k + 1];
      b[k + 1] = tb - mult * b[k + 1];
    }
  }
  if (d[n - 1] == cd(0.0, 0.0)) return n;
  b[n - 1] /= d[n - 1];
  if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
  for (int k = n - 3; k >= 0; --k) b[k] = (b[k] - du[k] * b[k + 1] - dl[k] * b[k + 2]) / d[k];
  return 0;
}

struct Solver {
  int nx, ny, nz, nxg, nyg, nzg, nxp, nzp;
  double nu;
  int x_mass_cte, epg, nthreads;
  double cfl;
  std::vector<double> x, y, z, xg, yg, zg;   // Fortran-indexed (index 0 unused)
  std::vector<double> kxx, kzz, Dd, Dl, Du;
  Arr U, V, W, P, Pint, Uo, Vo, Wo;
  Arr Fu[3], Fv[3], Fw[3];
  Arr rhs;
  std::vector<cd> hat;                       // [j][k'][i'] spectrum
  Fft fx, fz;
  double dPdx = 0, dPdy = 0, dPdz = 0, Q0 = 0, t = 0;

  void apply_bc() {
    // src/boundary_conditions.f90:20-55: periodic x (:67-86), periodic z
    // (:91-224, one domain), walls in y (:237-252)
    auto bcx = [&](Arr& F, bool face) {
#pragma omp parallel for collapse(2) num_threads(nthreads)
      for (int k = 1; k <= F.n3; ++k)
        for (int j = 1; j <= F.n2; ++j) {
          if (face) {
            F(1, j, k) = F(nx - 1, j, k);
            F(nx, j, k) = F(2, j, k);
          } else {
            F(1, j, k) = F(nxg - 2, j, k);
            F(nxg - 1, j, k) = F(2, j, k);
            F(nxg, j, k) = F(3, j, k);
          }
        }
    };
    auto bcz = [&](Arr& F, bool face) {
#pragma omp parallel for num_threads(nthreads)
      for (int j = 1; j <= F.n2; ++j)
        for (int i = 1; i <= F.n1; ++i) {
          if (face) {
            const double top = F(i, j, nz - 1), bot = F(i, j, 2);
            F(i, j, 1) = top;
            F(i, j, nz) = bot;
          } else {
            const double top = F(i, j, nzg - 2), b2 = F(i, j, 2), b3 = F(i, j, 3);
            F(i, j, 1) = top;
            F(i, j, nzg - 1) = b2;
            F(i, j, nzg) = b3;
          }
        }
    };
    auto bcy = [&](Arr& F, bool face) {
#pragma omp parallel for num_threads(nthreads)
      for (int k = 1; k <= F.n3; ++k)
        for (int i = 1; i <= F.n1; ++i) {
          if (face) {
            F(i, 1, k) = 0.0;
            F(i, ny, k) = 0.0;
          } else {
            F(i, 1, k) = -F(i, 2, k);
            F(i, nyg, k) = -F(i, nyg - 1, k);
          }
        }
    };
    bcx(U, true); bcx(V, false); bcx(W, false);
    bcz(U, false); bcz(V, false); bcz(W, true);
    bcy(U, false); bcy(V, true); bcy(W, false);
  }

  // src/equations.f90:24-153 -> F(2:nx-1, 2:nyg-1, 2:nzg-1)
  void rhs_u(Arr& F) {
    const double dp = dPdx;
#pragma omp parallel for num_threads(nthreads)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          const double am = 0.5 * (U(i - 1, j, k) + U(i, j, k)), ap = 0.5 * (U(i, j, k) + U(i + 1, j, k));
          double r = -(ap * ap - am * am) / (xg[i + 1] - xg[i]);
          const double b1 = (0.5 * (U(i, j, k) + U(i, j + 1, k))) * (0.5 * (V(i, j, k) + V(i + 1, j, k)));
          const double b0 = (0.5 * (U(i, j - 1, k) + U(i, j, k))) * (0.5 * (V(i, j - 1, k) + V(i + 1, j - 1, k)));
          r = r + (-(b1 - b0) / (y[j] - y[j - 1]));
          const double c1 = (0.5 * (U(i, j, k) + U(i, j, k + 1))) * (0.5 * (W(i, j, k) + W(i + 1, j, k)));
          const double c0 = (0.5 * (U(i, j, k - 1) + U(i, j, k))) * (0.5 * (W(i, j, k - 1) + W(i + 1, j, k - 1)));
          r = r + (-(c1 - c0) / (z[k] - z[k - 1]));
          const double Uc = U(i, j, k);
          const double dyp = (U(i, j + 1, k) - Uc) / (yg[j + 1] - yg[j]);
          const double dym = (Uc - U(i, j - 1, k)) / (yg[j] - yg[j - 1]);
          const double dx1 = x[i] - x[i - 1], dx2 = x[i + 1] - x[i], dx3 = xg[i + 1] - xg[i];
          const double dy3 = y[j] - y[j - 1];
          const double dz1 = zg[k] - zg[k - 1], dz2 = zg[k + 1] - zg[k], dz3 = z[k] - z[k - 1];
          const double visc =
              1.0 / dx3 * (nu * 1.0 / dx2 * (U(i + 1, j, k) - Uc) - nu * 1.0 / dx1 * (Uc - U(i - 1, j, k))) +
              1.0 / dy3 * (nu * dyp - nu * dym) +
              1.0 / dz3 * (nu * 1.0 / dz2 * (U(i, j, k + 1) - Uc) - nu * 1.0 / dz1 * (Uc - U(i, j, k - 1)));
          r = r + visc;
          F(i, j, k) = r + dp;
        }
  }

  // src/equations.f90:160-288 -> F(2:nxg-1, 2:ny-1, 2:nzg-1)
  void rhs_v(Arr& F) {
    const double dp = dPdy;
#pragma omp parallel for num_threads(nthreads)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) {
          const double am = 0.5 * (V(i, j - 1, k) + V(i, j, k)), ap = 0.5 * (V(i, j, k) + V(i, j + 1, k));
          double r = -(ap * ap - am * am) / (yg[j + 1] - yg[j]);
          const double b1 = (0.5 * (U(i, j, k) + U(i, j + 1, k))) * (0.5 * (V(i, j, k) + V(i + 1, j, k)));
          const double b0 = (0.5 * (U(i - 1, j, k) + U(i - 1, j + 1, k))) * (0.5 * (V(i - 1, j, k) + V(i, j, k)));
          r = r + (-(b1 - b0) / (x[i] - x[i - 1]));
          const double c1 = (0.5 * (V(i, j, k) + V(i, j, k + 1))) * (0.5 * (W(i, j, k) + W(i, j + 1, k)));
          const double c0 = (0.5 * (V(i, j, k - 1) + V(i, j, k))) * (0.5 * (W(i, j, k - 1) + W(i, j + 1, k - 1)));
          r = r + (-(c1 - c0) / (z[k] - z[k - 1]));
          const double Vc = V(i, j, k);
          const double dx1 = xg[i] - xg[i - 1], dx2 = xg[i + 1] - xg[i], dx3 = x[i] - x[i - 1];
          const double dy1 = y[j] - y[j - 1], dy2 = y[j + 1] - y[j], dy3 = yg[j + 1] - yg[j];
          const double dz1 = zg[k] - zg[k - 1], dz2 = zg[k + 1] - zg[k], dz3 = z[k] - z[k - 1];
          const double visc =
              1.0 / dx3 * (nu * 1.0 / dx2 * (V(i + 1, j, k) - Vc) - nu * 1.0 / dx1 * (Vc - V(i - 1, j, k))) +
              1.0 / dy3 * (nu * 1.0 / dy2 * (V(i, j + 1, k) - Vc) - nu * 1.0 / dy1 * (Vc - V(i, j - 1, k))) +
              1.0 / dz3 * (nu * 1.0 / dz2 * (V(i, j, k + 1) - Vc) - nu * 1.0 / dz1 * (Vc - V(i, j, k - 1)));
          r = r + visc;
          F(i, j, k) = r + dp;
        }
  }

  // src/equations.f90:295-423 -> F(2:nxg-1, 2:nyg-1, 2:nz-1)
  void rhs_w(Arr& F) {
    const double dp = dPdz;
#pragma omp parallel for num_threads(nthreads)
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) {
          const double am = 0.5 * (W(i, j, k - 1) + W(i, j, k)), ap = 0.5 * (W(i, j, k) + W(i, j, k + 1));
          double r = -(ap * ap - am * am) / (zg[k + 1] - zg[k]);
          const double b1 = (0.5 * (U(i, j, k) + U(i, j, k + 1))) * (0.5 * (W(i, j, k) + W(i + 1, j, k)));
          const double b0 = (0.5 * (U(i - 1, j, k) + U(i - 1, j, k + 1))) * (0.5 * (W(i - 1, j, k) + W(i, j, k)));
          r = r + (-(b1 - b0) / (x[i] - x[i - 1]));
          const double c1 = (0.5 * (V(i, j, k) + V(i, j, k + 1))) * (0.5 * (W(i, j, k) + W(i, j + 1, k)));
          const double c0 = (0.5 * (V(i, j - 1, k) + V(i, j - 1, k + 1))) * (0.5 * (W(i, j - 1, k) + W(i, j, k)));
          r = r + (-(c1 - c0) / (y[j] - y[j - 1]));
          const double Wc = W(i, j, k);
          const double dyp = (W(i, j + 1, k) - Wc) / (yg[j + 1] - yg[j]);
          const double dym = (Wc - W(i, j - 1, k)) / (yg[j] - yg[j - 1]);
          const double dx1 = xg[i] - xg[i - 1], dx2 = xg[i + 1] - xg[i], dx3 = x[i] - x[i - 1];
          const double dy3 = y[j] - y[j - 1];
          const double dz1 = z[k] - z[k - 1], dz2 = z[k + 1] - z[k], dz3 = zg[k + 1] - zg[k];
          const double visc =
              1.0 / dx3 * (nu * 1.0 / dx2 * (W(i + 1, j, k) - Wc) - nu * 1.0 / dx1 * (Wc - W(i - 1, j, k))) +
              1.0 / dy3 * (nu * dyp - nu * dym) +
              1.0 / dz3 * (nu * 1.0 / dz2 * (W(i, j, k + 1) - Wc) - nu * 1.0 / dz1 * (Wc - W(i, j, k - 1)));
          r = r + visc;
          F(i, j, k) = r + dp;
        }
  }

  // src/poisson.f90:33-125 on rhs(2:nxg-1, 2:nyg-1, 2:nzg)
  int poisson(int rk_step, double dt) {
    const int nj = nyg - 2;
    const size_t plane = (size_t)nxp * nzp;
    int info = 0;
    // forward 2-D DFT of every y plane: x lines, then z lines
#pragma omp parallel num_threads(nthreads)
    {
      std::vector<cd> line(std::max(nxp, nzp)), tmp(std::max(nxp, nzp));
#pragma omp for
      for (int jj = 0; jj < nj; ++jj) {
        cd* h = hat.data() + (size_t)jj * plane;
        for (int kp = 0; kp < nzp; ++kp) {
          for (int ip = 0; ip < nxp; ++ip) line[ip] = cd(rhs(ip + 2, jj + 2, kp + 2), 0.0);
          fx.run(line.data(), tmp.data(), -1);
          for (int ip = 0; ip < nxp; ++ip) h[(size_t)kp * nxp + ip] = line[ip];
        }
        for (int ip = 0; ip < nxp; ++ip) {
          for (int kp = 0; kp < nzp; ++kp) line[kp] = h[(size_t)kp * nxp + ip];
          fz.run(line.data(), tmp.data(), -1);
          for (int kp = 0; kp < nzp; ++kp) h[(size_t)kp * nxp + ip] = line[kp];
        }
      }
      // per-mode tridiagonal solves in y (src/poisson.f90:50-75); the columns
      // of a block of kx modes are gathered plane by plane (contiguous runs)
      constexpr int kBlk = 16;
      std::vector<cd> dl(nj), dd(nj), du(nj), cols((size_t)kBlk * nj);
      const int nbi = (nxp + kBlk - 1) / kBlk;
#pragma omp for collapse(2) reduction(| : info)
      for (int kp = 0; kp < nzp; ++kp)
        for (int bi = 0; bi < nbi; ++bi) {
          const int i0 = bi * kBlk, ni = std::min(kBlk, nxp - i0);
          for (int r = 0; r < nj; ++r) {
            const cd* src = hat.data() + (size_t)r * plane + (size_t)kp * nxp + i0;
            for (int q = 0; q < ni; ++q) cols[(size_t)q * nj + r] = src[q];
          }
          const int ka = kp <= nzp - kp ? kp : nzp - kp;
          for (int q = 0; q < ni; ++q) {
            const int ip = i0 + q;
            const int ia = ip <= nxp - ip ? ip : nxp - ip;
            for (int r = 0; r < nj; ++r) {
              double D = (Dd[r + 2] + kxx[ia]) + kzz[ka];
              if (ip == 0 && kp == 0 && r == 0) D = 3.0 / 2.0 * D;
              dd[r] = D;
              if (r < nj - 1) {
                dl[r] = Dl[r + 3];
                du[r] = Du[r + 2];
              }
            }
            if (zgtsv(nj, dl.data(), dd.data(), du.data(), cols.data() + (size_t)q * nj) != 0) info |= 1;
          }
          for (int r = 0; r < nj; ++r) {
            cd* dst = hat.data() + (size_t)r * plane + (size_t)kp * nxp + i0;
            for (int q = 0; q < ni; ++q) dst[q] = cols[(size_t)q * nj + r];
          }
        }
      // inverse DFT, 1/(nxp*nzp), real part (:78-82)
      const double scale = 1.0 / ((double)nxp * (double)nzp);
#pragma omp for
      for (int jj = 0; jj < nj; ++jj) {
        cd* h = hat.data() + (size_t)jj * plane;
        for (int ip = 0; ip < nxp; ++ip) {
          for (int kp = 0; kp < nzp; ++kp) line[kp] = h[(size_t)kp * nxp + ip];
          fz.run(line.data(), tmp.data(), +1);
          for (int kp = 0; kp < nzp; ++kp) h[(size_t)kp * nxp + ip] = line[kp];
        }
        for (int kp = 0; kp < nzp; ++kp) {
          for (int ip = 0; ip < nxp; ++ip) line[ip] = h[(size_t)kp * nxp + ip];
          fx.run(line.data(), tmp.data(), +1);
          for (int ip = 0; ip < nxp; ++ip) rhs(ip + 2, jj + 2, kp + 2) = (line[ip] * scale).real();
        }
      }
    }
    if (info) return -1;
    // apply_periodic_xz_centers (:106-125)
    for (int k = 1; k <= rhs.n3; ++k)
      for (int j = 1; j <= rhs.n2; ++j) rhs(nxg - 1, j, k) = rhs(2, j, k);
    for (int j = 1; j <= rhs.n2; ++j)
      for (int i = 2; i <= nxg - 1; ++i) rhs(i, j, nzp + 2) = rhs(i, j, 2);
    if (rk_step == 1) {
      // P side effect (:91-99)
      const double den = dt * kRkCoef[0][0];
#pragma omp parallel for num_threads(nthreads)
      for (int k = 2; k <= nzg - 1; ++k)
        for (int j = 2; j <= nyg - 1; ++j)
          for (int i = 2; i <= nxg - 1; ++i) P(i, j, k) = rhs(i, j, k) / den;
      for (int k = 1; k <= nzg; ++k)
        for (int j = 1; j <= nyg; ++j) { P(1, j, k) = P(2, j, k); P(nxg, j, k) = P(nxg - 1, j, k); }
      for (int k = 1; k <= nzg; ++k)
        for (int i = 1; i <= nxg; ++i) { P(i, 1, k) = P(i, 2, k); P(i, nyg, k) = P(i, nyg - 1, k); }
      for (int j = 1; j <= nyg; ++j)
        for (int i = 1; i <= nxg; ++i) { P(i, j, 1) = P(i, j, 2); P(i, j, nzg) = P(i, j, nzg - 1); }
    }
    return 0;
  }

  // src/projection.f90:22-46 with divergence and gradient of
  // src/differential_operators.f90:16-74
  int projection(int rk_step, double dt) {
    std::fill(rhs.a.begin(), rhs.a.end(), 0.0);
#pragma omp parallel for num_threads(nthreads)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i)
          rhs(i, j, k) = (U(i, j, k) - U(i - 1, j, k)) / (x[i] - x[i - 1]) +
                         (V(i, j, k) - V(i, j - 1, k)) / (y[j] - y[j - 1]) +
                         (W(i, j, k) - W(i, j, k - 1)) / (z[k] - z[k - 1]);
    if (poisson(rk_step, dt)) return -1;
    // rhs_p = rhs_p / dt; P_interim = rhs_p; rhs_p = dt * rhs_p
#pragma omp parallel for num_threads(nthreads)
    for (int64_t q = 0; q < (int64_t)rhs.a.size(); ++q) {
      const double s = rhs.a[q] / dt;
      Pint.a[q] = s;
      rhs.a[q] = dt * s;
    }
    // U = U - G phi (gradient: zero outside its loops)
#pragma omp parallel for num_threads(nthreads)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          U(i, j, k) = U(i, j, k) - (rhs(i + 1, j, k) - rhs(i, j, k)) / (xg[i + 1] - xg[i]);
          if (j <= ny - 1) V(i, j, k) = V(i, j, k) - (rhs(i, j + 1, k) - rhs(i, j, k)) / (yg[j + 1] - yg[j]);
          if (k <= nz - 1) W(i, j, k) = W(i, j, k) - (rhs(i, j, k + 1) - rhs(i, j, k)) / (zg[k + 1] - zg[k]);
        }
    return 0;
  }

  // src/mass_flow.f90:144-175 (flux and its normaliser; extended-precision
  // accumulation keeps the thread split from changing the sums)
  void mass_flow(double* q, double* norm) {
    long double sq = 0.0L, sn = 0.0L;
#pragma omp parallel for reduction(+ : sq, sn) num_threads(nthreads)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 3; j <= nyg - 1; ++j) {
        const double w = 0.5 * (yg[j] - yg[j - 1]);
        for (int i = 2; i <= nx - 1; ++i) {
          sq += (U(i, j, k) + U(i, j - 1, k)) * w;
          sn += 2.0 * w;
        }
      }
    *q = (double)sq;
    *norm = (double)sn;
  }

  // src/time_integration.f90:219-267; with CFL < 0 the reference still scans
  // the three fields before taking dt = -CFL
  double compute_dt() {
    double lU = 0.0, lV = 0.0, lW = 0.0;
#pragma omp parallel for reduction(max : lU, lV, lW) num_threads(nthreads)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) {
          lU = std::max(lU, (xg[i + 1] - xg[i]) / std::fabs(U(i, j, k)));
          lV = std::max(lV, (yg[j + 1] - yg[j]) / std::fabs(V(i, j, k)));
          lW = std::max(lW, (zg[k + 1] - zg[k]) / std::fabs(W(i, j, k)));
        }
    if (cfl < 0) return -cfl;
    const double dt_conv = std::min(cfl * lU, std::min(cfl * lV, cfl * lW));
    double dxmin = 1e300, dymin = 1e300, dzmin = 1e300;
    for (int i = 1; i < nxg; ++i) dxmin = std::min(dxmin, xg[i + 1] - xg[i]);
    for (int j = 1; j < nyg; ++j) dymin = std::min(dymin, yg[j + 1] - yg[j]);
    for (int k = 1; k < nzg; ++k) dzmin = std::min(dzmin, zg[k + 1] - zg[k]);
    const double dt_vis = std::min(cfl * dxmin * dxmin / nu, std::min(cfl * dymin * dymin / nu, cfl * dzmin * dzmin / nu));
    return std::min(std::min(dt_conv, dt_vis), 1e-1);
  }

  // src/time_integration.f90:86-213
  int step(double dt) {
    const double to = t;
    Uo.a = U.a; Vo.a = V.a; Wo.a = W.a;
    for (int s = 0; s < 3; ++s) {
      rhs_u(Fu[s]); rhs_v(Fv[s]); rhs_w(Fw[s]);
      const double* c = kRkCoef[s];
      auto update = [&](Arr& A, const Arr& Ao, const Arr* F, int i1, int j1, int k1) {
#pragma omp parallel for num_threads(nthreads)
        for (int k = 2; k <= k1; ++k)
          for (int j = 2; j <= j1; ++j)
            for (int i = 2; i <= i1; ++i) {
              if (s == 0) {
                A(i, j, k) = Ao(i, j, k) + dt * c[0] * F[0](i, j, k);
              } else if (s == 1) {
                const double du = c[0] * F[0](i, j, k) + c[1] * F[1](i, j, k);
                A(i, j, k) = Ao(i, j, k) + dt * du;
              } else {
                const double du = c[0] * F[0](i, j, k) + c[1] * F[1](i, j, k) + c[2] * F[2](i, j, k);
                A(i, j, k) = Ao(i, j, k) + dt * du;
              }
            }
      };
      update(U, Uo, Fu, nx - 1, nyg - 1, nzg - 1);
      update(V, Vo, Fv, nxg - 1, ny - 1, nzg - 1);
      update(W, Wo, Fw, nxg - 1, nyg - 1, nz - 1);
      t = to + kRkT[s] * dt;
      apply_bc();
      if (projection(s + 1, dt)) return -1;
      apply_bc();
    }
    if (x_mass_cte == 1) {   // :187-193
      const double prev = dPdx;
      double q, norm;
      mass_flow(&q, &norm);
      const double shift = Q0 - q / norm;
#pragma omp parallel for num_threads(nthreads)
      for (int k = 2; k <= nzg - 1; ++k)
        for (int j = 2; j <= nyg - 1; ++j)
          for (int i = 2; i <= nx - 1; ++i) U(i, j, k) = U(i, j, k) + shift;
      dPdx = 0.5 * (prev + shift / dt);
      apply_bc();
    }
    return 0;
  }
};

void copy_in(const double* src, std::vector<double>& dst, int n) { dst.assign(src, src + n + 1); }

}  // namespace

extern "C" {

// x, y, z, xg, yg, zg: Fortran-indexed grids (index 0 unused) of lengths
// nx+1, ny+1, nz+1, nxg+1, nyg+1, nzg+1; kxx (nxp), kzz (nzp); Dd, Dl, Du:
// Fortran-indexed Dyy diagonals of length nyg+1.  Returns null on a length
// the FFT does not factor.
void* c3d_cpu_create(int nx, int ny, int nz, const double* x, const double* y, const double* z, const double* xg,
                     const double* yg, const double* zg, const double* kxx, const double* kzz, const double* Dd,
                     const double* Dl, const double* Du, double nu, double cfl, int x_mass_cte, int nthreads) {
  Solver* s = new Solver();
  s->nx = nx; s->ny = ny; s->nz = nz;
  s->nxg = nx + 1; s->nyg = ny + 1; s->nzg = nz + 1;
  s->nxp = nx - 2; s->nzp = nz - 2;
  s->nu = nu; s->cfl = cfl; s->x_mass_cte = x_mass_cte; s->epg = 1;
  s->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();
  copy_in(x, s->x, nx); copy_in(y, s->y, ny); copy_in(z, s->z, nz);
  copy_in(xg, s->xg, s->nxg); copy_in(yg, s->yg, s->nyg); copy_in(zg, s->zg, s->nzg);
  s->kxx.assign(kxx, kxx + s->nxp);
  s->kzz.assign(kzz, kzz + s->nzp);
  copy_in(Dd, s->Dd, s->nyg); copy_in(Dl, s->Dl, s->nyg); copy_in(Du, s->Du, s->nyg);
  s->fx.init(s->nxp);
  s->fz.init(s->nzp);
  if (!s->fx.ok() || !s->fz.ok()) { delete s; return nullptr; }
  s->U.init(nx, s->nyg, s->nzg);
  s->V.init(s->nxg, ny, s->nzg);
  s->W.init(s->nxg, s->nyg, nz);
  s->P.init(s->nxg, s->nyg, s->nzg);
  s->Uo = s->U; s->Vo = s->V; s->Wo = s->W;
  for (int q = 0; q < 3; ++q) {
    s->Fu[q].init(nx - 1, s->nyg - 1, s->nzg - 1);
    s->Fv[q].init(s->nxg - 1, ny - 1, s->nzg - 1);
    s->Fw[q].init(s->nxg - 1, s->nyg - 1, nz - 1);
  }
  s->rhs.init(s->nxg - 1, s->nyg - 1, s->nzg);
  s->Pint = s->rhs;
  s->hat.assign((size_t)(s->nyg - 2) * s->nxp * s->nzp, cd(0.0, 0.0));
  return s;
}

void c3d_cpu_destroy(void* h) { delete static_cast<Solver*>(h); }

// field: 1 U, 2 V, 3 W, 4 P, 5 P_interim; data in the padded Fortran-indexed
// layout (x fastest) of the extents above
static Arr* field_of(Solver* s, int field) {
  switch (field) {
    case 1: return &s->U;
    case 2: return &s->V;
    case 3: return &s->W;
    case 4: return &s->P;
    case 5: return &s->Pint;
    default: return nullptr;
  }
}

int c3d_cpu_field_size(void* h, int field, int64_t* n) {
  Arr* a = field_of(static_cast<Solver*>(h), field);
  if (!a) return -1;
  *n = (int64_t)a->a.size();
  return 0;
}

int c3d_cpu_set_field(void* h, int field, const double* src) {
  Arr* a = field_of(static_cast<Solver*>(h), field);
  if (!a) return -1;
  std::memcpy(a->a.data(), src, sizeof(double) * a->a.size());
  return 0;
}

int c3d_cpu_get_field(void* h, int field, double* dst) {
  Arr* a = field_of(static_cast<Solver*>(h), field);
  if (!a) return -1;
  std::memcpy(dst, a->a.data(), sizeof(double) * a->a.size());
  return 0;
}

void c3d_cpu_set_scalars(void* h, double dPdx, double dPdy, double dPdz, double t, double q0) {
  Solver* s = static_cast<Solver*>(h);
  s->dPdx = dPdx; s->dPdy = dPdy; s->dPdz = dPdz; s->t = t; s->Q0 = q0;
}

double c3d_cpu_dpdx(void* h) { return static_cast<Solver*>(h)->dPdx; }

// nsteps of compute_dt + compute_time_step_RK3; 0 OK, -1 singular mode
int c3d_cpu_steps(void* h, int nsteps) {
  Solver* s = static_cast<Solver*>(h);
  for (int n = 0; n < nsteps; ++n) {
    const double dt = s->compute_dt();
    if (s->step(dt)) return -1;
  }
  return 0;
}

int c3d_cpu_threads(void* h) { return static_cast<Solver*>(h)->nthreads; }

// Known-answer hooks for the two restated third-party steps; complex values
// interleaved (re, im).  c3d_cpu_fft: in-place unnormalised DFT of n values
// (sign -1 forward, +1 inverse), -1 if n is not 2^a 3^b 5^c.
int c3d_cpu_fft(int n, double* x, int sign) {
  Fft f;
  f.init(n);
  if (!f.ok()) return -1;
  std::vector<cd> a(n), t(n);
  for (int i = 0; i < n; ++i) a[i] = cd(x[2 * i], x[2 * i + 1]);
  f.run(a.data(), t.data(), sign);
  for (int i = 0; i < n; ++i) { x[2 * i] = a[i].real(); x[2 * i + 1] = a[i].imag(); }
  return 0;
}

// c3d_cpu_zgtsv: solves the tridiagonal system (dl, d, du of n-1, n, n-1
// values) for one right-hand side b in place; returns LAPACK's info.
int c3d_cpu_zgtsv(int n, const double* dl, const double* d, const double* du, double* b) {
  std::vector<cd> L(n > 1 ? n - 1 : 1), D(n), U(n > 1 ? n - 1 : 1), B(n);
  for (int i = 0; i < n; ++i) { D[i] = cd(d[2 * i], d[2 * i + 1]); B[i] = cd(b[2 * i], b[2 * i + 1]); }
  for (int i = 0; i + 1 < n; ++i) { L[i] = cd(dl[2 * i], dl[2 * i + 1]); U[i] = cd(du[2 * i], du[2 * i + 1]); }
  const int info = zgtsv(n, L.data(), D.data(), U.data(), B.data());
  for (int i = 0; i < n; ++i) { b[2 * i] = B[i].real(); b[2 * i + 1] = B[i].imag(); }
  return info;
}

}  // extern "C"
