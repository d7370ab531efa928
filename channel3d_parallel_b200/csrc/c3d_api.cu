// extern "C" entry points of libc3d (declared in include/c3d.h).
//
// Host-side restatement of the reference's set-up (read_input_parameters,
// create_grid, initialize) and of the control flow of
// compute_time_step_RK3 (src/time_integration.f90:86-213); all field
// arithmetic runs in the kernels of k_*.cu on the handle's stream.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>

#include "c3d_internal.cuh"

namespace c3d {

static std::mutex g_mu;
static std::map<int, Handle*> g_handles;
static int g_next = 1;
static std::string g_global_error;

void set_global_error(const std::string& msg) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_global_error = msg;
}

static Handle* lookup(int id) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_handles.find(id);
  return it == g_handles.end() ? nullptr : it->second;
}

static const double kPi = 4.0 * std::atan(1.0);   // src/global.f90:30

// ---------------------------------------------------------------------------
// grids: create_grid (src/input_output.f90:140-247)
// ---------------------------------------------------------------------------
static int create_stretched(const Params& p, std::vector<double>& y, std::string& err) {
  const int ny = p.ny_global;
  const int suppy = 2;
  int n_uniform = 1;
  for (;;) {
    const int m = ny - 2 * (n_uniform - 1);
    std::vector<double> gu(m);
    double mx = 0;
    for (int i = 0; i < m; ++i) { gu[i] = (double)i; mx = gu[i] > mx ? gu[i] : mx; }
    for (int i = 0; i < m; ++i) gu[i] = 2.0 * gu[i] / mx - 1.0;
    if (p.alpha_stretch > 0.0)
      for (int i = 0; i < m; ++i) gu[i] = std::tanh(p.alpha_stretch * gu[i]) / std::tanh(p.alpha_stretch);
    const double ds_un = gu[1] - gu[0];
    const double ds_sc = p.Ly_channel * ds_un / (2.0 + (n_uniform - 1) * ds_un);
    std::vector<double> g(ny + 1, 0.0);
    for (int i = 0; i < m; ++i) g[n_uniform + i] = gu[i] * ds_sc / ds_un;
    for (int i = 2; i <= n_uniform; ++i) {
      g[ny - n_uniform + i] = g[ny - n_uniform + i - 1] + ds_sc;
      g[n_uniform - i + 1] = g[n_uniform - i + 2] - ds_sc;
    }
    const double dymin = g[2] - g[1];
    if (n_uniform * dymin >= p.min_buffer_width + (2 * suppy + 2) * dymin) {
      y.assign(ny, 0.0);
      for (int i = 0; i < ny; ++i) y[i] = g[i + 1] + 1.0;
      return 0;
    }
    ++n_uniform;
    if (2 * n_uniform >= ny - 1) { err = "Number of buffer points exceeds the total number of grid points"; return C3D_ERR_PARAM; }
  }
}

static int create_grid(const Params& p, std::vector<double>& x, std::vector<double>& y,
                       std::vector<double>& z, std::string& err) {
  const int nx = p.nx_global, ny = p.ny_global, nz = p.nz_global;
  x.resize(nx); y.resize(ny); z.resize(nz);
  for (int i = 0; i < nx; ++i) x[i] = (double)i;
  const double xd = x[nx - 2];
  for (int i = 0; i < nx; ++i) x[i] = p.Lxp * x[i] / xd;
  for (int i = 0; i < nz; ++i) z[i] = (double)i;
  const double zd = z[nz - 2];
  for (int i = 0; i < nz; ++i) z[i] = p.Lzp * z[i] / zd;
  if (p.grid_type == 0) {
    for (int i = 0; i < ny; ++i) y[i] = (double)i;
    const double mx = (double)(ny - 1);
    for (int i = 0; i < ny; ++i) y[i] = p.Ly_channel * y[i] / mx;
  } else if (p.grid_type == 1) {
    for (int i = 0; i < ny; ++i) y[i] = (double)i;
    const double mx = (double)(ny - 1);
    for (int i = 0; i < ny; ++i) y[i] = p.Ly_channel * y[i] / mx - 1.0;
    if (p.alpha_stretch > 0.0)
      for (int i = 0; i < ny; ++i) y[i] = std::tanh(p.alpha_stretch * y[i]) / std::tanh(p.alpha_stretch);
    double mn = y[0];
    for (int i = 0; i < ny; ++i) mn = y[i] < mn ? y[i] : mn;
    for (int i = 0; i < ny; ++i) y[i] = y[i] - mn;
    double mxv = y[0];
    for (int i = 0; i < ny; ++i) mxv = y[i] > mxv ? y[i] : mxv;
    for (int i = 0; i < ny; ++i) y[i] = y[i] * p.Ly_channel / mxv;
  } else if (p.grid_type == 2) {
    return create_stretched(p, y, err);
  } else {
    err = "grid_type must be 0, 1 or 2";
    return C3D_ERR_PARAM;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// metric set-up: initialize (src/initialization.f90:166-391)
// ---------------------------------------------------------------------------
static int setup_metric(Handle* h, const double* xf, const double* yf, const double* zf) {
  const Dims& d = h->d;
  const int nx = d.nx, ny = d.ny, nz = d.nz, nxg = d.nxg, nyg = d.nyg, nzg = d.nzg;
  const int nxm = nx - 1, nym = ny - 1, nzm = nz - 1;
  auto& x = h->x; auto& y = h->y; auto& z = h->z;
  x.assign(nx + 2, 0.0); y.assign(ny + 2, 0.0); z.assign(nz + 2, 0.0);
  for (int i = 1; i <= nx; ++i) x[i] = xf[i - 1];
  for (int i = 1; i <= ny; ++i) y[i] = yf[i - 1];
  for (int i = 1; i <= nz; ++i) z[i] = zf[i - 1];
  h->xm.assign(nxm + 2, 0.0); h->ym.assign(nym + 2, 0.0); h->zm.assign(nzm + 2, 0.0);
  for (int i = 1; i <= nxm; ++i) h->xm[i] = 0.5 * (x[i] + x[i + 1]);
  for (int i = 1; i <= nym; ++i) h->ym[i] = 0.5 * (y[i] + y[i + 1]);
  for (int i = 1; i <= nzm; ++i) h->zm[i] = 0.5 * (z[i] + z[i + 1]);
  auto ghost = [](const std::vector<double>& cm, const std::vector<double>& cf, int nm, int n) {
    std::vector<double> g(nm + 4, 0.0);
    for (int i = 2; i <= nm + 1; ++i) g[i] = cm[i - 1];
    g[1] = cm[1] - 2.0 * (cm[1] - cf[1]);
    g[nm + 2] = cm[nm] + 2.0 * (cf[n] - cm[nm]);
    return g;
  };
  h->xg = ghost(h->xm, x, nxm, nx);
  h->yg = ghost(h->ym, y, nym, ny);
  h->zg = ghost(h->zm, z, nzm, nz);
  const auto& xg = h->xg; const auto& yg = h->yg; const auto& zg = h->zg;
  auto minstep = [](const std::vector<double>& g, int n) {
    double m = g[2] - g[1];
    for (int i = 1; i < n; ++i) { double v = g[i + 1] - g[i]; m = v < m ? v : m; }
    return m;
  };
  h->dxmin = minstep(xg, nxg);
  h->dymin = minstep(yg, nyg);
  h->dzmin = minstep(zg, nzg);
  h->Lx = x[nx] - x[1];
  h->Ly = y[ny] - y[1];
  h->Lz = z[nz] - z[1];
  h->dx = h->dxmin;
  h->dz = h->dzmin;
  h->Lxp = h->Lx - h->dx;
  h->Lzp = h->Lz - h->dz;
  // modified wavenumbers, :289-305
  const int nxp = d.Nx, nzp = d.Nz;
  h->kxx.assign(nxp, 0.0);
  h->kzz.assign(nzp, 0.0);
  const int cx = (int)std::ceil((float)nxp / 2.0);
  const int cz = (int)std::ceil((float)nzp / 2.0);
  for (int i = 0; i <= cx && i < nxp; ++i)
    h->kxx[i] = 2.0 * (std::cos(2.0 * kPi * (double)i / (double)nxp) - 1.0) / (h->dx * h->dx);
  for (int i = cx + 1; i < nxp; ++i)
    h->kxx[i] = 2.0 * (std::cos(2.0 * kPi * (double)(-nxp + i) / (double)nxp) - 1.0) / (h->dx * h->dx);
  for (int k = 0; k <= cz && k < nzp; ++k)
    h->kzz[k] = 2.0 * (std::cos(2.0 * kPi * (double)k / (double)nzp) - 1.0) / (h->dz * h->dz);
  for (int k = cz + 1; k < nzp; ++k)
    h->kzz[k] = 2.0 * (std::cos(2.0 * kPi * (double)(-nzp + k) / (double)nzp) - 1.0) / (h->dz * h->dz);
  // Dyy with Neumann rows, :352-383
  h->Dd.assign(nyg + 1, 0.0); h->Dl.assign(nyg + 1, 0.0); h->Du.assign(nyg + 1, 0.0);
  auto abc = [&](int j, double& a, double& b, double& c) {
    a = 1.0 / (y[j] - y[j - 1]) / (yg[j + 1] - yg[j]);
    b = 1.0 / (y[j] - y[j - 1]) * (-1.0 / (yg[j + 1] - yg[j]) - 1.0 / (yg[j] - yg[j - 1]));
    c = 1.0 / (y[j] - y[j - 1]) / (yg[j] - yg[j - 1]);
  };
  for (int j = 3; j <= nyg - 2; ++j) {
    double a, b, c;
    abc(j, a, b, c);
    h->Du[j] = a; h->Dl[j] = c; h->Dd[j] = b;
  }
  {
    double a, b, c;
    abc(2, a, b, c);
    h->Dd[2] = b + c;
    h->Du[2] = a;
    abc(nyg - 1, a, b, c);
    h->Dd[nyg - 1] = a + b;
    h->Dl[nyg - 1] = c;
  }
  // kernel coefficient tables (Fortran-indexed)
  const double nu = h->p.nu;
  const int LX = nxg + 2, LY = nyg + 2, LZ = nzg + 2;
  std::vector<double> buf;
  std::vector<std::pair<const double**, int64_t>> slots;
  auto add = [&](std::vector<double> v, const double** slot) {
    slots.push_back({slot, (int64_t)buf.size()});
    buf.insert(buf.end(), v.begin(), v.end());
  };
  std::vector<double> rdx(LX, 0), rdxg(LX, 0), cxpF(LX, 0), cxmF(LX, 0), cxpC(LX, 0), cxmC(LX, 0);
  for (int i = 2; i <= nxg - 1; ++i) rdx[i] = 1.0 / (x[i] - x[i - 1]);
  for (int i = 1; i <= nxg - 1; ++i) rdxg[i] = 1.0 / (xg[i + 1] - xg[i]);
  for (int i = 2; i <= nx - 1; ++i) {
    cxpF[i] = nu / ((x[i + 1] - x[i]) * (xg[i + 1] - xg[i]));
    cxmF[i] = nu / ((x[i] - x[i - 1]) * (xg[i + 1] - xg[i]));
  }
  for (int i = 2; i <= nxg - 1; ++i) {
    cxpC[i] = nu / ((xg[i + 1] - xg[i]) * (x[i] - x[i - 1]));
    cxmC[i] = nu / ((xg[i] - xg[i - 1]) * (x[i] - x[i - 1]));
  }
  std::vector<double> rdy(LY, 0), rdyg(LY, 0), cypC(LY, 0), cymC(LY, 0), cypF(LY, 0), cymF(LY, 0), wq(LY, 0),
      wqv(LY, 0);
  for (int j = 2; j <= ny; ++j) rdy[j] = 1.0 / (y[j] - y[j - 1]);
  for (int j = 1; j <= nyg - 1; ++j) rdyg[j] = 1.0 / (yg[j + 1] - yg[j]);
  for (int j = 2; j <= nyg - 1; ++j) {
    cypC[j] = nu / ((yg[j + 1] - yg[j]) * (y[j] - y[j - 1]));
    cymC[j] = nu / ((yg[j] - yg[j - 1]) * (y[j] - y[j - 1]));
  }
  for (int j = 2; j <= ny - 1; ++j) {
    cypF[j] = nu / ((y[j + 1] - y[j]) * (yg[j + 1] - yg[j]));
    cymF[j] = nu / ((y[j] - y[j - 1]) * (yg[j + 1] - yg[j]));
  }
  for (int j = 3; j <= nyg - 1; ++j) wq[j] = 0.5 * (yg[j] - yg[j - 1]);
  for (int j = 2; j <= ny; ++j) wqv[j] = 0.5 * (y[j] - y[j - 1]);
  std::vector<double> cqu(LY, 0);
  for (int j = 2; j <= nyg - 1; ++j) cqu[j] = wq[j] + wq[j + 1];
  {
    // norm of compute_mean_mass_flow_U (src/mass_flow.f90:24-53): rows
    // j = 3..nyg-1 and k = 2..nzg-1, nx-2 points each, weight 2 wq(j)
    double sw = 0.0;
    for (int j = 3; j <= nyg - 1; ++j) sw += 2.0 * wq[j];
    h->norm_u = sw * (double)(nx - 2) * (double)(nzg - 2);
    double dev = 0.0;
    for (int i = 2; i <= nx - 1; ++i) dev = std::max(dev, std::fabs(rdxg[i] - rdxg[2]));
    h->x_uniform = dev <= 1e-9 * std::fabs(rdxg[2]);
  }
  std::vector<double> rdz(LZ, 0), rdzg(LZ, 0), czpC(LZ, 0), czmC(LZ, 0), czpF(LZ, 0), czmF(LZ, 0);
  for (int k = 2; k <= nz; ++k) rdz[k] = 1.0 / (z[k] - z[k - 1]);
  for (int k = 1; k <= nzg - 1; ++k) rdzg[k] = 1.0 / (zg[k + 1] - zg[k]);
  for (int k = 2; k <= nzg - 1; ++k) {
    czpC[k] = nu / ((zg[k + 1] - zg[k]) * (z[k] - z[k - 1]));
    czmC[k] = nu / ((zg[k] - zg[k - 1]) * (z[k] - z[k - 1]));
  }
  for (int k = 2; k <= nz - 1; ++k) {
    czpF[k] = nu / ((z[k + 1] - z[k]) * (zg[k + 1] - zg[k]));
    czmF[k] = nu / ((z[k] - z[k - 1]) * (zg[k + 1] - zg[k]));
  }
  Metric& m = h->m;
  add(rdx, &m.rdx); add(rdxg, &m.rdxg); add(cxpF, &m.cxpF); add(cxmF, &m.cxmF);
  add(cxpC, &m.cxpC); add(cxmC, &m.cxmC);
  add(rdy, &m.rdy); add(rdyg, &m.rdyg); add(cypC, &m.cypC); add(cymC, &m.cymC);
  add(cypF, &m.cypF); add(cymF, &m.cymF); add(wq, &m.wq); add(wqv, &m.wqv); add(cqu, &m.cqu);
  add(rdz, &m.rdz); add(rdzg, &m.rdzg); add(czpC, &m.czpC); add(czmC, &m.czmC);
  add(czpF, &m.czpF); add(czmF, &m.czmF);
  if (h->metric_buf == nullptr) {
    int rc = dev_alloc(h, &h->metric_buf, (int64_t)buf.size());
    if (rc) return rc;
  }
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->metric_buf, buf.data(), sizeof(double) * buf.size(),
                                  cudaMemcpyHostToDevice, h->stream));
  for (auto& s : slots) *s.first = h->metric_buf + s.second;
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

static void free_handle(Handle* h) {
  if (!h) return;
  if (h->device >= 0) cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  ib_free(h);
  mlp_free(h);
  mixed_free(h);
  if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
  for (void* p : h->allocations) cudaFree(p);
  if (h->h2d) cudaStreamSynchronize(h->h2d);
  if (h->d2h) cudaStreamSynchronize(h->d2h);
  for (cudaEvent_t e : h->ev_slab) cudaEventDestroy(e);
  if (h->ev_up) cudaEventDestroy(h->ev_up);
  if (h->ev_done) cudaEventDestroy(h->ev_done);
  if (h->h2d) cudaStreamDestroy(h->h2d);
  if (h->d2h) cudaStreamDestroy(h->d2h);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

static int build(Handle* h, const std::vector<double>* xg_in = nullptr) {
  (void)xg_in;
  Params& p = h->p;
  if (p.nx_global < 6 || p.nz_global < 6 || p.ny_global < 5) {
    h->last_error = "grid too small: need nx_global, nz_global >= 6 and ny_global >= 5";
    return C3D_ERR_PARAM;
  }
  if (p.nx_global % 2 || p.nz_global % 2) {   // src/initialization.f90:46-47
    h->last_error = p.nx_global % 2 ? "Error: nx must be even" : "Error: nz must be even";
    return C3D_ERR_PARAM;
  }
  if (!(p.nu > 0.0)) { h->last_error = "nu must be positive"; return C3D_ERR_PARAM; }
  Dims& d = h->d;
  d.nx = p.nx_global; d.ny = p.ny_global; d.nz = p.nz_global;
  d.nxg = d.nx + 1; d.nyg = d.ny + 1; d.nzg = d.nz + 1;
  d.Nx = d.nx - 2; d.Ny = d.ny - 1; d.Nz = d.nz - 2;
  d.nkx = d.Nx / 2 + 1;
  d.nkzs = d.Nz / 2 + 1;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    h->last_error = "no CUDA device visible";
    return C3D_ERR_NO_DEVICE;
  }
  C3D_CUDA_TRY(h, cudaGetDevice(&h->device));
  C3D_CUDA_TRY(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  C3D_CUDA_TRY(h, cudaEventCreate(&h->ev0));
  C3D_CUDA_TRY(h, cudaEventCreate(&h->ev1));
  std::vector<double> x, y, z;
  std::string err;
  int rc = create_grid(p, x, y, z, err);
  if (rc) { h->last_error = err; return rc; }
  if ((rc = setup_metric(h, x.data(), y.data(), z.data()))) return rc;
  // fields
  if ((rc = dev_alloc(h, &h->U, sizeU(d)))) return rc;
  if ((rc = dev_alloc(h, &h->V, sizeV(d)))) return rc;
  if ((rc = dev_alloc(h, &h->W, sizeW(d)))) return rc;
  if ((rc = dev_alloc(h, &h->P, sizeP(d)))) return rc;
  if ((rc = dev_alloc(h, &h->Us, sizeU(d)))) return rc;
  if ((rc = dev_alloc(h, &h->Vs, sizeV(d)))) return rc;
  if ((rc = dev_alloc(h, &h->Ws, sizeW(d)))) return rc;
  if ((rc = dev_alloc(h, &h->Gu, sizeU(d)))) return rc;
  if ((rc = dev_alloc(h, &h->Gv, sizeV(d)))) return rc;
  if ((rc = dev_alloc(h, &h->Gw, sizeW(d)))) return rc;
  if ((rc = dev_alloc(h, &h->rhs_p, sizeR(d)))) return rc;
  if ((rc = dev_alloc(h, &h->P_interim, sizeR(d)))) return rc;
  if ((rc = dev_alloc(h, &h->phi1, sizeR(d)))) return rc;
  if ((rc = dev_alloc(h, &h->rhsU, (int64_t)(d.nx - 2) * (d.nyg - 2) * (d.nzg - 2)))) return rc;
  if ((rc = dev_alloc(h, &h->rhsV, (int64_t)(d.nxg - 2) * (d.ny - 2) * (d.nzg - 2)))) return rc;
  if ((rc = dev_alloc(h, &h->rhsW, (int64_t)(d.nxg - 2) * (d.nyg - 2) * (d.nz - 2)))) return rc;
  h->red_len = 4 * 148 * 4 + d.nxg + d.nyg + d.nzg + 64;
  if ((rc = dev_alloc(h, &h->red, h->red_len))) return rc;
  if ((rc = dev_alloc(h, &h->sc, 1))) return rc;
  if ((rc = poisson_setup(h))) return rc;
  if ((rc = rhs_setup(h))) return rc;
  // module scalars
  h->t = p.t_init;
  h->dPdx = p.dPdx;
  h->dPdz = p.dPdz;
  h->dPdy = 0.0;
  h->Qflow_x_0 = p.Qflow_x_0;
  h->Qflow_z_0 = p.Qflow_z_0;
  h->dt = p.CFL < 0 ? -p.CFL : 0.0;
  DevScalars s{};
  s.dPdx = h->dPdx; s.dPdy = h->dPdy; s.dPdz = h->dPdz;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->sc, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  if (p.body_type != "none") {
    if ((rc = ib_create(h))) return rc;
  }
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

static int create_from_params(const Params& p, int* handle) {
  Handle* h = new Handle();
  h->p = p;
  int rc = build(h);
  if (rc) {
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_global_error = h->last_error;
    }
    free_handle(h);
    return rc;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  int id = g_next++;
  g_handles[id] = h;
  *handle = id;
  return 0;
}

// ---------------------------------------------------------------------------
// field table
// ---------------------------------------------------------------------------
struct FieldRef {
  double* ptr;
  int64_t lb[3];
  int64_t n[3];
};

static bool field_ref(Handle* h, int id, FieldRef& f) {
  const Dims& d = h->d;
  auto set = [&](double* p, int l1, int l2, int l3, int64_t n1, int64_t n2, int64_t n3) {
    f.ptr = p; f.lb[0] = l1; f.lb[1] = l2; f.lb[2] = l3; f.n[0] = n1; f.n[1] = n2; f.n[2] = n3;
    return p != nullptr;
  };
  switch (id) {
    case C3D_FIELD_U: return set(h->U, 1, 1, 1, d.nx, d.nyg, d.nzg);
    case C3D_FIELD_V: return set(h->V, 1, 1, 1, d.nxg, d.ny, d.nzg);
    case C3D_FIELD_W: return set(h->W, 1, 1, 1, d.nxg, d.nyg, d.nz);
    case C3D_FIELD_P: return set(h->P, 1, 1, 1, d.nxg, d.nyg, d.nzg);
    case C3D_FIELD_RHS_P: return set(h->rhs_p, 2, 2, 2, d.nxg - 2, d.nyg - 2, d.nzg - 1);
    case C3D_FIELD_P_INTERIM: return set(h->P_interim, 2, 2, 2, d.nxg - 2, d.nyg - 2, d.nzg - 1);
    case C3D_FIELD_RHS_U: return set(h->rhsU, 2, 2, 2, d.nx - 2, d.nyg - 2, d.nzg - 2);
    case C3D_FIELD_RHS_V: return set(h->rhsV, 2, 2, 2, d.nxg - 2, d.ny - 2, d.nzg - 2);
    case C3D_FIELD_RHS_W: return set(h->rhsW, 2, 2, 2, d.nxg - 2, d.nyg - 2, d.nz - 2);
    case C3D_FIELD_U_WORK: return set(h->Us, 1, 1, 1, d.nx, d.nyg, d.nzg);
    case C3D_FIELD_V_WORK: return set(h->Vs, 1, 1, 1, d.nxg, d.ny, d.nzg);
    case C3D_FIELD_W_WORK: return set(h->Ws, 1, 1, 1, d.nxg, d.nyg, d.nz);
    case C3D_FIELD_U_REG: case C3D_FIELD_HU_INTERIOR:
      return set(ib_field_ptr(h, id), 1, 1, 1, d.nx, d.nyg, d.nzg);
    case C3D_FIELD_V_REG: case C3D_FIELD_HV_INTERIOR:
      return set(ib_field_ptr(h, id), 1, 1, 1, d.nxg, d.ny, d.nzg);
    case C3D_FIELD_W_REG: case C3D_FIELD_HW_INTERIOR:
      return set(ib_field_ptr(h, id), 1, 1, 1, d.nxg, d.nyg, d.nz);
    case C3D_FIELD_HC_EXTERIOR:
      return set(ib_field_ptr(h, id), 2, 2, 2, d.nxg - 2, d.nyg - 2, d.nzg - 1);
    default: break;
  }
  int64_t len = 0;
  double* mp = ib_marker_ptr(h, id, &len);
  if (mp) return set(mp, 1, 1, 1, len, 1, 1);
  return false;
}

static int transfer(Handle* h, int id, double* host, const int64_t lb[3], const int64_t ub[3], bool up) {
  FieldRef f{};
  if (!field_ref(h, id, f)) {
    h->last_error = "unknown or unavailable field id " + std::to_string(id);
    return C3D_ERR_PARAM;
  }
  if (host == nullptr) { h->last_error = "null host buffer"; return C3D_ERR_PARAM; }
  int64_t o[3], c[3];
  for (int a = 0; a < 3; ++a) {
    o[a] = lb[a] - f.lb[a];
    c[a] = ub[a] - lb[a] + 1;
    if (o[a] < 0 || c[a] <= 0 || o[a] + c[a] > f.n[a]) {
      std::ostringstream s;
      s << "box out of range for field " << id << " in dim " << a + 1 << ": [" << lb[a] << "," << ub[a]
        << "] vs [" << f.lb[a] << "," << f.lb[a] + f.n[a] - 1 << "]";
      h->last_error = s.str();
      return C3D_ERR_PARAM;
    }
  }
  cudaStream_t s = h->stream;
  const size_t es = sizeof(double);
  if (c[0] == f.n[0] && c[1] == f.n[1]) {
    double* dev = f.ptr + o[2] * f.n[0] * f.n[1];
    const size_t bytes = (size_t)(c[0] * c[1] * c[2]) * es;
    if (up) C3D_CUDA_TRY(h, cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s));
    else C3D_CUDA_TRY(h, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
  } else {
    for (int64_t k = 0; k < c[2]; ++k) {
      double* dev = f.ptr + o[0] + f.n[0] * (o[1] + f.n[1] * (o[2] + k));
      double* hp = host + k * c[0] * c[1];
      if (up)
        C3D_CUDA_TRY(h, cudaMemcpy2DAsync(dev, f.n[0] * es, hp, c[0] * es, c[0] * es, c[1],
                                          cudaMemcpyHostToDevice, s));
      else
        C3D_CUDA_TRY(h, cudaMemcpy2DAsync(hp, c[0] * es, dev, f.n[0] * es, c[0] * es, c[1],
                                          cudaMemcpyDeviceToHost, s));
    }
  }
  C3D_CUDA_TRY(h, cudaStreamSynchronize(s));
  return 0;
}

static int sync_scalars_to_device(Handle* h) {
  DevScalars s{};
  C3D_CUDA_TRY(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  s.dPdx = h->dPdx; s.dPdy = h->dPdy; s.dPdz = h->dPdz;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->sc, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

static int sync_scalars_from_device(Handle* h) {
  DevScalars s{};
  C3D_CUDA_TRY(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->dPdx = s.dPdx; h->dPdy = s.dPdy; h->dPdz = s.dPdz;
  if (s.err) {
    h->last_error = "a kernel gave up waiting for an asynchronous copy (device state is suspect)";
    return C3D_ERR_CUDA;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// one RK3 step, src/time_integration.f90:86-213
// ---------------------------------------------------------------------------
static int enqueue_step(Handle* h, double dt, double to) {
  static const double rk_t[3] = {8.0 / 15.0, 2.0 / 3.0, 1.0};
  int rc, warn = 0;
  // The constant x mass flow (:187-193) inside the last stage: over the
  // periodic, uniformly spaced x grid the bulk flux of d(phi)/dx telescopes
  // to zero, so the flux of the projected u is that of U* (up to rounding);
  // the stage-3 divergence kernel reduces it and the projection adds the shift.
  const bool xflux = h->p.x_mass_cte == 1 && h->ib == nullptr && h->x_uniform && !h->write_pinterim;
  for (int s = 1; s <= 3; ++s) {
    const bool fx = xflux && s == 3;
    if ((rc = launch_rhs_stage(h, s, dt))) return rc;
    // the projection reads the ghosts of U*, V*, W* as the boundary
    // conditions define them; the immersed-boundary operators need them set
    if (h->ib && (rc = launch_fill_ghosts3(h, h->Us, h->Vs, h->Ws))) return rc;
    const double ts = to + rk_t[s - 1] * dt;
    if (h->ib && ib_moving(h)) {                         // :111-115
      if ((rc = ib_setup_geometry(h, ts))) return rc;
      if ((rc = ib_setup_operators(h))) return rc;
      if ((rc = ib_heaviside(h))) return rc;
    }
    if ((rc = launch_projection_step(h, s, dt, fx ? &h->sc->shift : nullptr))) return rc;   // :117-118, :123
    if (h->ib) {
      // a Schur solve that reached cg_max_iter is a warning: the reference
      // stops iterating and completes the step (src/projection.f90:60)
      rc = ib_projection(h, dt, s);                           // :119-122
      if (rc < 0) return rc;
      if (rc > 0) warn = rc;
    }
  }
  if ((h->p.x_mass_cte == 1 && !xflux) || h->p.y_mass_cte == 1 || h->p.z_mass_cte == 1) {   // :187-211
    if ((rc = launch_massflow_correction(h, dt, false, xflux))) return rc;
  }
  return warn;
}

// one explicit Euler step, src/time_integration.f90:25-81: rk_step = 3 (no
// P side effect), the non-IB projection only (the reference's Euler never
// calls the IB projection), x and y constant-flux corrections
static int enqueue_euler_step(Handle* h, double dt) {
  int rc;
  if ((rc = launch_rhs_euler(h, dt))) return rc;                // :34-52
  if (h->ib && (rc = launch_fill_ghosts3(h, h->Us, h->Vs, h->Ws))) return rc;
  if ((rc = launch_projection_step(h, 3, dt))) return rc;       // :58-61
  if (h->p.x_mass_cte == 1 || h->p.y_mass_cte == 1) {           // :65-78
    if ((rc = launch_massflow_correction(h, dt, true))) return rc;
  }
  return 0;
}

static int run_steps(Handle* h, int nsteps, bool euler = false) {
  int rc, warn = 0;
  C3D_CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
  for (int n = 0; n < nsteps; ++n) {
    double dt;
    if ((rc = compute_dt_cfl(h, &dt))) return rc;   // compute_dt, app/main.f90:105
    h->dt = dt;
    const double to = h->t;
    if (euler) {
      if ((rc = enqueue_euler_step(h, dt))) return rc;
      h->t = to + dt;
      h->stats.steps++;
      continue;
    }
    const bool graphable = h->use_graph && h->ib == nullptr;
    if (graphable) {
      if (h->step_exec == nullptr || h->graph_dt != dt) {
        if (h->step_exec) { cudaGraphExecDestroy(h->step_exec); h->step_exec = nullptr; }
        cudaGraph_t g = nullptr;
        const int64_t l0 = h->launches, p0 = h->stats.poisson_solves;
        C3D_CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_step(h, dt, to);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) { h->last_error = std::string("graph capture: ") + cudaGetErrorString(e); return C3D_ERR_CUDA; }
        e = cudaGraphInstantiate(&h->step_exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { h->last_error = std::string("graph instantiate: ") + cudaGetErrorString(e); return C3D_ERR_CUDA; }
        h->graph_dt = dt;
        h->graph_launches = h->launches - l0;
        h->graph_solves = h->stats.poisson_solves - p0;
        h->launches = l0;
        h->stats.poisson_solves = p0;
      }
      C3D_CUDA_TRY(h, cudaGraphLaunch(h->step_exec, h->stream));
      h->launches += h->graph_launches;
      h->stats.poisson_solves += h->graph_solves;
      h->P_pending = true;
      h->P_pending_dt = dt;
    } else {
      rc = enqueue_step(h, dt, to);
      if (rc < 0) return rc;
      if (rc > 0) warn = rc;
    }
    h->t = to + 1.0 * dt;
    h->stats.steps++;
  }
  C3D_CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
  C3D_CUDA_TRY(h, cudaEventSynchronize(h->ev1));
  float ms = 0;
  C3D_CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->last_step_ms = nsteps > 0 ? ms / nsteps : 0.0;
  C3D_CUDA_TRY(h, cudaGetLastError());
  if ((rc = sync_scalars_from_device(h))) return rc;
  if (warn) h->last_error = "a Schur solve stopped at cg_max_iter before reaching cg_tol";
  return warn;
}

Handle* lookup_handle(int id) { return lookup(id); }

// ---- stepping with u, v, w resident in host arrays -----------------------
// Every step uploads the three arrays, advances one RK3 step and downloads
// them back into the same arrays.  The copies go in slabs of kHostSlab bytes
// on two copy streams: the upload of a slab for step n+1 waits only for the
// download of that slab in step n, so one slab's download and the previous
// slab's upload use the two directions of the host link at once.  The step
// itself waits for all uploads, and the downloads for the step.
constexpr size_t kHostSlab = size_t(4) << 20;

static int host_copy_setup(Handle* h, size_t nslab) {
  if (!h->h2d) C3D_CUDA_TRY(h, cudaStreamCreateWithFlags(&h->h2d, cudaStreamNonBlocking));
  if (!h->d2h) C3D_CUDA_TRY(h, cudaStreamCreateWithFlags(&h->d2h, cudaStreamNonBlocking));
  if (!h->ev_up) C3D_CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_up, cudaEventDisableTiming));
  if (!h->ev_done) C3D_CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_done, cudaEventDisableTiming));
  while (h->ev_slab.size() < nslab) {
    cudaEvent_t e = nullptr;
    C3D_CUDA_TRY(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    h->ev_slab.push_back(e);
  }
  return 0;
}

static int run_steps_host(Handle* h, double* const host[3], int nsteps) {
  const int ids[3] = {C3D_FIELD_U, C3D_FIELD_V, C3D_FIELD_W};
  double* dev[3];
  size_t bytes[3], nsl[3], total = 0;
  for (int a = 0; a < 3; ++a) {
    FieldRef f{};
    if (!field_ref(h, ids[a], f)) { h->last_error = "velocity field not allocated"; return C3D_ERR_PARAM; }
    dev[a] = f.ptr;
    bytes[a] = (size_t)(f.n[0] * f.n[1] * f.n[2]) * sizeof(double);
    nsl[a] = (bytes[a] + kHostSlab - 1) / kHostSlab;
    total += nsl[a];
  }
  int rc = host_copy_setup(h, total);
  if (rc) return rc;
  // the first uploads follow whatever the caller queued on the step stream
  C3D_CUDA_TRY(h, cudaEventRecord(h->ev_done, h->stream));
  C3D_CUDA_TRY(h, cudaStreamWaitEvent(h->h2d, h->ev_done, 0));
  int warn = 0;
  for (int n = 0; n < nsteps && rc >= 0; ++n) {
    size_t e = 0;
    for (int a = 0; a < 3; ++a)
      for (size_t s = 0; s < nsl[a]; ++s) {
        const size_t off = s * kHostSlab, len = std::min(kHostSlab, bytes[a] - off);
        if (n > 0) C3D_CUDA_TRY(h, cudaStreamWaitEvent(h->h2d, h->ev_slab[e + s], 0));
        C3D_CUDA_TRY(h, cudaMemcpyAsync(reinterpret_cast<char*>(dev[a]) + off,
                                        reinterpret_cast<const char*>(host[a]) + off, len,
                                        cudaMemcpyHostToDevice, h->h2d));
      }
    C3D_CUDA_TRY(h, cudaEventRecord(h->ev_up, h->h2d));
    C3D_CUDA_TRY(h, cudaStreamWaitEvent(h->stream, h->ev_up, 0));
    rc = run_steps(h, 1);
    if (rc > 0) warn = rc;
    if (rc < 0) break;
    C3D_CUDA_TRY(h, cudaEventRecord(h->ev_done, h->stream));
    C3D_CUDA_TRY(h, cudaStreamWaitEvent(h->d2h, h->ev_done, 0));
    e = 0;
    for (int a = 0; a < 3; ++a) {
      for (size_t s = 0; s < nsl[a]; ++s) {
        const size_t off = s * kHostSlab, len = std::min(kHostSlab, bytes[a] - off);
        C3D_CUDA_TRY(h, cudaMemcpyAsync(reinterpret_cast<char*>(host[a]) + off,
                                        reinterpret_cast<const char*>(dev[a]) + off, len,
                                        cudaMemcpyDeviceToHost, h->d2h));
        C3D_CUDA_TRY(h, cudaEventRecord(h->ev_slab[e + s], h->d2h));
      }
      e += nsl[a];
    }
  }
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->h2d));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->d2h));
  return rc < 0 ? rc : warn;
}

}  // namespace c3d

using namespace c3d;

#define GET_HANDLE(id)                                      \
  Handle* h = lookup(id);                                   \
  if (!h) return C3D_ERR_HANDLE;                            \
  cudaSetDevice(h->device);

#define RET(h, expr)                  \
  do {                                \
    int _rc = (expr);                 \
    (h)->stats.status = _rc;          \
    return _rc;                       \
  } while (0)

extern "C" {

int c3d_create_from_text(const char* text, int* handle) {
  if (!text || !handle) return C3D_ERR_PARAM;
  Params p;
  std::string err;
  int rc = parse_namelist(text, p, err);
  if (rc) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_global_error = err;
    return rc;
  }
  return create_from_params(p, handle);
}

int c3d_create(const char* path, int* handle) {
  if (!path || !handle) return C3D_ERR_PARAM;
  std::ifstream f(path);
  if (!f) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_global_error = std::string("cannot open namelist file ") + path;
    return C3D_ERR_IO;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  return c3d_create_from_text(ss.str().c_str(), handle);
}

int c3d_destroy(int id) {
  Handle* h = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_handles.find(id);
    if (it == g_handles.end()) return C3D_ERR_HANDLE;
    h = it->second;
    g_handles.erase(it);
  }
  free_handle(h);
  return 0;
}

const char* c3d_last_error(int id) {
  Handle* h = lookup(id);
  if (!h) return g_global_error.c_str();
  return h->last_error.c_str();
}

int c3d_get_dims(int id, c3d_dims* out) {
  GET_HANDLE(id);
  if (!out) return C3D_ERR_PARAM;
  const Dims& d = h->d;
  out->nx = d.nx; out->ny = d.ny; out->nz = d.nz;
  out->nxg = d.nxg; out->nyg = d.nyg; out->nzg = d.nzg;
  out->nxp = d.Nx; out->nzp = d.Nz; out->nym = d.Ny;
  out->nb = ib_nb(h);
  return 0;
}

int c3d_set_grid(int id, const double* x, const double* y, const double* z) {
  GET_HANDLE(id);
  if (!x || !y || !z) return C3D_ERR_PARAM;
  int rc = setup_metric(h, x, y, z);
  if (rc) RET(h, rc);
  // rebuild the spectral tables for the new spacings
  rc = poisson_setup(h);
  if (rc) RET(h, rc);
  if (h->step_exec) { cudaGraphExecDestroy(h->step_exec); h->step_exec = nullptr; }
  if (h->ib) {
    ib_grids_changed(h);
    rc = ib_setup_geometry(h, h->t);
    if (!rc) rc = ib_setup_operators(h);
  }
  RET(h, rc);
}

int c3d_get_grid(int id, double* x, double* y, double* z, double* xg, double* yg, double* zg) {
  GET_HANDLE(id);
  const Dims& d = h->d;
  if (x) std::memcpy(x, h->x.data() + 1, sizeof(double) * d.nx);
  if (y) std::memcpy(y, h->y.data() + 1, sizeof(double) * d.ny);
  if (z) std::memcpy(z, h->z.data() + 1, sizeof(double) * d.nz);
  if (xg) std::memcpy(xg, h->xg.data() + 1, sizeof(double) * d.nxg);
  if (yg) std::memcpy(yg, h->yg.data() + 1, sizeof(double) * d.nyg);
  if (zg) std::memcpy(zg, h->zg.data() + 1, sizeof(double) * d.nzg);
  return 0;
}

int c3d_upload(int id, int field, const double* host, const int64_t lb[3], const int64_t ub[3]) {
  GET_HANDLE(id);
  if (!lb || !ub) return C3D_ERR_PARAM;
  RET(h, transfer(h, field, const_cast<double*>(host), lb, ub, true));
}

int c3d_download(int id, int field, double* host, const int64_t lb[3], const int64_t ub[3]) {
  GET_HANDLE(id);
  if (!lb || !ub) return C3D_ERR_PARAM;
  if (field == C3D_FIELD_P) {
    int rc = rebuild_pressure(h);
    if (rc) RET(h, rc);
  }
  RET(h, transfer(h, field, host, lb, ub, false));
}

int c3d_set_scalars(int id, double dPdx, double dPdy, double dPdz, double t, double q0) {
  GET_HANDLE(id);
  h->dPdx = dPdx; h->dPdy = dPdy; h->dPdz = dPdz; h->t = t; h->Qflow_x_0 = q0;
  if (h->step_exec) { cudaGraphExecDestroy(h->step_exec); h->step_exec = nullptr; }
  RET(h, sync_scalars_to_device(h));
}

int c3d_synchronize(int id) {
  GET_HANDLE(id);
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

int c3d_time_step_rk3(int id, int nsteps) {
  GET_HANDLE(id);
  if (nsteps < 0) return C3D_ERR_PARAM;
  RET(h, run_steps(h, nsteps));
}

int c3d_time_step_rk3_host(int id, double* U, double* V, double* W, int nsteps) {
  GET_HANDLE(id);
  if (nsteps < 0 || !U || !V || !W) return C3D_ERR_PARAM;
  double* const host[3] = {U, V, W};
  RET(h, run_steps_host(h, host, nsteps));
}

int c3d_time_step_euler(int id, int nsteps) {
  GET_HANDLE(id);
  if (nsteps < 0) return C3D_ERR_PARAM;
  RET(h, run_steps(h, nsteps, true));
}

int c3d_compute_dt(int id, double* dt) {
  GET_HANDLE(id);
  if (!dt) return C3D_ERR_PARAM;
  int rc = compute_dt_cfl(h, dt);
  if (!rc) h->dt = *dt;
  RET(h, rc);
}

int c3d_compute_mean_mass_flow_u(int id, double* q) {
  GET_HANDLE(id);
  if (!q) return C3D_ERR_PARAM;
  RET(h, massflow(h, 0, false, q));
}

int c3d_compute_mean_mass_flow_v(int id, double* q) {
  GET_HANDLE(id);
  if (!q) return C3D_ERR_PARAM;
  RET(h, massflow(h, 1, false, q));
}

int c3d_compute_mean_mass_flow_w(int id, double* q) {
  GET_HANDLE(id);
  if (!q) return C3D_ERR_PARAM;
  RET(h, massflow(h, 2, false, q));
}

int c3d_set_flow_targets(int id, double qx, double qy, double qz) {
  GET_HANDLE(id);
  h->Qflow_x_0 = qx; h->Qflow_y_0 = qy; h->Qflow_z_0 = qz;
  if (h->step_exec) { cudaGraphExecDestroy(h->step_exec); h->step_exec = nullptr; }
  RET(h, 0);
}

int c3d_compute_rhs_u(int id) { GET_HANDLE(id); RET(h, launch_rhs_only(h, 1)); }
int c3d_compute_rhs_v(int id) { GET_HANDLE(id); RET(h, launch_rhs_only(h, 2)); }
int c3d_compute_rhs_w(int id) { GET_HANDLE(id); RET(h, launch_rhs_only(h, 3)); }

int c3d_divergence(int id) {
  GET_HANDLE(id);
  RET(h, launch_divergence(h, h->U, h->V, h->W, h->rhs_p));
}

int c3d_solve_poisson_equation(int id, int rk_step) {
  GET_HANDLE(id);
  RET(h, launch_poisson_solve(h, h->rhs_p, rk_step, h->dt));
}

int c3d_compute_non_IB_projection(int id, int rk_step) {
  GET_HANDLE(id);
  const Dims& d = h->d;
  const double dt = h->dt;
  if (!(dt > 0)) { h->last_error = "dt is not set (call c3d_compute_dt)"; RET(h, C3D_ERR_PARAM); }
  cudaStream_t s = h->stream;
  // U_interim = U (src/projection.f90:26-28)
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->Us, h->U, sizeU(d) * 8, cudaMemcpyDeviceToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->Vs, h->V, sizeV(d) * 8, cudaMemcpyDeviceToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->Ws, h->W, sizeW(d) * 8, cudaMemcpyDeviceToDevice, s));
  int rc = launch_divergence(h, h->U, h->V, h->W, h->rhs_p);
  if (rc) RET(h, rc);
  rc = launch_poisson_solve(h, h->rhs_p, rk_step, dt);
  if (rc) RET(h, rc);
  h->write_pinterim = true;
  rc = launch_gradient_subtract(h, h->Us, h->Vs, h->Ws, h->rhs_p, dt, h->U, h->V, h->W);
  h->write_pinterim = false;
  if (rc) RET(h, rc);
  C3D_CUDA_TRY(h, cudaStreamSynchronize(s));
  RET(h, 0);
}

int c3d_apply_boundary_conditions(int id, int which) {
  GET_HANDLE(id);
  if (which == 0) RET(h, launch_fill_ghosts3(h, h->U, h->V, h->W));
  if (which == 2) RET(h, launch_fill_ghosts3(h, h->Us, h->Vs, h->Ws));
  if (which == 1) {
    FieldRef a{}, b{}, c{};
    if (!field_ref(h, C3D_FIELD_U_REG, a) || !field_ref(h, C3D_FIELD_V_REG, b) ||
        !field_ref(h, C3D_FIELD_W_REG, c)) {
      h->last_error = "U_reg/V_reg/W_reg exist only with an immersed body";
      RET(h, C3D_ERR_UNSUPPORTED);
    }
    RET(h, launch_fill_ghosts3(h, a.ptr, b.ptr, c.ptr));
  }
  return C3D_ERR_PARAM;
}

int c3d_compute_dPx_for_constant_mass_flow(int id, double* dPdx) {
  GET_HANDLE(id);
  if (!dPdx) return C3D_ERR_PARAM;
  double q = 0;
  int rc = massflow(h, 0, false, &q);
  if (rc) RET(h, rc);
  *dPdx = h->Qflow_x_0 - q;
  RET(h, 0);
}

int c3d_compute_dPy_for_constant_mass_flow(int id, double* dPdy) {
  GET_HANDLE(id);
  if (!dPdy) return C3D_ERR_PARAM;
  double q = 0;
  int rc = massflow(h, 1, false, &q);
  if (rc) RET(h, rc);
  *dPdy = h->Qflow_y_0 - q;
  RET(h, 0);
}

int c3d_compute_dPz_for_constant_mass_flow(int id, double* dPdz) {
  GET_HANDLE(id);
  if (!dPdz) return C3D_ERR_PARAM;
  double q = 0;
  int rc = massflow(h, 2, true, &q);
  if (rc) RET(h, rc);
  *dPdz = h->Qflow_z_0 - q;
  RET(h, 0);
}

static int marker_out(Handle* h, double* dev, double* host, int64_t n);

int c3d_compute_statistics(int id, double* profiles, double* scalars) {
  GET_HANDLE(id);
  if (!profiles || !scalars) return C3D_ERR_PARAM;
  RET(h, compute_statistics(h, profiles, scalars));
}

int c3d_write_statistics(int id, const char* path, int istep) {
  GET_HANDLE(id);
  if (!path) return C3D_ERR_PARAM;
  const int nyg = h->d.nyg;
  std::vector<double> prof(7 * (size_t)nyg);
  double sc[8];
  int rc = compute_statistics(h, prof.data(), sc);
  if (rc) RET(h, rc);
  // output_statistics, src/input_output.f90:733-754
  FILE* f = std::fopen(path, "w");
  if (!f) { h->last_error = std::string("cannot open ") + path; RET(h, C3D_ERR_IO); }
  std::fprintf(f, "%%%15.8f%15.8f%15.8f%15.8f%12d%12d%12d%12d\n", h->t, sc[2], sc[0], h->p.nu, h->p.nx_global,
               h->p.ny_global, h->p.nz_global, istep);
  for (int j = 0; j < nyg; ++j) {
    std::fprintf(f, "%15.8f", h->yg[j + 1]);
    for (int q = 0; q < 7; ++q) std::fprintf(f, "%15.8f", prof[(size_t)q * nyg + j]);
    std::fprintf(f, "\n");
  }
  if (std::fclose(f) != 0) { h->last_error = std::string("write error on ") + path; RET(h, C3D_ERR_IO); }
  RET(h, 0);
}

int c3d_monitor(int id, double* out) {
  GET_HANDLE(id);
  if (!out) return C3D_ERR_PARAM;
  int rc = monitor_values(h, out);
  if (rc) RET(h, rc);
  out[7] = 0.0;
  if (h->ib) {
    // check_slip, src/monitor.f90:223-231: max |E u - E1nH_exterior dudn_jump - ub|
    const int nb = ib_nb(h);
    std::vector<double> Eu(3 * (size_t)nb), e1(3 * (size_t)nb), fb(4 * (size_t)nb), ub(3 * (size_t)nb);
    double* dev = ib_scratch(h, 0);
    if ((rc = ib_regT(h, h->U, h->V, h->W, dev))) RET(h, rc);
    if ((rc = marker_out(h, dev, Eu.data(), 3 * (int64_t)nb))) RET(h, rc);
    int64_t len = 0;
    double* p = ib_marker_ptr(h, C3D_MARKER_E1NH_EXT, &len);
    if ((rc = marker_out(h, p, e1.data(), 3 * (int64_t)nb))) RET(h, rc);
    p = ib_marker_ptr(h, C3D_MARKER_FB, &len);
    if ((rc = marker_out(h, p, fb.data(), 4 * (int64_t)nb))) RET(h, rc);
    p = ib_marker_ptr(h, C3D_MARKER_UB, &len);
    if ((rc = marker_out(h, p, ub.data(), 3 * (int64_t)nb))) RET(h, rc);
    double mx = 0.0;
    for (size_t q = 0; q < 3 * (size_t)nb; ++q) mx = std::max(mx, std::fabs(Eu[q] - e1[q] * fb[q] - ub[q]));
    out[7] = mx;
  }
  RET(h, 0);
}

int c3d_compute_pressure(int id) {
  GET_HANDLE(id);
  RET(h, compute_pressure(h));
}

int c3d_set_mode(int id, int poisson_mode, int precond_mode) {
  GET_HANDLE(id);
  if (poisson_mode != C3D_POISSON_FP64 && poisson_mode != C3D_POISSON_MIXED &&
      poisson_mode != C3D_POISSON_MIXED_UNREFINED) RET(h, C3D_ERR_PARAM);
  if (precond_mode < C3D_PRECOND_NONE || precond_mode > C3D_PRECOND_BAND) RET(h, C3D_ERR_PARAM);
  if ((precond_mode == C3D_PRECOND_BAND || precond_mode == C3D_PRECOND_LEARNED) && h->ib && !band_supported(h)) {
    h->last_error = "C3D_PRECOND_BAND and C3D_PRECOND_LEARNED need a marker lattice whose geometry repeats "
                    "along z (every body type except wall_plates)";
    RET(h, C3D_ERR_UNSUPPORTED);
  }
  if (poisson_mode != C3D_POISSON_FP64) {
    int rc = mixed_setup(h);
    if (rc) RET(h, rc);
  }
  h->refine_sweeps = (poisson_mode == C3D_POISSON_MIXED_UNREFINED) ? 0 : 1;
  if (poisson_mode == C3D_POISSON_MIXED_UNREFINED) poisson_mode = C3D_POISSON_MIXED;
  h->poisson_mode = poisson_mode;
  h->precond_mode = precond_mode;
  if (h->step_exec) { cudaGraphExecDestroy(h->step_exec); h->step_exec = nullptr; }
  RET(h, 0);
}

int c3d_get_stats(int id, c3d_stats* out) {
  GET_HANDLE(id);
  if (!out) return C3D_ERR_PARAM;
  int rc = sync_scalars_from_device(h);
  if (rc) return rc;
  h->stats.dPdx = h->dPdx; h->stats.dPdy = h->dPdy; h->stats.dPdz = h->dPdz;
  h->stats.t = h->t; h->stats.dt = h->dt; h->stats.qflow_x_0 = h->Qflow_x_0;
  h->stats.qflow_y_0 = h->Qflow_y_0; h->stats.qflow_z_0 = h->Qflow_z_0;
  h->stats.slab_cluster[0] = h->sp.cs64; h->stats.slab_cluster[1] = h->sp.cs32;
  h->stats.slab_narrow[0] = h->sp.nw64; h->stats.slab_narrow[1] = h->sp.nw32;
  ib_rows(h, h->stats.ib_rows);
  *out = h->stats;
  return 0;
}

int c3d_check_divergence(int id, double* mx) {
  GET_HANDLE(id);
  if (!mx) return C3D_ERR_PARAM;
  RET(h, max_abs_divergence(h, h->U, h->V, h->W, mx));
}

int c3d_check_finite(int id) {
  GET_HANDLE(id);
  bool ok = true;
  int rc = check_finite(h, &ok);
  if (rc) RET(h, rc);
  if (!ok) { h->last_error = "non-finite value in U, V or W"; RET(h, C3D_ERR_NAN); }
  RET(h, 0);
}

int c3d_last_step_time_ms(int id, double* ms) {
  GET_HANDLE(id);
  if (!ms) return C3D_ERR_PARAM;
  *ms = h->last_step_ms;
  return 0;
}

int c3d_kernel_launches(int id, int64_t* count) {
  GET_HANDLE(id);
  if (!count) return C3D_ERR_PARAM;
  *count = h->launches;
  return 0;
}

int c3d_profile_kernels(int id, int nrep, double* ms, int nmax) {
  GET_HANDLE(id);
  if (!ms || nrep <= 0) return C3D_ERR_PARAM;
  if (h->step_exec) { cudaGraphExecDestroy(h->step_exec); h->step_exec = nullptr; }
  const double dt = h->dt > 0 ? h->dt : 1e-3;
  const int ncls = 7;
  double out[ncls] = {0};
  for (int c = 0; c < ncls; ++c) {
    int rc = 0;
    // one untimed launch, then nrep timed ones
    for (int r = 0; r <= nrep; ++r) {
      if (r == 1) C3D_CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
      switch (c) {
        case 0: rc = launch_rhs_stage(h, 2, dt); break;
        case 1: rc = launch_fill_ghosts3(h, h->Us, h->Vs, h->Ws); break;
        case 2: case 3: case 4: rc = profile_spectral(h, c - 2); break;
        case 5: rc = launch_gradient_subtract(h, h->Us, h->Vs, h->Ws, h->rhs_p, dt, h->U, h->V, h->W, false, true); break;
        case 6: rc = launch_massflow_correction(h, dt); break;
      }
      if (rc) RET(h, rc);
    }
    C3D_CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
    C3D_CUDA_TRY(h, cudaEventSynchronize(h->ev1));
    float t = 0;
    C3D_CUDA_TRY(h, cudaEventElapsedTime(&t, h->ev0, h->ev1));
    out[c] = t / nrep;
  }
  for (int c = 0; c < ncls && c < nmax; ++c) ms[c] = out[c];
  RET(h, 0);
}

// ---- immersed boundary entries -------------------------------------------
static int need_ib(Handle* h) {
  if (h->ib) return 0;
  h->last_error = "no immersed body (body_type = 'none')";
  return C3D_ERR_UNSUPPORTED;
}

int c3d_setup_IB_geometry(int id) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  RET(h, ib_setup_geometry(h, h->t));
}
int c3d_setup_IB_operators(int id) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  RET(h, ib_setup_operators(h));
}
int c3d_compute_heaviside(int id) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  RET(h, ib_heaviside(h));
}

static int marker_out(Handle* h, double* dev, double* host, int64_t n) {
  C3D_CUDA_TRY(h, cudaMemcpyAsync(host, dev, n * 8, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

int c3d_regT(int id, double* Eu) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  double* dev = ib_scratch(h, 0);
  rc = ib_regT(h, h->U, h->V, h->W, dev);
  if (rc) RET(h, rc);
  RET(h, marker_out(h, dev, Eu, 3 * (int64_t)ib_nb(h)));
}
int c3d_regT_1n(int id, double* E) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  double* dev = ib_scratch(h, 0);
  rc = ib_regT_1n(h, h->U, h->V, h->W, dev);
  if (rc) RET(h, rc);
  RET(h, marker_out(h, dev, E, 3 * (int64_t)ib_nb(h)));
}
int c3d_regTc_1n(int id, int field, double* E) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  FieldRef f{};
  if (!field_ref(h, field, f) || f.lb[0] != 2) { h->last_error = "regTc_1n needs an rhs_p-shaped field"; RET(h, C3D_ERR_PARAM); }
  double* dev = ib_scratch(h, 0);
  rc = ib_regTc_1n(h, f.ptr, dev);
  if (rc) RET(h, rc);
  RET(h, marker_out(h, dev, E, (int64_t)ib_nb(h)));
}
int c3d_reg(int id, int comp, const double* f) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  if (comp < 1 || comp > 3 || !f) RET(h, C3D_ERR_PARAM);
  double* dev = ib_scratch(h, 1);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(dev, f, 8 * (int64_t)ib_nb(h), cudaMemcpyHostToDevice, h->stream));
  FieldRef F{};
  field_ref(h, C3D_FIELD_U_REG + comp - 1, F);
  rc = ib_reg(h, comp, dev, F.ptr);
  if (rc) RET(h, rc);
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  RET(h, 0);
}
int c3d_schur(int id, const double* f, double* Sf) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  const int64_t n = 4 * (int64_t)ib_nb(h);
  double* df = ib_scratch(h, 1);
  double* ds = ib_scratch(h, 0);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(df, f, n * 8, cudaMemcpyHostToDevice, h->stream));
  rc = ib_schur(h, df, ds, h->dt);
  if (rc) RET(h, rc);
  RET(h, marker_out(h, ds, Sf, n));
}
int c3d_bicgstab(int id, const double* rhs) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  const int64_t n = 4 * (int64_t)ib_nb(h);
  double* dr = ib_scratch(h, 2);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(dr, rhs, n * 8, cudaMemcpyHostToDevice, h->stream));
  RET(h, ib_bicgstab(h, dr, h->dt));
}
int c3d_precond_apply(int id, const double* in, double* out) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  const int64_t n = 4 * (int64_t)ib_nb(h);
  double* din = ib_scratch(h, 1);
  double* dout = ib_scratch(h, 0);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(din, in, n * 8, cudaMemcpyHostToDevice, h->stream));
  rc = ib_precond_apply(h, din, dout, h->dt);
  if (rc) RET(h, rc);
  RET(h, marker_out(h, dout, out, n));
}
int c3d_compute_IB_projection(int id) {
  GET_HANDLE(id);
  int rc = need_ib(h); if (rc) RET(h, rc);
  RET(h, ib_projection(h, h->dt, 0));
}

}  // extern "C"
