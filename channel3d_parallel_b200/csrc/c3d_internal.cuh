// Internal declarations of the channel3D B200 library (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/c3d.h"

namespace c3d {

// ---------------------------------------------------------------------------
// sizes of the single-domain reference arrays (src/initialization.f90:60-94)
// ---------------------------------------------------------------------------
struct Dims {
  int nx, ny, nz;      // faces incl. periodic extras: nx_global, ny_global, nz_global
  int nxg, nyg, nzg;   // centres incl. ghosts: nx+1, ny+1, nz+1
  int Nx, Ny, Nz;      // unique cells: nxp = nx-2, nym = ny-1, nzp = nz-2
  int nkx;             // Nx/2+1 retained x modes
  int nkzs;            // Nz/2+1 distinct kzz values
};

// Fortran-order linear index helpers (1-based Fortran indices).
__host__ __device__ inline int64_t idxU(const Dims& d, int i, int j, int k) {
  return (int64_t)(i - 1) + (int64_t)d.nx * ((j - 1) + (int64_t)d.nyg * (k - 1));
}
__host__ __device__ inline int64_t idxV(const Dims& d, int i, int j, int k) {
  return (int64_t)(i - 1) + (int64_t)d.nxg * ((j - 1) + (int64_t)d.ny * (k - 1));
}
__host__ __device__ inline int64_t idxW(const Dims& d, int i, int j, int k) {
  return (int64_t)(i - 1) + (int64_t)d.nxg * ((j - 1) + (int64_t)d.nyg * (k - 1));
}
__host__ __device__ inline int64_t idxP(const Dims& d, int i, int j, int k) {
  return (int64_t)(i - 1) + (int64_t)d.nxg * ((j - 1) + (int64_t)d.nyg * (k - 1));
}
// rhs_p(2:nxg-1, 2:nyg-1, 2:nzg)
__host__ __device__ inline int64_t idxR(const Dims& d, int i, int j, int k) {
  return (int64_t)(i - 2) + (int64_t)(d.nxg - 2) * ((j - 2) + (int64_t)(d.nyg - 2) * (k - 2));
}
inline int64_t sizeU(const Dims& d) { return (int64_t)d.nx * d.nyg * d.nzg; }
inline int64_t sizeV(const Dims& d) { return (int64_t)d.nxg * d.ny * d.nzg; }
inline int64_t sizeW(const Dims& d) { return (int64_t)d.nxg * d.nyg * d.nz; }
inline int64_t sizeP(const Dims& d) { return (int64_t)d.nxg * d.nyg * d.nzg; }
inline int64_t sizeR(const Dims& d) { return (int64_t)(d.nxg - 2) * (d.nyg - 2) * (d.nzg - 1); }

// ---------------------------------------------------------------------------
// 1-D metric coefficients, Fortran-indexed device arrays (entry 0 unused).
// Built on the host from the reference grids; every coefficient folds the
// divisions of src/equations.f90, src/differential_operators.f90 into one
// precomputed factor so kernels only multiply.
// ---------------------------------------------------------------------------
struct Metric {
  // x
  const double *rdx;     // 1/(x(i)-x(i-1))
  const double *rdxg;    // 1/(xg(i+1)-xg(i))
  const double *cxpF, *cxmF;   // viscous x for x-face fields (U)
  const double *cxpC, *cxmC;   // viscous x for x-centre fields (V, W)
  // y
  const double *rdy;     // 1/(y(j)-y(j-1))
  const double *rdyg;    // 1/(yg(j+1)-yg(j))
  const double *cypC, *cymC;   // viscous y for y-centre fields (U, W)
  const double *cypF, *cymF;   // viscous y for y-face fields (V)
  // z
  const double *rdz;     // 1/(z(k)-z(k-1))
  const double *rdzg;    // 1/(zg(k+1)-zg(k))
  const double *czpC, *czmC;   // viscous z for z-centre fields (U, V)
  const double *czpF, *czmF;   // viscous z for z-face fields (W)
  // mass-flow weights 0.5*(yg(j)-yg(j-1)) (U, W) and 0.5*(y(j)-y(j-1)) (V)
  const double *wq, *wqv;
  // weight of u(j) in the x bulk flux, wq(j) + wq(j+1) (zero outside the pairs)
  const double *cqu;
};

// device scalars shared by kernels of one step (kept on device so the step
// can be captured in one CUDA graph)
struct DevScalars {
  double dPdx, dPdy, dPdz;
  double shift;          // last constant-mass-flow correction of U
  double shift_v, shift_w;  // same for V and W (y_mass_cte, z_mass_cte)
  double qflow;          // last bulk flux (Int_U / norm)
  double dpdx_prev;
  unsigned long long err;   // sticky kernel error bits (bit 0: a bounded copy wait gave up)
  unsigned int ticket;      // blocks done in the current reduction (reset by the last one)
  unsigned int pad;
};

// Spectral Poisson state: twiddles, Thomas factor tables and spectra for the
// FP64 path and the FP32 (mixed-precision) path.
struct SpectralState {
  double2 *twx = nullptr, *twz = nullptr;    // exp(-2 pi i m / n) (device)
  float2 *twx32 = nullptr, *twz32 = nullptr;
  int* posx = nullptr;                       // digit-reversed position of x coefficient m
  // Thomas factors of every (kx, kz') mode, layout [(m*Ny + j)*nkzs + kz']:
  // multipliers DL(j)/D'(j) and reciprocal pivots 1/D'(j)
  double *mult = nullptr, *rdp = nullptr;
  float *mult32 = nullptr, *rdp32 = nullptr;
  double *dl = nullptr, *du = nullptr;       // Dyy(j+1, j) and Dyy(j, j+1), j = 0..Ny-1 (0 past the end)
  // x(j)/y(j) of the homogeneous tail (right-hand side zero from row j on),
  // same layout as rdp; built on first use by the band-restricted solve
  double* tail = nullptr;
  float *dl32 = nullptr, *du32 = nullptr;
  // spectra, layout [m][j][k] = [(m*Ny + (j-2))*pz + (k-2)]: one kx slab is
  // Ny rows of pz complex values (pz*sizeof(complex) a multiple of 16 bytes)
  double2* spec = nullptr;
  float2* spec32 = nullptr;
  int pz64 = 0, pz32 = 0;
  // FP64 kx = kz = 0 mode of the FP32 path
  double* linesum = nullptr;                 // per (j, k) line sum of the right-hand side
  double* phi00 = nullptr;                   // mean solution / (Nx*Nz) per j
  // cluster decomposition of a kx slab: cs CTAs of jc rows of j, shared
  // memory row stride rs complex values, nt threads, smem bytes
  int cs64 = 1, jc64 = 1, rs64 = 0, nt64 = 256, smem64 = 0, nw64 = 0;   // nw: narrow slab CTAs
  int cs32 = 1, jc32 = 1, rs32 = 0, nt32 = 256, smem32 = 0, nw32 = 0;
};

struct Params {
  // defaults of src/input_output.f90:43-62 (pi = 4*atan(1), src/global.f90:30)
  double Lxp = 8.0 * 0.78539816339744830962, Lzp = 4.0 * 0.78539816339744830962;
  double Ly_channel = 2.0, alpha_stretch = 2.6;
  int nx_global = 0, ny_global = 0, nz_global = 0, nxb = 0, nzb = 0;
  double CFL = 0, nu = 0, dPdx = 0, dPdz = 0, Qflow_x_0 = -999999.0, Qflow_z_0 = -999999.0;
  int x_mass_cte = 0, y_mass_cte = 0, z_mass_cte = 0;
  int nsteps = 0, nsave = 0, nstats = 0, nmonitor = 0;
  std::string filein, fileout;
  int nstep_init = 0;
  double t_init = 0;
  int init_type = 1, grid_type = 0;
  std::string body_type = "none";
  bool exterior_pressure_gradient = true;
  double body_param_1 = 0, body_param_2 = 0, body_param_3 = 0, body_ramp_up_time = 0;
  // extension (no reference counterpart): mean y of the single plane of
  // body_type 'wall_standing_wave'
  double body_param_4 = 0;
  double min_buffer_width = 0, cg_tol = (double)1e-8f;
  int cg_max_iter = 50;
  double perturb_scale = 0.5;
};

int parse_namelist(const std::string& text, Params& p, std::string& err);
// message returned by c3d_last_error for calls that have no handle
void set_global_error(const std::string& msg);

struct IbState;   // immersed-boundary state (k_ib.cu)
struct MlpState;  // learned preconditioner network (k_mlp.cu)
struct MixedState;  // mixed-precision work buffers (k_poisson.cu)

struct Handle {
  Params p;
  Dims d;
  cudaStream_t stream = nullptr;
  int device = 0;
  // host grids (Fortran-indexed)
  std::vector<double> x, y, z, xm, ym, zm, xg, yg, zg;
  double dxmin = 0, dymin = 0, dzmin = 0, dx = 0, dz = 0, Lx = 0, Ly = 0, Lz = 0, Lxp = 0, Lzp = 0;
  std::vector<double> kxx, kzz;           // modified wavenumbers
  std::vector<double> Dd, Dl, Du;         // Dyy diagonals (Fortran rows 2..nyg-1)
  double mass_norm = 0;                   // constant-H norm of the mass-flow integral
  // device memory
  std::vector<void*> allocations;
  double* metric_buf = nullptr;
  Metric m{};
  double *U = nullptr, *V = nullptr, *W = nullptr, *P = nullptr;
  double *Us = nullptr, *Vs = nullptr, *Ws = nullptr;       // star / work fields
  double* pbc = nullptr;          // compute_pressure wall conditions bc_1, bc_2 (2 x nxg x nzg)
  double* stat_buf = nullptr;     // compute_statistics partials and profiles
  int64_t stat_cap = 0;
  double *Gu = nullptr, *Gv = nullptr, *Gw = nullptr;       // RK accumulators
  double *rhs_p = nullptr;                                  // rhs_p / phi
  double *P_interim = nullptr;
  double *phi1 = nullptr;                                   // stage-1 phi for P
  double *rhsU = nullptr, *rhsV = nullptr, *rhsW = nullptr; // fine-entry rhs arrays
  double* red = nullptr;                                    // reduction partials
  double* flux_part = nullptr;    // per-block x bulk-flux partials (forward x FFT of the last stage)
  int64_t flux_part_len = 0;
  double norm_u = 0;             // norm of the x bulk flux (the flux of u = 1)
  bool x_uniform = false;        // x spacing uniform (the flux of d(phi)/dx telescopes to zero)
  int red_len = 0;
  DevScalars* sc = nullptr;
  SpectralState sp;
  int refine_sweeps = 1;          // mixed precision: refinement projections per stage
  // state
  double t = 0, dt = 0;
  double dPdx = 0, dPdy = 0, dPdz = 0, Qflow_x_0 = 0, Qflow_y_0 = 0, Qflow_z_0 = 0;
  bool P_pending = false;        // P must be rebuilt from phi1 before download
  double P_pending_dt = 0;
  int poisson_mode = C3D_POISSON_FP64;
  int precond_mode = C3D_PRECOND_NONE;
  c3d_stats stats{};
  std::string last_error;
  int64_t launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // host-resident stepping: copy streams and per-slab download events
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_up = nullptr, ev_done = nullptr;
  std::vector<cudaEvent_t> ev_slab;
  double last_step_ms = 0;
  IbState* ib = nullptr;
  MixedState* mixed = nullptr;
  MlpState* mlp = nullptr;
  // one RK3 step captured as a CUDA graph (valid for graph_dt)
  cudaGraphExec_t step_exec = nullptr;
  double graph_dt = 0;
  int64_t graph_launches = 0;     // kernels per captured step
  int64_t graph_solves = 0;       // Poisson solves per captured step
  bool use_graph = true;
  bool write_pinterim = false;   // projection also stores P_interim = phi/dt
  int rhs_kernel = 0;             // 0: shared-memory tiled stage kernel, 1: per-point kernel
  // programmatic dependent launch of the time step's kernels: off, the
  // captured step graph ran slower with it (1118 against 1124 steps/s at
  // 192x129x192) although each kernel alone starts 2-3 us earlier
  bool use_pdl = false;
};

const double* ib_hu(Handle* h);
const double* ib_hv(Handle* h);
const double* ib_hw(Handle* h);
bool ib_moving(Handle* h);

// ---- error helpers --------------------------------------------------------
struct Status {
  int code = 0;
  std::string msg;
};

#define C3D_CUDA_TRY(h, expr)                                                   \
  do {                                                                          \
    cudaError_t _e = (expr);                                                    \
    if (_e != cudaSuccess) {                                                    \
      (h)->last_error = std::string(#expr) + ": " + cudaGetErrorString(_e);     \
      return C3D_ERR_CUDA;                                                      \
    }                                                                           \
  } while (0)

#define C3D_LAUNCH_CHECK(h)                                                     \
  do {                                                                          \
    (h)->launches++;                                                            \
    cudaError_t _e = cudaGetLastError();                                        \
    if (_e != cudaSuccess) {                                                    \
      (h)->last_error = std::string("kernel launch: ") + cudaGetErrorString(_e);\
      return C3D_ERR_CUDA;                                                      \
    }                                                                           \
  } while (0)

// ---- programmatic dependent launch ----------------------------------------
// The time step's kernels are launched so that a kernel's CTAs may start
// while its predecessor in the stream finishes: each kernel reads only
// set-up tables (twiddles, metric, digit reversal) before pdl_wait(), which
// returns once the preceding grid has completed and its writes are visible;
// it then calls pdl_trigger(), so the next kernel launches once every CTA of
// this one has passed its wait.  Both are no-ops for an ordinary launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t stream, Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// ---- kernels / drivers implemented in the .cu files ----------------------
// boundary conditions (k_bc.cu)
enum FieldKind { KIND_U = 0, KIND_V = 1, KIND_W = 2 };
int launch_fill_ghosts(Handle* h, double* F, FieldKind kind);
int launch_fill_ghosts3(Handle* h, double* U, double* V, double* W);
// rhs (k_rhs.cu)
int rhs_setup(Handle* h);
int launch_rhs_stage(Handle* h, int stage, double dt);
int launch_rhs_euler(Handle* h, double dt);
int launch_rhs_only(Handle* h, int component);
// poisson + projection (k_poisson.cu)
int poisson_setup(Handle* h);
int launch_divergence(Handle* h, const double* U, const double* V, const double* W, double* rhs);
int launch_poisson_solve(Handle* h, double* rhs, int rk_step, double dt);
int launch_poisson_of_div(Handle* h, const double* U, const double* V, const double* W, double* out,
                          int rk_step, double dt);
int launch_poisson_of_div_band(Handle* h, const double* U, const double* V, const double* W, double* out,
                               int jlo, int jhi);
int launch_projection_step(Handle* h, int rk_step, double dt, const double* ushift = nullptr);
int launch_gradient_subtract(Handle* h, const double* Ui, const double* Vi, const double* Wi,
                             const double* phi, double dt, double* Uo, double* Vo, double* Wo,
                             bool dup_plane = true, bool with_ghosts = false,
                             const double* ushift = nullptr);
int rebuild_pressure(Handle* h);
int compute_pressure(Handle* h);
int profile_spectral(Handle* h, int part);   // 0 div_xfft, 1 spectral_yz, 2 xfft inv
int mixed_setup(Handle* h);
void mixed_free(Handle* h);
// mass flow and reductions (k_massflow.cu)
int launch_massflow_correction(Handle* h, double dt, bool euler = false, bool skip_x = false);
int massflow(Handle* h, int comp, bool u_view, double* q_out);
int massflow_w_as_v(Handle* h, double* q_out);
// diagnostics (k_stats.cu)
int compute_statistics(Handle* h, double* profiles, double* scalars);
int monitor_values(Handle* h, double* out);
int max_abs_divergence(Handle* h, const double* U, const double* V, const double* W, double* out);
int check_finite(Handle* h, bool* ok);
int compute_dt_cfl(Handle* h, double* dt);
// immersed boundary (k_ib.cu)
int ib_create(Handle* h);
void ib_free(Handle* h);
void mlp_free(Handle* h);
int ib_setup_geometry(Handle* h, double t);
int ib_setup_operators(Handle* h);
void ib_grids_changed(Handle* h);   // the next operator set-up re-uploads the grids
int ib_heaviside(Handle* h);
int ib_projection(Handle* h, double dt, int rk_step);
int ib_regT(Handle* h, const double* U, const double* V, const double* W, double* Eu_dev);
int ib_regTc_1n(Handle* h, const double* P, double* E_dev);
int ib_regT_1n(Handle* h, const double* U, const double* V, const double* W, double* E_dev);
int ib_reg(Handle* h, int comp, const double* f_dev, double* F);
int ib_schur(Handle* h, const double* f_dev, double* Sf_dev, double dt);
int ib_bicgstab(Handle* h, const double* rhs_dev, double dt);
// y rows (Fortran j) that the markers' stencils reach; 0 0 without IB
void ib_rows(const Handle* h, int32_t rows[2]);
int ib_precond_apply(Handle* h, const double* in_dev, double* out_dev, double dt);
double* ib_marker_ptr(Handle* h, int id, int64_t* len);
double* ib_field_ptr(Handle* h, int id);
double* ib_scratch(Handle* h, int which);
int ib_nb(Handle* h);
bool band_supported(Handle* h);   // banded Schur preconditioner available (k_ib_band.cu)

// allocation helper
template <typename T>
int dev_alloc(Handle* h, T** ptr, int64_t count) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, sizeof(T) * (size_t)(count > 0 ? count : 1));
  if (e != cudaSuccess) {
    h->last_error = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return C3D_ERR_CUDA;
  }
  cudaMemsetAsync(p, 0, sizeof(T) * (size_t)(count > 0 ? count : 1), h->stream);
  h->allocations.push_back(p);
  *ptr = (T*)p;
  return 0;
}

}  // namespace c3d
