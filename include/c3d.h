/*
 * c3d.h -- C-ABI of the B200 (sm_100a) channel3D RK3 fractional-step path.
 *
 * Every entry point replaces one Fortran module procedure of
 * MetamaterialFSI/channel3D_parallel; the citation beside each declaration
 * names the reference interface (file:line).  The unchanged Fortran driver
 * (app/main.f90) binds these through an ISO_C_BINDING interface module.
 *
 * Conventions
 *  - Every function returns int: 0 = OK, < 0 = error (C3D_ERR_*), > 0 =
 *    warning (C3D_WARN_*).  c3d_last_error() returns the message of the last
 *    non-zero status on that handle.  Nothing is thrown across the ABI and
 *    nothing calls exit().
 *  - Fields live in device memory owned by the library for the lifetime of
 *    the handle; they move to and from the host only through
 *    c3d_upload / c3d_download (and, for U, V, W, c3d_time_step_rk3_host).
 *    Host buffers are caller-owned, FP64,
 *    Fortran (column-major) order, and hold exactly the box lb..ub (inclusive,
 *    Fortran indices of the field, see C3D_FIELD_* below).
 *  - The domain is the reference's global array set for one z slab:
 *    nx = nx_global, ny = ny_global, nz = nz_global, nxg = nx+1, nyg = ny+1,
 *    nzg = nz+1 (src/initialization.f90:60-94 with nprocs = 1).
 *  - One host thread per handle; each handle owns one CUDA stream for its
 *    kernels (and two copy streams once c3d_time_step_rk3_host is used).
 */
#ifndef C3D_H
#define C3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define C3D_OK                  0
#define C3D_ERR_PARAM          -1   /* bad argument / namelist value          */
#define C3D_ERR_CUDA           -2   /* CUDA runtime error                     */
#define C3D_ERR_NAN            -3   /* non-finite value found in a field      */
#define C3D_ERR_HANDLE         -4   /* unknown or destroyed handle            */
#define C3D_ERR_IO             -5   /* file could not be read                 */
#define C3D_ERR_UNSUPPORTED    -6   /* option not available for this set-up  */
#define C3D_ERR_NO_DEVICE      -7   /* no CUDA device visible                 */
#define C3D_WARN_NOT_CONVERGED  1   /* BiCGSTAB stopped at cg_max_iter        */

/* ---- field identifiers (Fortran extents, lower bound 1 unless stated) ---- */
#define C3D_FIELD_U             1   /* U(nx, nyg, nzg)        src/global.f90:106 */
#define C3D_FIELD_V             2   /* V(nxg, ny, nzg)                           */
#define C3D_FIELD_W             3   /* W(nxg, nyg, nz)                           */
#define C3D_FIELD_P             4   /* P(nxg, nyg, nzg)                          */
#define C3D_FIELD_RHS_P         5   /* rhs_p(2:nxg-1, 2:nyg-1, 2:nzg)  src/initialization.f90:155 */
#define C3D_FIELD_P_INTERIM     6   /* P_interim, rhs_p extents  src/projection.f90:36 */
#define C3D_FIELD_RHS_U         7   /* rhs_u(2:nx-1, 2:nyg-1, 2:nzg-1) src/equations.f90:29 */
#define C3D_FIELD_RHS_V         8   /* rhs_v(2:nxg-1, 2:ny-1, 2:nzg-1) */
#define C3D_FIELD_RHS_W         9   /* rhs_w(2:nxg-1, 2:nyg-1, 2:nz-1) */
#define C3D_FIELD_U_WORK       10   /* U-shaped work field (e.g. U_interim)      */
#define C3D_FIELD_V_WORK       11
#define C3D_FIELD_W_WORK       12
/* immersed-boundary fields */
#define C3D_FIELD_U_REG        13   /* U_reg (U extents)  src/global.f90:107 */
#define C3D_FIELD_V_REG        14
#define C3D_FIELD_W_REG        15
#define C3D_FIELD_HU_INTERIOR  16   /* Heaviside fields   src/global.f90:255-259 */
#define C3D_FIELD_HV_INTERIOR  17
#define C3D_FIELD_HW_INTERIOR  18
#define C3D_FIELD_HC_EXTERIOR  19   /* Hc_exterior, rhs_p extents */
/* Lagrangian (marker) arrays: 1-D, lb[0]..ub[0] index the vector */
#define C3D_MARKER_FB          40   /* fb(4*nb)       src/global.f90:238 */
#define C3D_MARKER_UB          41   /* ub(3*nb)       src/global.f90:232 */
#define C3D_MARKER_XB          42   /* xb(nb)  */
#define C3D_MARKER_YB          43   /* yb(nb)  */
#define C3D_MARKER_ZB          44   /* zb(nb)  */
#define C3D_MARKER_NORMALS     45   /* normals(3*nb)  */
#define C3D_MARKER_SB          46   /* sb(nb)  */
#define C3D_MARKER_E1NH_EXT    47   /* E1nH_exterior(3*nb) */
#define C3D_MARKER_E1NHC_EXT   48   /* E1nHc_exterior(nb)  */

/* ---- solver options ------------------------------------------------------ */
#define C3D_POISSON_FP64        0   /* plain FP64 spectral Poisson solve        */
#define C3D_POISSON_MIXED       1   /* FP32 spectral solve + FP64 refinement    */
#define C3D_POISSON_MIXED_UNREFINED 2 /* FP32 spectral solve, no refinement (accuracy studies) */
#define C3D_PRECOND_NONE        0   /* reference BiCGSTAB (unpreconditioned)    */
#define C3D_PRECOND_JACOBI      1   /* diagonal (Jacobi) preconditioner         */
#define C3D_PRECOND_LEARNED     2   /* learned preconditioner + warm start      */
#define C3D_PRECOND_SPAI        3   /* probed 4x4 block sparse approximate inverse */
#define C3D_PRECOND_BAND        4   /* probed local band of S, solved exactly per z wavenumber */

typedef struct c3d_dims {
  int32_t nx, ny, nz;          /* nx_global, ny_global, nz_global            */
  int32_t nxg, nyg, nzg;       /* centre extents incl. ghosts                 */
  int32_t nxp, nzp, nym;       /* periodic cells in x, z; cells in y          */
  int32_t nb;                  /* Lagrangian markers (0 without IB)          */
} c3d_dims;

typedef struct c3d_stats {
  int64_t steps;               /* RK3 steps taken                             */
  int64_t poisson_solves;      /* Poisson solves issued                       */
  int64_t bicgstab_solves;     /* IB Schur solves                             */
  int64_t bicgstab_iters;      /* accumulated BiCGSTAB iterations (cg_accum_iter) */
  int32_t last_bicgstab_iters; /* iterations of the last Schur solve          */
  int32_t refinement_sweeps;   /* mixed-precision refinement sweeps, last solve */
  int64_t precond_fallbacks;   /* learned-preconditioner hand-overs to the probed band */
  double  last_residual;       /* ||r||_2 at exit of the last Schur solve     */
  double  dPdx, dPdy, dPdz;    /* current mean pressure gradients             */
  double  t, dt;               /* simulation time and last dt                 */
  double  qflow_x_0;           /* target bulk flow                            */
  int32_t status;              /* last status code                            */
  int32_t precond_mode;        /* preconditioner of the last Schur solve      */
  double  last_bicgstab_ms;    /* device time of the last Schur solve (ms)    */
  double  bicgstab_ms;         /* accumulated device time of Schur solves     */
  int32_t slab_cluster[2];     /* CTAs per kx-slab cluster of the y-z solve: FP64, FP32 */
  int32_t slab_narrow[2];      /* 1: narrow slab CTAs (<= 192 threads, 3 per SM); FP64, FP32 */
  double  qflow_y_0, qflow_z_0;/* targets of the y and z constant-flux corrections */
  int64_t precond_builds;      /* probed (or predicted) band preconditioners built */
  double  precond_build_ms;    /* accumulated device time of those builds (ms) */
  int32_t ib_rows[2];          /* y rows (Fortran j) the markers' stencils reach; 0 0 without IB */
} c3d_stats;

/* ---- lifecycle ------------------------------------------------------------
 * c3d_create: read the &params namelist (src/input_output.f90:21-132), build
 * the grid (create_grid, src/input_output.f90:140-206), metrics, Fourier and
 * tridiagonal set-up (initialize, src/initialization.f90:24-460) and allocate
 * the device fields.  The fields start at zero (init_type 1); upload a state
 * with c3d_upload or a snapshot grid with c3d_set_grid.                      */
int c3d_create(const char* namelist_path, int* handle);
/* same, from namelist text in memory */
int c3d_create_from_text(const char* namelist_text, int* handle);
/* finalize, src/finalization.f90:19-33 */
int c3d_destroy(int handle);
/* replace the face grids (read_input_data mesh, src/input_output.f90:347-358) */
int c3d_set_grid(int handle, const double* x, const double* y, const double* z);
int c3d_get_dims(int handle, c3d_dims* dims);
/* read back the grids: x(nx), y(ny), z(nz), xg(nxg), yg(nyg), zg(nzg) */
int c3d_get_grid(int handle, double* x, double* y, double* z,
                 double* xg, double* yg, double* zg);
const char* c3d_last_error(int handle);

/* ---- field transfer ------------------------------------------------------ */
int c3d_upload(int handle, int field_id, const double* host,
               const int64_t lb[3], const int64_t ub[3]);
int c3d_download(int handle, int field_id, double* host,
                 const int64_t lb[3], const int64_t ub[3]);
/* scalars: dPdx, dPdy, dPdz, t, Qflow_x_0 (module globals, src/global.f90:167-173) */
int c3d_set_scalars(int handle, double dPdx, double dPdy, double dPdz,
                    double t, double qflow_x_0);
int c3d_synchronize(int handle);

/* ---- coarse entries (hot path) -------------------------------------------- */
/* compute_time_step_RK3, src/time_integration.f90:86-213; nsteps steps, each
 * preceded by compute_dt (src/time_integration.f90:219-267).               */
int c3d_time_step_rk3(int handle, int nsteps);
/* compute_time_step_RK3 for a driver whose u, v, w stay in its own arrays, as
 * the reference's time loop keeps them (app/main.f90:101-117): every one of
 * the nsteps steps uploads U(nx,nyg,nzg), V(nxg,ny,nzg) and W(nxg,nyg,nz)
 * (whole Fortran arrays, lower bounds 1), advances one step and writes the
 * fields back into the same arrays.  With page-locked arrays the download of
 * step n and the upload of step n+1 overlap slab by slab; returns when the
 * last download has landed.                                                  */
int c3d_time_step_rk3_host(int handle, double* U, double* V, double* W, int nsteps);
/* compute_time_step_Euler, src/time_integration.f90:25-81 (explicit Euler,
 * non-IB projection, x and y constant-flux corrections); nsteps steps, each
 * preceded by compute_dt.                                                   */
int c3d_time_step_euler(int handle, int nsteps);
/* compute_dt, src/time_integration.f90:219-267 */
int c3d_compute_dt(int handle, double* dt);
/* compute_mean_mass_flow_U with Hu, src/mass_flow.f90:24-53 (app/main.f90:90) */
int c3d_compute_mean_mass_flow_u(int handle, double* qflow);
/* compute_mean_mass_flow_V / _W, src/mass_flow.f90:62-129 (app/main.f90:91-92) */
int c3d_compute_mean_mass_flow_v(int handle, double* qflow);
int c3d_compute_mean_mass_flow_w(int handle, double* qflow);
/* Qflow_x_0, Qflow_y_0, Qflow_z_0 (src/global.f90:180): the targets of the
 * constant-flux corrections enabled by x/y/z_mass_cte                       */
int c3d_set_flow_targets(int handle, double qflow_x_0, double qflow_y_0, double qflow_z_0);

/* ---- fine entries mirroring the module interfaces ------------------------- */
/* compute_rhs_u/v/w(U,V,W,rhs), src/equations.f90:24,160,295: reads the
 * current U,V,W fields, writes C3D_FIELD_RHS_U/V/W.                         */
int c3d_compute_rhs_u(int handle);
int c3d_compute_rhs_v(int handle);
int c3d_compute_rhs_w(int handle);
/* solve_poisson_equation(rhs), src/poisson.f90:33-101: in place on
 * C3D_FIELD_RHS_P; rk_step == 1 also sets P (src/poisson.f90:91-99).        */
int c3d_solve_poisson_equation(int handle, int rk_step);
/* divergence(rhs_p, U, V, W), src/differential_operators.f90:54-74 */
int c3d_divergence(int handle);
/* compute_non_IB_projection, src/projection.f90:22-46 */
int c3d_compute_non_IB_projection(int handle, int rk_step);
/* apply_boundary_conditions(U,V,W), src/boundary_conditions.f90:20-55;
 * which: 0 = U,V,W; 1 = U_reg,V_reg,W_reg; 2 = the U/V/W work fields       */
int c3d_apply_boundary_conditions(int handle, int which);
/* compute_dPx_for_constant_mass_flow(U, dPdx), src/mass_flow.f90:144-175 */
int c3d_compute_dPx_for_constant_mass_flow(int handle, double* dPdx);
/* compute_dPy_for_constant_mass_flow(V, dPdy), src/mass_flow.f90:190-221 */
int c3d_compute_dPy_for_constant_mass_flow(int handle, double* dPdy);
/* compute_dPz_for_constant_mass_flow(W, dPdz), src/mass_flow.f90:236-267; reads
 * W through the routine's declared extents Dimension(nx,nyg,nzg) (:238), as the
 * reference does                                                            */
int c3d_compute_dPz_for_constant_mass_flow(int handle, double* dPdz);
/* compute_pressure, src/pressure.f90:21-341: the actual pressure into P
 * (wall conditions d/dy(nu dV/dy), divergence of the right-hand sides, the
 * Poisson solve with inhomogeneous Neumann rows); the reference's call sites
 * are commented out (src/statistics.f90:37, src/input_output.f90:508).       */
int c3d_compute_pressure(int handle);

/* ---- snapshots and diagnostics (the calls of app/main.f90:97-118) --------- */
/* output_data, src/input_output.f90:498-728: binary snapshot of the current
 * state (big-endian stream: mesh, U, V, W, P, Hu/Hv/Hw_interior, t, dt, dPdx,
 * nu, marker arrays); original_format = 1 stops after P (tools/file_io.py's
 * original format).                                                          */
int c3d_write_snapshot(int handle, const char* path, int original_format);
/* read_input_data, src/input_output.f90:335-489: mesh and U, V, W of a
 * snapshot; every size must match the handle (C3D_ERR_PARAM otherwise, with
 * the reference's message); replaces the grid (as c3d_set_grid) and fields.  */
int c3d_read_snapshot(int handle, const char* path);
/* compute_statistics, src/statistics.f90:22-148: profiles[7*nyg] = Umean,
 * Vmean, Wmean, U2mean, V2mean, W2mean, UVmean at yg(1:nyg); scalars[8] =
 * utau, wtau, Retau_u, Retau_w, Qflow_x, Qflow_y, Qflow_z, and 1 if U, V or
 * W holds a non-finite value (the reference stops there).                    */
int c3d_compute_statistics(int handle, double* profiles, double* scalars);
/* output_statistics, src/input_output.f90:733-754: the statistics text file */
int c3d_write_statistics(int handle, const char* path, int istep);
/* output_monitor reductions, src/monitor.f90:21-110: out[8] = mean U, V, W
 * (divided by nxm*nym*nzm as printed), max U, V, W, max |div u|, max IB slip
 * (check_slip, :223-231; 0 without a body).                                 */
int c3d_monitor(int handle, double* out);

/* ---- immersed boundary ---------------------------------------------------- */
/* setup_IB_geometry (src/immersed_boundary_geometry.f90:70-398) at time t   */
int c3d_setup_IB_geometry(int handle);
/* setup_IB_operators, src/immersed_boundary_operators.f90:19-256 */
int c3d_setup_IB_operators(int handle);
/* compute_heaviside, src/heaviside.f90:20-54 */
int c3d_compute_heaviside(int handle);
/* regT(Eu, U, V, W), src/immersed_boundary_operators.f90:296-318: host out (3*nb) */
int c3d_regT(int handle, double* Eu);
/* regTc_1n(E1np, P_interim), src/immersed_boundary_operators.f90:344-357 (nb) */
int c3d_regTc_1n(int handle, int field_id, double* E1np);
/* regT_1n(E1nu, U, V, W), src/immersed_boundary_operators.f90:320-342 (3*nb) */
int c3d_regT_1n(int handle, double* E1nu);
/* regu/regv/regw(F, f), src/immersed_boundary_operators.f90:359-400:
 * component 1/2/3 spread of f (nb) into U_reg/V_reg/W_reg                 */
int c3d_reg(int handle, int component, const double* f);
/* schur(Sf, f), src/projection.f90:98-144 (host vectors of 4*nb) */
int c3d_schur(int handle, const double* f, double* Sf);
/* bicgstab(fb, rhs_ib), src/projection.f90:146-186: solves for the device
 * fb (warm start = current fb) with right-hand side rhs (4*nb, host).       */
int c3d_bicgstab(int handle, const double* rhs);
/* No counterpart in the reference (its BiCGSTAB is unpreconditioned): apply
 * the Schur-solve preconditioner selected by c3d_set_mode to a host marker
 * vector, out = M in (4*nb each), building it first when it is missing or
 * stale; C3D_PRECOND_NONE copies.  For tests and diagnostics.             */
int c3d_precond_apply(int handle, const double* in, double* out);
/* compute_IB_projection, src/projection.f90:48-96 */
int c3d_compute_IB_projection(int handle);

/* ---- options and telemetry ------------------------------------------------ */
int c3d_set_mode(int handle, int poisson_mode, int precond_mode);
int c3d_get_stats(int handle, c3d_stats* stats);
/* max |div u| over interior cells, src/monitor.f90:210-221 */
int c3d_check_divergence(int handle, double* max_divergence);
/* NaN scan of U,V,W (statistics NaN stop, src/statistics.f90:142-144):
 * returns C3D_ERR_NAN if any entry is not finite.                           */
int c3d_check_finite(int handle);

/* ---- timing support (kernel-level evidence) ------------------------------- */
/* device time in ms of the last c3d_time_step_rk3 call, from CUDA events     */
int c3d_last_step_time_ms(int handle, double* ms);
/* number of kernels launched by the library since the handle was created   */
int c3d_kernel_launches(int handle, int64_t* count);
/* time every kernel class of one RK3 stage separately, each launched nrep
 * times between CUDA events on the handle's stream (the fields are used as
 * scratch); ms[c] = average device time of class c in the order
 * rhs_stage, ghosts, div_xfft, spectral_yz, xfft_inv, grad_sub, massflow
 * (FP64 kernels).  Writes min(nmax, 7) entries.                              */
int c3d_profile_kernels(int handle, int nrep, double* ms, int nmax);

/* ---- learned preconditioner / warm start of the IB Schur solve ------------
 * No reference counterpart (the reference's bicgstab, src/projection.f90:146-186,
 * is unpreconditioned).  A per-marker 4x4 block z_b = A_b r_b with A_b predicted
 * from 32 geometry features by an MLP 32-128-128-16 (BF16 weights, FP32
 * accumulation, tcgen05 tensor cores); selected with c3d_set_mode(...,
 * C3D_PRECOND_LEARNED).  The solve falls back to Jacobi when it stalls.
 *
 * c3d_precond_collect: while enabled, converged Schur solves keep up to
 *   max_store iterates and add one training set (moments of the residual /
 *   correction pairs of that geometry); up to max_sets sets are kept.
 * c3d_precond_train: full-batch Adam over the collected sets; final_loss is
 *   the relative least-squares loss (1 = no better than zero correction).
 * c3d_precond_probe: probe the Schur operator on the current geometry with
 *   lattice colour classes (100 applications) and add one training set of
 *   (unit correction, response) moments: the block sparse-approximate-inverse
 *   target min ||I - S M||_F.  All sets of one network use one kind of pairs.
 * c3d_precond_info: pairs used, sets, epochs trained, last loss.
 * c3d_precond_get_params / set_params: the packed FP32 parameters
 *   (C3D_PRECOND_NPARAM values; get_params appends sig_r[4], sig_e[4]).
 * c3d_precond_eval: forward, loss and parameter gradient on caller data
 *   (m rows of 32 features and 36 moments; sig = sig_r[4], sig_e[4]). */
#define C3D_PRECOND_NPARAM 22800
int c3d_precond_collect(int handle, int enable, int max_store, int max_sets);
int c3d_precond_probe(int handle);
int c3d_precond_train(int handle, int epochs, double lr, double* final_loss);
int c3d_precond_info(int handle, int64_t* pairs, int* sets, int* epochs, double* last_loss);
int c3d_precond_get_params(int handle, float* params, int n);
int c3d_precond_set_params(int handle, const float* params, int n, const float* sig);
int c3d_precond_eval(int handle, const float* feats, const float* moments, int m, const float* sig,
                     float* out, float* grad, double* loss);

/* ---- allocation-free entry ------------------------------------------------
 * No counterpart in the reference.  Bulk flux of U, the value of
 * c3d_compute_mean_mass_flow_u for a field without immersed body (Hu = 1),
 * for callers that must not allocate device memory -- a driver that checks
 * the flux inside its own time loop, where cudaMalloc would synchronise the
 * device, or a program whose device memory belongs to another runtime's
 * fixed pool.  No handle is needed and nothing is allocated: the per-plane
 * partial sums live in a static device array of 4096 z planes (64 KiB per
 * GPU that loads the library, held until exit); nzg-2 > 4096 is rejected
 * with C3D_ERR_PARAM.  The first call on a device looks up that array's
 * address, so make it before any stream capture; the address is kept until
 * exit, so do not use this entry across a cudaDeviceReset of that device.
 * A CUDA error already pending when the call is made is reported (and left
 * pending) without launching anything.  Calls share the array: calls that
 * overlap on the GPU race, so serialise them (one stream).
 *   U      device pointer, U(nx, nyg, nzg) in Fortran order
 *   yg     device pointer, yg(1:nyg)
 *   qflow  device pointer to one double: Int_U / norm
 *   stream cudaStream_t to launch on (NULL: the legacy default stream)
 * Errors are reported through c3d_last_error(0).                            */
int c3d_mean_mass_flow_u_noalloc(const double* U, int nx, int nyg, int nzg,
                                 const double* yg, double* qflow, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* C3D_H */
