// Immersed-boundary state shared by the IB operators (k_ib.cu) and the
// learned preconditioner (k_mlp.cu).
#pragma once
#include <string>
#include <vector>

#include "c3d_internal.cuh"

namespace c3d {

struct BandState;   // banded z-Fourier preconditioner (k_ib_band.cu)

struct IbState {
  std::string kind;
  bool moving = false;
  int nb = 0, nbodies = 0;
  // host geometry
  std::vector<double> xb, yb, zb, ub, nrm, sb;
  std::vector<double> tan1, tan2;   // tangents_1, tangents_2 (3*nb; written to snapshots only)
  std::vector<int> yref, body;
  std::vector<int> body_count;
  // device geometry
  double *xb_d = nullptr, *yb_d = nullptr, *zb_d = nullptr, *ub_d = nullptr, *nrm_d = nullptr, *sb_d = nullptr;
  int *yref_d = nullptr, *body_d = nullptr;
  double* binv_d = nullptr;          // 1/markers per body
  // page-locked staging of the geometry uploads; stage_ev marks the end of
  // the last upload from it
  char* stage_h = nullptr;
  size_t stage_bytes = 0;
  cudaEvent_t stage_ev = nullptr;
  // 1-D grids (Fortran-indexed) for the weight kernel
  double *x_d = nullptr, *y_d = nullptr, *z_d = nullptr, *xm_d = nullptr, *ym_d = nullptr, *zm_d = nullptr;
  bool grids_current = false;      // the device grids match the handle's (set_grid clears it)
  // operator tables: [type(4)][axis(3)][a(5)][nb]
  int* idx_d = nullptr;
  double* w1_d = nullptr;
  double* off_d = nullptr;
  int* flag_d = nullptr;
  // inverse maps of the u, v, w stencils for the spreading gather
  int* sp_cnt[3] = {nullptr, nullptr, nullptr};
  int* sp_off[3] = {nullptr, nullptr, nullptr};
  uint32_t* sp_ent[3] = {nullptr, nullptr, nullptr};
  double* sp_w[3] = {nullptr, nullptr, nullptr};
  int* sp_sums = nullptr;            // prefix-sum chunk totals
  double* amp = nullptr;             // [3][nb] spread amplitudes
  // fields
  double *Ureg = nullptr, *Vreg = nullptr, *Wreg = nullptr;
  double *Hu = nullptr, *Hv = nullptr, *Hw = nullptr;     // interior Heaviside
  double *Hce = nullptr;                                  // Hc exterior (rhs_p extents)
  double *Ut = nullptr, *Vt = nullptr, *Wt = nullptr;     // scratch fields
  // marker vectors
  double *fb = nullptr, *E1nHc = nullptr, *E1nH = nullptr;
  double *rhs = nullptr, *scr0 = nullptr, *scr1 = nullptr, *scr2 = nullptr;
  double *r = nullptr, *rhat = nullptr, *p = nullptr, *nu = nullptr, *ph = nullptr, *s = nullptr;
  double *sh = nullptr, *t = nullptr;
  double* red = nullptr;             // partial sums
  double* sc = nullptr;              // BiCGSTAB scalars
  unsigned* ticket = nullptr;        // last-block counter of the body sums
  int iy_lo = 1, iy_hi = 1 << 30;    // y rows touched by any stencil
  // marker lattice: index = ix + lat_nx * iz (every body type lays its markers
  // out row by row); lat_nx = nb when there is no second direction
  int lat_nx = 0;
  // preconditioner: per-marker 4x4 blocks [nb][4][4] acting on
  // (r[b], r[nb+b], r[2nb+b], r[3nb+b]); the Jacobi blocks are diagonal
  double* jac_blk = nullptr;
  double* spai_blk = nullptr;        // probed block sparse approximate inverse
  double* prb = nullptr;             // [4][4nb] probe responses of one colour class
  bool have_jac = false, have_lrn = false;
  std::vector<double> yb_at_jac;     // marker y when the Jacobi diagonal was probed
  int jac_clipped[4] = {0, 0, 0, 0}; // safeguarded diagonal entries per component
  double dt_at_jac = 0;
  BandState* band = nullptr;         // banded z-Fourier preconditioner
  // warm start of the learned mode: the last solutions of each RK stage
  // (newest first) and the stage of the solve in progress (-1: none)
  static constexpr int kHist = 4;
  double* hist[3][kHist] = {};
  int nhist[3] = {0, 0, 0};
  int stage = -1;
  int warm_order = -1;               // extrapolation order of the last warm start
  // LEARNED against the probed band: iterations per solve of the recent
  // BAND solves, and consecutive LEARNED solves that were slow against them
  double band_iters_ref = 0.0;
  int lrn_slow = 0;
  // marker positions and dt when the network last predicted the band: like
  // the probed band it is predicted again once a marker moved 0.03 dymin
  std::vector<double> yb_at_lrn, xb_at_lrn;
  double dt_at_lrn = 0.0;
  double* ext_part = nullptr;        // block partials of the extrapolation errors
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;   // Schur-solve timing
  // the BiCGSTAB iteration loop as a CUDA graph (a conditional WHILE node
  // whose body is one iteration), rebuilt when what it bakes in changes
  cudaGraph_t bcg_graph = nullptr;
  cudaGraphExec_t bcg_exec = nullptr;
  std::vector<double> bcg_key;       // mode, factors, operands, dt, tolerance, stencil rows
  int64_t bcg_body_launches = 0;     // kernels in one iteration
  bool bcg_graph_off = false;        // conditional graphs unavailable: host-driven loop
  int* loop_d = nullptr;             // [0] iterations done, [1] limit of this launch
  double* hist_d = nullptr;          // squared residual after each iteration
  int hist_cap = 0;
  ~IbState() {
    if (bcg_exec) cudaGraphExecDestroy(bcg_exec);
    if (bcg_graph) cudaGraphDestroy(bcg_graph);
    if (ev_a) cudaEventDestroy(ev_a);
    if (ev_b) cudaEventDestroy(ev_b);
  }
};


// learned-preconditioner entry points used by the Schur solver (k_mlp.cu):
// the band factors from the network's prediction at the current geometry,
// and, while collection is on, a training set from each probed band
bool learned_stale(Handle* h, double dt);
int mlp_prepare_band(Handle* h);
int mlp_build_band(Handle* h, double dt);
bool mlp_collecting(const Handle* h);
int mlp_add_probe_set(Handle* h);
// probe pass of the Schur operator (k_ib.cu): Jacobi and SPAI blocks, and,
// when mom is not null, per-marker SPAI moments [nb][36]
int ib_probe(Handle* h, double dt, float* mom);
// banded z-Fourier preconditioner (k_ib_band.cu): supported lattices, build
// by probing, staleness after the geometry moved, application out = B^-1 in
bool band_supported(Handle* h);
int band_build(Handle* h, double dt);
bool band_stale(Handle* h, double dt);
void band_invalidate(Handle* h);
int band_apply(Handle* h, const double* in, double* out);
bool band_is_block(Handle* h);
struct BandView {
  int lat = 0, nzl = 0, nq = 0;   // lattice columns, z rows, z wavenumbers 0..nzl/2
  const int* nbr = nullptr;       // [lat][5] neighbour columns d = -2..2
  double2* That = nullptr;        // [nq][80 lat] band symbol, L = ((cp lat + i1) 5 + d) 4 + c
};
BandView band_view(Handle* h);
int band_factor_symbol(Handle* h, double dt);
int band_probe_count(Handle* h);
void band_free(IbState* s);

}  // namespace c3d
