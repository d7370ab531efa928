// Immersed boundary: geometry, delta-function operators, Heaviside fields,
// Schur complement, BiCGSTAB and the IB projection.
//
// Restates src/immersed_boundary_geometry.f90, src/immersed_boundary_operators.f90,
// src/heaviside.f90 and src/projection.f90:48-186 for one GPU:
//  - marker geometry is evaluated on the host with the reference formulas and
//    uploaded (once for static bodies, every RK stage for moving ones);
//  - the Yang3 weights are a tensor product, so setup_IB_operators keeps per
//    marker and per location (u, v, w, centre) the 5 one-dimensional delta
//    values, grid offsets and folded grid indices of each axis; a stencil
//    weight is dx*dymin*dz*dx_w*dy_w*dz_w in the reference's multiplication
//    order;
//  - E / E1n gather one warp per (marker, component); R spreads with FP64
//    atomics (so R is order-dependent at round-off level);
//  - the reference's marker partition, support planes and MPI gathers are
//    replaced by direct indexing of the resident fields: a stencil point on
//    the periodic duplicate centre plane nzg-1 is folded onto plane 2.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <climits>
#include "c3d_internal.cuh"
#include "ib_state.cuh"

namespace c3d {

static const double kPiIb = 4.0 * std::atan(1.0);

// ---------------------------------------------------------------------------
// host geometry: setup_IB_geometry (src/immersed_boundary_geometry.f90:70-398)
// ---------------------------------------------------------------------------
static int geometry_host(Handle* h, IbState* s, double t, std::string& err) {
  const Params& p = h->p;
  const int nxb = p.nxb, nzb = p.nzb;
  const double Lxp = h->Lxp, Lzp = h->Lzp;
  // every body type writes the same entries at every time, so the arrays
  // are cleared only when their size changes
  auto resize = [&](int nb) {
    if (s->nb != nb || (int)s->xb.size() != nb) {
      s->nb = nb;
      s->xb.assign(nb, 0); s->yb.assign(nb, 0); s->zb.assign(nb, 0);
      s->ub.assign(3 * nb, 0); s->nrm.assign(3 * nb, 0); s->sb.assign(nb, 0);
      s->tan1.assign(3 * nb, 0); s->tan2.assign(3 * nb, 0);
      s->yref.assign(nb, 1); s->body.assign(nb, 0);
    }
    s->lat_nx = nb;
  };
  // Lattices whose markers differ from row to row only in z (every value
  // but zb depends on the x index and the time): the first row is computed
  // and copied to the others, zb set per row.
  auto replicate_rows = [&](int rl, int nrows, double dzb) {
    const int nb = s->nb;
    for (int j = 2; j <= nrows; ++j) {
      const int o = rl * (j - 1);
      std::copy(s->xb.begin(), s->xb.begin() + rl, s->xb.begin() + o);
      std::copy(s->yb.begin(), s->yb.begin() + rl, s->yb.begin() + o);
      std::copy(s->sb.begin(), s->sb.begin() + rl, s->sb.begin() + o);
      std::copy(s->yref.begin(), s->yref.begin() + rl, s->yref.begin() + o);
      std::copy(s->body.begin(), s->body.begin() + rl, s->body.begin() + o);
      for (int c = 0; c < 3; ++c)
        for (std::vector<double>* v : {&s->ub, &s->nrm, &s->tan1, &s->tan2})
          std::copy(v->begin() + (size_t)c * nb, v->begin() + (size_t)c * nb + rl, v->begin() + (size_t)c * nb + o);
      for (int e = 0; e < rl; ++e) s->zb[o + e] = ((double)j - 0.5) * dzb;
    }
  };
  if (s->kind == "center_wall") {                                     // :80-115
    if (p.grid_type != 0) { err = "Error: body type is incompatible with grid type"; return C3D_ERR_PARAM; }
    const int nb = nxb * nzb;
    resize(nb);
    s->lat_nx = nxb;
    const double dxb = Lxp / nxb, dzb = Lzp / nzb;
    for (int j = 1; j <= nzb; ++j)
      for (int i = 1; i <= nxb; ++i) {
        const int k = i + (j - 1) * nxb - 1;
        s->xb[k] = ((double)i - 0.5) * dxb;
        s->yb[k] = 0.5 * p.Ly_channel;
        s->zb[k] = ((double)j - 0.5) * dzb;
        s->yref[k] = p.ny_global / 2;
      }
    for (int k = 0; k < nb; ++k) {                                  // :108-115
      s->sb[k] = dxb * dzb;
      s->nrm[nb + k] = -1.0;
      s->tan1[k] = 1.0;
      s->tan2[2 * nb + k] = -1.0;
    }
    s->nbodies = 1;
  } else if (s->kind == "standing_wave" || s->kind == "wall_standing_wave") {   // :176-269
    const bool two = (s->kind == "standing_wave");
    if (two && p.body_param_1 > p.min_buffer_width) {
      err = "Error: IB amplitude is bigger than the minimum buffer width";
      return C3D_ERR_PARAM;
    }
    const int nw = two ? 2 : 1;
    const int nb = nw * nxb * nzb;
    resize(nb);
    s->lat_nx = nw * nxb;
    const double dxb = Lxp / nxb, dzb = Lzp / nzb;
    const double A = p.body_param_1, om = p.body_param_2, b3 = p.body_param_3;
    const double y0 = two ? 0.0 : p.body_param_4;
    for (int j = 1; j <= 1; ++j)   // the first row (replicate_rows copies it)
      for (int i = 1; i <= nxb; ++i) {
        const int k = i + nw * nxb * (j - 1) - 1;
        const double x = ((double)i - 0.5) * dxb;
        s->xb[k] = x;
        s->yb[k] = y0 + A * std::sin(2.0 * kPiIb * b3 * x / Lxp) * std::cos(om * t);
        s->zb[k] = ((double)j - 0.5) * dzb;
        s->yref[k] = 1;
        s->body[k] = 0;
        if (two) {
          s->xb[k + nxb] = x;
          s->yb[k + nxb] = p.Ly_channel + A * std::sin(2.0 * kPiIb * b3 * x / Lxp) * std::cos(om * t);
          s->zb[k + nxb] = ((double)j - 0.5) * dzb;
          s->yref[k + nxb] = p.ny_global;
          s->body[k + nxb] = 1;
        }
      }
    for (int j = 1; j <= 1; ++j)   // the first row (replicate_rows copies it)
      for (int i = 1; i <= nxb; ++i) {
        const int k = i + nw * nxb * (j - 1) - 1;
        const double phase = 2.0 * kPiIb * b3 * s->xb[k] / Lxp;
        const double vy = -A * om * std::sin(phase) * std::sin(om * t);
        const double slope = A * 2.0 * kPiIb * b3 / Lxp * std::cos(phase) * std::cos(om * t);
        const double t1x = 1.0 / std::sqrt(1.0 + slope * slope);
        const double t1y = slope / std::sqrt(1.0 + slope * slope);
        s->ub[nb + k] = vy;
        s->nrm[k] = t1y;
        s->nrm[nb + k] = -t1x;
        s->tan1[k] = t1x;                                            // :236-244
        s->tan1[nb + k] = t1y;
        s->tan2[2 * nb + k] = 1.0;
        if (two) {
          s->ub[nb + k + nxb] = vy;
          s->nrm[k + nxb] = -t1y;
          s->nrm[nb + k + nxb] = t1x;
          s->tan1[k + nxb] = t1x;
          s->tan1[nb + k + nxb] = t1y;
          s->tan2[2 * nb + k + nxb] = 1.0;
        }
      }
    for (int j = 1; j <= 1; ++j)   // the first row (replicate_rows copies it)
      for (int i = 1; i <= nxb; ++i) {
        const int k = i + nw * nxb * (j - 1) - 1;
        const int first = nw * nxb * (j - 1), last = nxb - 1 + nw * nxb * (j - 1);
        const auto& X = s->xb;
        const auto& Y = s->yb;
        double a1, a2;
        if (i == 1) {
          a1 = std::sqrt(std::pow(X[k] - (X[last] - Lxp), 2) + std::pow(Y[k] - Y[last], 2));
          a2 = std::sqrt(std::pow(X[k] - X[k + 1], 2) + std::pow(Y[k] - Y[k + 1], 2));
        } else if (i == nxb) {
          a1 = std::sqrt(std::pow(X[k] - X[k - 1], 2) + std::pow(Y[k] - Y[k - 1], 2));
          a2 = std::sqrt(std::pow(X[k] - (X[first] + Lxp), 2) + std::pow(Y[k] - Y[first], 2));
        } else {
          a1 = std::sqrt(std::pow(X[k] - X[k - 1], 2) + std::pow(Y[k] - Y[k - 1], 2));
          a2 = std::sqrt(std::pow(X[k] - X[k + 1], 2) + std::pow(Y[k] - Y[k + 1], 2));
        }
        s->sb[k] = dzb * (0.5 * a1 + 0.5 * a2);
        if (two) s->sb[k + nxb] = dzb * (0.5 * a1 + 0.5 * a2);
      }
    replicate_rows(nw * nxb, nzb, dzb);
    s->nbodies = nw;
  } else if (s->kind == "traveling_wave_x") {                          // :271-390
    const int nb = 2 * nxb * nzb;
    resize(nb);
    s->lat_nx = 2 * nxb;
    const double dxb = Lxp / nxb, dzb = Lzp / nzb;
    const double b1 = p.body_param_1, b2 = p.body_param_2, b3 = p.body_param_3, tr = p.body_ramp_up_time;
    double amp, damp;
    if (t < tr && tr > 0.0) {
      const double tau = t / tr;
      amp = b1 * 0.5 * (1.0 - std::cos(kPiIb * tau));
      damp = b1 * 0.5 * (kPiIb / tr) * std::sin(kPiIb * tau);
    } else { amp = b1; damp = 0.0; }
    const double phi = kPiIb;
    for (int j = 1; j <= 1; ++j)   // the first row (replicate_rows copies it)
      for (int i = 1; i <= nxb; ++i) {
        const int k = i + 2 * nxb * (j - 1) - 1;
        const double x = ((double)i - 0.5) * dxb;
        const double ph = b3 * (x - b2 * t);
        s->xb[k] = x; s->xb[k + nxb] = x;
        s->yb[k] = amp / (b2 * b3) * std::sin(ph);
        s->yb[k + nxb] = p.Ly_channel + amp / (b2 * b3) * std::sin(ph + phi);
        s->zb[k] = ((double)j - 0.5) * dzb; s->zb[k + nxb] = s->zb[k];
        s->yref[k] = 1; s->yref[k + nxb] = p.ny_global;
        s->body[k] = 0; s->body[k + nxb] = 1;
        s->ub[nb + k] = -amp * std::cos(ph) + (damp / (b2 * b3)) * std::sin(ph);
        s->ub[nb + k + nxb] = -amp * std::cos(ph + phi) + (damp / (b2 * b3)) * std::sin(ph + phi);
        const double sbot = amp / b2 * std::cos(ph), stop = amp / b2 * std::cos(ph + phi);
        const double tbx = 1.0 / std::sqrt(1.0 + sbot * sbot), tby = sbot / std::sqrt(1.0 + sbot * sbot);
        const double ttx = 1.0 / std::sqrt(1.0 + stop * stop), tty = stop / std::sqrt(1.0 + stop * stop);
        s->nrm[k] = tby; s->nrm[k + nxb] = -tty;
        s->nrm[nb + k] = -tbx; s->nrm[nb + k + nxb] = ttx;
        s->tan1[k] = tbx; s->tan1[k + nxb] = ttx;                    // :344-352
        s->tan1[nb + k] = tby; s->tan1[nb + k + nxb] = tty;
        s->tan2[2 * nb + k] = 1.0; s->tan2[2 * nb + k + nxb] = 1.0;
      }
    for (int j = 1; j <= 1; ++j)   // the first row (replicate_rows copies it)
      for (int i = 1; i <= nxb; ++i)
        for (int wall = 0; wall < 2; ++wall) {
          const int k = i + wall * nxb + 2 * nxb * (j - 1) - 1;
          const int first = wall * nxb + 2 * nxb * (j - 1), last = nxb - 1 + wall * nxb + 2 * nxb * (j - 1);
          const auto& X = s->xb;
          const auto& Y = s->yb;
          double a1, a2;
          if (i == 1) {
            a1 = std::sqrt(std::pow(X[k] - (X[last] - Lxp), 2) + std::pow(Y[k] - Y[last], 2));
            a2 = std::sqrt(std::pow(X[k] - X[k + 1], 2) + std::pow(Y[k] - Y[k + 1], 2));
          } else if (i == nxb) {
            a1 = std::sqrt(std::pow(X[k] - X[k - 1], 2) + std::pow(Y[k] - Y[k - 1], 2));
            a2 = std::sqrt(std::pow(X[k] - (X[first] + Lxp), 2) + std::pow(Y[k] - Y[first], 2));
          } else {
            a1 = std::sqrt(std::pow(X[k] - X[k - 1], 2) + std::pow(Y[k] - Y[k - 1], 2));
            a2 = std::sqrt(std::pow(X[k] - X[k + 1], 2) + std::pow(Y[k] - Y[k + 1], 2));
          }
          s->sb[k] = dzb * (0.5 * a1 + 0.5 * a2);
        }
    replicate_rows(2 * nxb, nzb, dzb);
    s->nbodies = 2;
  } else if (s->kind == "double_cylinders_z") {                         // :117-174
    if (p.grid_type != 0) { err = "Error: body type is incompatible with grid type"; return C3D_ERR_PARAM; }
    const double r1 = p.body_param_1, r2 = p.body_param_2;
    const double dzb = Lzp / nzb;
    const double dxb = dzb * h->dx / h->dz;
    const int nxb1 = (int)(2 * 3.14159 * r1 / dxb), nxb2 = (int)(2 * 3.14159 * r2 / dxb);
    const int nxbt = nxb1 + nxb2;
    const int nb = nxbt * nzb;
    resize(nb);
    s->lat_nx = nxbt;
    const double xc = 0.5 * Lxp, yc = 0.5 * p.Ly_channel;
    const double dsb1 = 2 * 3.14159 * r1 / nxb1, dsb2 = 2 * 3.14159 * r2 / nxb2;
    for (int j = 1; j <= nzb; ++j) {
      for (int i = 1; i <= nxb1; ++i) {
        const int k = i + (j - 1) * nxbt - 1;
        const double th = (double)(i - 1) * dsb1 / r1;
        s->xb[k] = r1 * std::cos(th) + xc;
        s->yb[k] = r1 * std::sin(th) + yc;
        s->zb[k] = ((double)j - 0.5) * dzb;
        s->ub[k] = -std::sin(th) * p.body_param_3;
        s->ub[nb + k] = std::cos(th) * p.body_param_3;
        s->sb[k] = dsb1 * dzb;
        s->nrm[k] = -std::cos(th);
        s->nrm[nb + k] = -std::sin(th);
        s->tan1[k] = std::sin(th);                                   // :146-147
        s->tan1[nb + k] = -std::cos(th);
        s->body[k] = 0;
      }
      for (int i = 1; i <= nxb2; ++i) {
        const int k = i + (j - 1) * nxbt + nxb1 - 1;
        const double th = (double)(i - 1) * dsb2 / r2;
        s->xb[k] = r2 * std::cos(th) + xc;
        s->yb[k] = r2 * std::sin(th) + yc;
        s->zb[k] = ((double)j - 0.5) * dzb;
        s->sb[k] = dsb2 * dzb;
        s->nrm[k] = std::cos(th);
        s->nrm[nb + k] = std::sin(th);
        s->tan1[k] = -std::sin(th);                                  // :160-161
        s->tan1[nb + k] = std::cos(th);
        s->body[k] = 1;
      }
    }
    for (int k = 0; k < nb; ++k) s->tan2[2 * nb + k] = 1.0;         // :164-166
    s->nbodies = 2;
  } else if (s->kind == "two_cylinders_z") {
    // extension: two separate spanwise cylinders of radius body_param_1,
    // counter-rotating with surface speeds +-body_param_2, centred at
    // (body_param_3, Ly/2) and (2 body_param_3, Ly/2 + body_param_4); nxb
    // markers around each, nzb spanwise; conventions of double_cylinders_z
    // (src/immersed_boundary_geometry.f90:117-174): normals point out of the
    // fluid (into each cylinder), sb = arc length x dz, one body per cylinder
    if (p.grid_type != 0) { err = "Error: body type is incompatible with grid type"; return C3D_ERR_PARAM; }
    const double r = p.body_param_1, us = p.body_param_2;
    const double dzb = Lzp / nzb, dsb = 2.0 * kPiIb * r / nxb;
    const int nb = 2 * nxb * nzb;
    resize(nb);
    s->lat_nx = 2 * nxb;
    const double xc[2] = {p.body_param_3, 2.0 * p.body_param_3};
    const double yc[2] = {0.5 * p.Ly_channel, 0.5 * p.Ly_channel + p.body_param_4};
    const double sgn[2] = {1.0, -1.0};
    for (int j = 1; j <= nzb; ++j)
      for (int c = 0; c < 2; ++c)
        for (int i = 1; i <= nxb; ++i) {
          const int k = i + c * nxb + 2 * nxb * (j - 1) - 1;
          const double th = (double)(i - 1) * 2.0 * kPiIb / nxb;
          s->xb[k] = xc[c] + r * std::cos(th);
          s->yb[k] = yc[c] + r * std::sin(th);
          s->zb[k] = ((double)j - 0.5) * dzb;
          s->ub[k] = -sgn[c] * us * std::sin(th);
          s->ub[nb + k] = sgn[c] * us * std::cos(th);
          s->sb[k] = dsb * dzb;
          s->nrm[k] = -std::cos(th);
          s->nrm[nb + k] = -std::sin(th);
          s->tan1[k] = std::sin(th);
          s->tan1[nb + k] = -std::cos(th);
          s->tan2[2 * nb + k] = 1.0;
          s->body[k] = c;
        }
    s->nbodies = 2;
  } else if (s->kind == "wall_plates") {
    // extension: nxb x nzb thin plates standing on the lower wall, height
    // h = body_param_1, width half the spanwise pitch, 32 x 16 markers each
    // (up x across); plate (pi, pj) bends in x with the tip displacement
    // a sin(omega t + phi), a = body_param_2, omega = body_param_3, phase phi
    // from the splitmix64 stream seeded with body_param_4:
    //   x = x_p + a (y/h)^2 sin(omega t + phi),  u_b = d/dt of it,
    //   n = (1, -dx/dy, 0)/|.|,  32 marker rows from y0 = 3 dymin (the
    //   lowest height whose delta stencil stays above the wall) to the tip h.
    // Marker (k, m) of plate (pi, pj) sits at lattice (ix, iz) =
    // ((pi-1)*32 + k-1, (pj-1)*16 + m-1); all plates form one body.
    constexpr int my = 32, mz = 16;
    const double hh = p.body_param_1, amp = p.body_param_2, om = p.body_param_3;
    const double pitchx = Lxp / nxb, pitchz = Lzp / nzb, wz = 0.5 * pitchz;
    const int nb = nxb * nzb * my * mz;
    resize(nb);
    s->lat_nx = nxb * my;
    uint64_t st = (uint64_t)(int64_t)std::llround(p.body_param_4);
    std::vector<double> phase(nxb * nzb);
    for (auto& ph : phase) {
      st += 0x9E3779B97F4A7C15ull;
      uint64_t z = st;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      ph = 2.0 * kPiIb * (double)(z >> 11) * (1.0 / 9007199254740992.0);
    }
    std::vector<double> psn(nxb * nzb), pcs(nxb * nzb);   // per plate: sin, cos(omega t + phi)
    for (int e = 0; e < nxb * nzb; ++e) {
      psn[e] = std::sin(om * t + phase[e]);
      pcs[e] = std::cos(om * t + phase[e]);
    }
    for (int pj = 1; pj <= nzb; ++pj)
      for (int m = 1; m <= mz; ++m)
        for (int pi = 1; pi <= nxb; ++pi)
          for (int kk = 1; kk <= my; ++kk) {
            const int ix = (pi - 1) * my + kk - 1, iz = (pj - 1) * mz + m - 1;
            const int k = ix + s->lat_nx * iz;
            const double y0 = 3.0 * h->dymin;
            const double y = y0 + (kk - 1) * (hh - y0) / (my - 1), eta = y / hh;
            const double sn = psn[(pi - 1) + nxb * (pj - 1)], cs = pcs[(pi - 1) + nxb * (pj - 1)];
            s->xb[k] = (pi - 0.5) * pitchx + amp * eta * eta * sn;
            s->yb[k] = y;
            s->zb[k] = (pj - 0.5) * pitchz + ((double)m - 0.5 - 0.5 * mz) * (wz / mz);
            s->ub[k] = amp * eta * eta * om * cs;
            const double slope = 2.0 * amp * y / (hh * hh) * sn;
            const double nn = std::sqrt(1.0 + slope * slope);
            s->nrm[k] = 1.0 / nn;
            s->nrm[nb + k] = -slope / nn;
            s->tan1[k] = slope / nn;                                    // along the plate, up
            s->tan1[nb + k] = 1.0 / nn;
            s->tan2[2 * nb + k] = 1.0;
            s->sb[k] = ((hh - 3.0 * h->dymin) / (my - 1)) * (wz / mz);
            s->yref[k] = 1;
            s->body[k] = 0;
          }
    s->nbodies = 1;
  } else {
    err = "Error: No corresponding body type found for: " + s->kind;
    return C3D_ERR_PARAM;
  }
  // the stencil must stay inside the y grid (the reference stops on
  // src/immersed_boundary_geometry.f90:198-213 and :595-598)
  const int ny = h->d.ny, nym = h->d.Ny;
  for (int l = 0; l < s->nb; ++l) {
    const int yr = s->yref[l];
    const double yrv = h->y[yr];
    const int yp = (int)std::floor((s->yb[l] - yrv) / h->dymin) + yr;
    const int ymp = (int)std::floor((s->yb[l] - (yrv + 0.5 * h->dymin)) / h->dymin) + yr;
    if (yp - 2 < 1 || yp + 2 > ny || ymp - 2 < 1 || ymp + 2 > nym) {
      err = "Error: body points support exceeds grid dimensions (marker " + std::to_string(l + 1) + ")";
      return C3D_ERR_PARAM;
    }
  }
  s->body_count.assign(s->nbodies, 0);
  for (int l = 0; l < s->nb; ++l) s->body_count[s->body[l]]++;
  return 0;
}

// ---------------------------------------------------------------------------
// device weights: setup_IB_operators (src/immersed_boundary_operators.f90:19-256)
// ---------------------------------------------------------------------------
__device__ double delta_yang3(double x1, double x2, double dr) {
  const double r = fabs(x1 - x2);
  const double r1 = r / dr;
  const double r2 = r1 * r1;
  const double s3 = 1.7320508075688772;   // sqrt(3)
  const double pi = 3.141592653589793;
  double v;
  if (r1 <= 1.0) {
    v = 17.0 / 48.0 + s3 * pi / 108.0 + r1 / 4.0 - r2 / 4.0 +
        (1.0 - 2.0 * r1) / 16.0 * sqrt(-12.0 * r2 + 12.0 * r1 + 1.0) -
        s3 / 12.0 * asin(s3 / 2.0 * (2.0 * r1 - 1.0));
  } else if (r1 <= 2.0) {
    v = 55.0 / 48.0 - s3 * pi / 108.0 - 13.0 * r1 / 12.0 + r2 / 4.0 +
        (2.0 * r1 - 3.0) / 48.0 * sqrt(-12.0 * r2 + 36.0 * r1 - 23.0) +
        s3 / 36.0 * asin(s3 / 2.0 * (2.0 * r1 - 3.0));
  } else {
    v = 0.0;
  }
  return v / dr;
}

struct IbGeomArgs {
  Dims d;
  int nb;
  const double *xb, *yb, *zb;
  const int* yref;
  const double *x, *y, *z, *xm, *ym, *zm;
  double dx, dz, dymin, Lxp, Lzp;
  int* idx;
  double* w1;
  double* off;
  int* flag;
};

// table slot of (type t, axis a, point q, marker l)
__host__ __device__ inline int64_t tslot(int nb, int t, int a, int q, int l) {
  return (((int64_t)t * 3 + a) * 5 + q) * nb + l;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi, int* flag) {
  if (v < lo) { *flag = 1; return lo; }
  if (v > hi) { *flag = 1; return hi; }
  return v;
}

__global__ void k_ib_weights(IbGeomArgs a) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.nb) return;
  const Dims& d = a.d;
  const int nxg_ = d.nx, nzg_ = d.nz;         // nx_global, nz_global
  const int nxm_ = d.nx - 1, nzm_ = d.nz - 1; // nxm_global, nzm_global
  const double xb = a.xb[l], yb = a.yb[l], zb = a.zb[l];
  const int yr = a.yref[l];
  const double yrv = a.y[yr];
  const int x_piv = (int)floor(xb / a.dx) + 1;
  const int xm_piv = (int)floor((xb + 0.5 * a.dx) / a.dx);
  const int y_piv = (int)floor((yb - yrv) / a.dymin) + yr;
  const int ym_piv = (int)floor((yb - (yrv + 0.5 * a.dymin)) / a.dymin) + yr;
  const int z_piv = (int)floor(zb / a.dz) + 1;
  const int zm_piv = (int)floor((zb + 0.5 * a.dz) / a.dz) + 1;
  int* flag = a.flag;
  for (int t = 0; t < 4; ++t) {      // 0 u, 1 v, 2 w, 3 centre
    for (int q = 0; q < 5; ++q) {
      const int o = q - 2;
      // ---- x
      int ix;
      double xg;
      if (t == 0) {
        const int ii = x_piv + o;
        const int sh = (int)floor((double)(ii - 1) / (double)(nxg_ - 2));
        const int iip = clampi(ii - sh * (nxg_ - 2), 1, nxg_ - 2, flag);
        ix = (iip == 1) ? nxg_ - 1 : iip;
        xg = a.x[iip] + sh * a.Lxp;
      } else {
        const int ii = xm_piv + o - (t == 2 ? 1 : 0);
        const int sh = (int)floor((double)(ii - 1) / (double)(nxm_ - 1));
        const int iip = clampi(ii - sh * (nxm_ - 1), 1, nxm_ - 1, flag);
        ix = iip + 1;
        xg = a.xm[iip] + sh * a.Lxp;
      }
      // ---- y
      int iy;
      double yg;
      if (t == 1) {
        const int jj = clampi(y_piv + o, 1, d.ny, flag);
        iy = jj;
        yg = a.y[jj];
      } else {
        const int jj = clampi(ym_piv + o, 1, d.Ny, flag);
        iy = jj + 1;
        yg = a.ym[jj];
      }
      // ---- z
      int iz;
      double zg;
      if (t == 2) {
        const int kk = z_piv + o;
        const int sh = (int)floor((double)(kk - 2) / (double)(nzg_ - 2));
        const int kkp = clampi(kk - sh * (nzg_ - 2), 2, nzg_ - 1, flag);
        iz = kkp;
        zg = a.z[kkp] + sh * a.Lzp;
      } else {
        const int kk = zm_piv + o;
        const int sh = (int)floor((double)(kk - 2) / (double)nzm_);
        const int kkp = clampi(kk - sh * (nzm_ - 1), 2, nzm_ + 1, flag);
        iz = (kkp == d.nzg - 1) ? 2 : kkp;       // duplicate plane nzg-1 is plane 2
        zg = a.zm[kkp - 1] + sh * a.Lzp;
      }
      a.idx[tslot(a.nb, t, 0, q, l)] = ix;
      a.idx[tslot(a.nb, t, 1, q, l)] = iy;
      a.idx[tslot(a.nb, t, 2, q, l)] = iz;
      a.w1[tslot(a.nb, t, 0, q, l)] = delta_yang3(xg, xb, a.dx);
      a.w1[tslot(a.nb, t, 1, q, l)] = delta_yang3(yg, yb, a.dymin);
      a.w1[tslot(a.nb, t, 2, q, l)] = delta_yang3(zg, zb, a.dz);
      a.off[tslot(a.nb, t, 0, q, l)] = xg - xb;
      a.off[tslot(a.nb, t, 1, q, l)] = yg - yb;
      a.off[tslot(a.nb, t, 2, q, l)] = zg - zb;
    }
  }
}

// ---------------------------------------------------------------------------
// gather (E, E1n) and spread (R)
// ---------------------------------------------------------------------------
struct OpTables {
  int nb;
  const int* idx;
  const double* w1;
  const double* off;
  const double* nrm;
  const double* sb;
  double scale;    // dx*dymin*dz
  double factor;   // 1/(dx*dymin*dz)
};

// field description for a gather
struct GField {
  const double* F;    // field (U/V/W extents, or rhs_p extents when rhsp)
  int n1, n2;         // extents of dims 1 and 2
  int rhsp;           // 1: index with rhs_p lower bounds (2,2,2)
  double mul;         // value multiplier
};

enum GatherMode { G_E = 0, G_E1N = 1 };

// one component of a gather: its field, stencil table and epilogue
// out[c*nb + l] = sign * gathered - sub[i] * subv[i] + addv[i], i = c*nb + l
struct GComp {
  GField f;
  int type;           // table type: 0 u, 1 v, 2 w, 3 centre
  int mode;           // G_E or G_E1N
  double sign;
  const double* sub;  // optional (with subv)
  const double* subv;
  const double* addv; // optional
};

struct GatherArgs {
  OpTables T;
  Dims d;
  GComp comp[4];      // blockIdx.y picks the component
  int ncomp;
  double* out;
};

__device__ __forceinline__ int64_t lin(int n1, int n2, int i, int j, int k, int rhsp) {
  if (rhsp) return (int64_t)(i - 2) + (int64_t)n1 * ((j - 2) + (int64_t)n2 * (k - 2));
  return (int64_t)(i - 1) + (int64_t)n1 * ((j - 1) + (int64_t)n2 * (k - 1));
}

// Gather of grid values to the markers, E (src/immersed_boundary_operators.f90
// regT) and E1n (regT_1n, weights times the stencil point's offset along the
// normal), with the field box of a tile of markers staged in shared memory: a
// CTA takes kTileMarkers consecutive markers of one component (one thread
// each), finds the box of grid points their stencils touch (periodic x and z
// indices unwrapped around the tile's first marker), copies that box from the
// field once (consecutive threads along x, eight loads in flight) and gathers
// from shared memory.  Per stencil row (qj, qk) the thread forms the row sums
// s0 = sum_qi wx v and, for E1n, s1 = sum_qi wx ox v, and adds
// scale wy wz (s1 + (oy + oz) s0) -- the regT / regT_1n sums
// (src/immersed_boundary_operators.f90) regrouped by rows.  A stencil point of
// zero weight reads a point inside the box and adds an exact zero.  A tile
// whose box does not fit gathers from the field directly.
constexpr int kTileMarkers = 64;
constexpr int kTileBox = 3072;     // doubles of shared memory for the box (24 KB)
// Components of both variants may share one launch (the Schur operator's
// E1n of phi beside the three E components); each CTA runs one variant.
template <bool E1N>
__device__ __forceinline__ void gather_tile(const GatherArgs& a, const GComp& cp, int c, double* box,
                                            int* s_ref, int* s_lo, int* s_hi) {
  const int nb = a.T.nb;
  const int tid = threadIdx.x;
  const int l = blockIdx.x * kTileMarkers + tid;
  const bool valid = l < nb;
  const int t = cp.type;
  const OpTables& T = a.T;
  const GField& g = cp.f;
  const int px = a.d.Nx, pz = a.d.Nz;        // index periods of x and z (indices 2 .. N+1)
  if (tid == 0) {
    const int l0 = blockIdx.x * kTileMarkers;
    s_ref[0] = T.idx[tslot(nb, t, 0, 2, l0)];
    s_ref[1] = T.idx[tslot(nb, t, 2, 2, l0)];
#pragma unroll
    for (int a3 = 0; a3 < 3; ++a3) { s_lo[a3] = INT_MAX; s_hi[a3] = INT_MIN; }
  }
  __syncthreads();
  const int rx = s_ref[0], rz = s_ref[1];
  auto unwrap = [](int i, int r, int p) {
    if (i - r > p / 2) return i - p;
    if (r - i > p / 2) return i + p;
    return i;
  };
  int ix[5], iy[5], iz[5];
  double wx[5], wy[5], wz[5];
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    ix[q] = iy[q] = iz[q] = 0;
    wx[q] = wy[q] = wz[q] = 0.0;
    if (valid) {
      ix[q] = unwrap(T.idx[tslot(nb, t, 0, q, l)], rx, px);
      iy[q] = T.idx[tslot(nb, t, 1, q, l)];
      iz[q] = unwrap(T.idx[tslot(nb, t, 2, q, l)], rz, pz);
      wx[q] = T.w1[tslot(nb, t, 0, q, l)];
      wy[q] = T.w1[tslot(nb, t, 1, q, l)];
      wz[q] = T.w1[tslot(nb, t, 2, q, l)];
    }
    if (wx[q] != 0.0) { lo[0] = min(lo[0], ix[q]); hi[0] = max(hi[0], ix[q]); }
    if (wy[q] != 0.0) { lo[1] = min(lo[1], iy[q]); hi[1] = max(hi[1], iy[q]); }
    if (wz[q] != 0.0) { lo[2] = min(lo[2], iz[q]); hi[2] = max(hi[2], iz[q]); }
  }
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[a3] = min(lo[a3], __shfl_xor_sync(0xffffffffu, lo[a3], o));
      hi[a3] = max(hi[a3], __shfl_xor_sync(0xffffffffu, hi[a3], o));
    }
    if ((tid & 31) == 0) { atomicMin(&s_lo[a3], lo[a3]); atomicMax(&s_hi[a3], hi[a3]); }
  }
  __syncthreads();
  const int bx0 = s_lo[0], by0 = s_lo[1], bz0 = s_lo[2];
  const bool any = s_hi[0] >= bx0 && s_hi[1] >= by0 && s_hi[2] >= bz0;
  const int bx = any ? s_hi[0] - bx0 + 1 : 0, by = any ? s_hi[1] - by0 + 1 : 0,
            bz = any ? s_hi[2] - bz0 + 1 : 0;
  const bool staged = any && bx <= 2 * kTileMarkers && (int64_t)bx * by * bz <= kTileBox;
  // periodic index back into 2 .. p+1 (one period away after the unwrap)
  auto wrap = [](int i, int p) {
    i = i < 2 ? i + p : (i > p + 1 ? i - p : i);
    if (i < 2 || i > p + 1) i = 2 + ((i - 2) % p + p) % p;
    return i;
  };
  auto field = [&](int i, int j, int k) { return g.F[lin(g.n1, g.n2, wrap(i, px), j, wrap(k, pz), g.rhsp)]; };
  if (staged) {
    // the box row by row (j fastest, then k), four rows per round with two
    // x points per thread and row: eight loads in flight
    const int nrow = by * bz;
    const int xa = wrap(bx0 + tid, px), xb = wrap(bx0 + tid + kTileMarkers, px);
    const bool ha = tid < bx, hb = tid + kTileMarkers < bx;
    int jj = 0, kk = 0;
    for (int r0 = 0; r0 < nrow; r0 += 4) {
      double ta[4], tb[4];
      int cj = jj, ck = kk;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        ta[u] = tb[u] = 0.0;
        if (r0 + u < nrow) {
          const int j = by0 + cj, k = wrap(bz0 + ck, pz);
          if (ha) ta[u] = g.F[lin(g.n1, g.n2, xa, j, k, g.rhsp)];
          if (hb) tb[u] = g.F[lin(g.n1, g.n2, xb, j, k, g.rhsp)];
        }
        if (++cj == by) { cj = 0; ++ck; }
      }
      jj = cj; kk = ck;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (r0 + u < nrow) {
          if (ha) box[tid + bx * (r0 + u)] = ta[u];
          if (hb) box[tid + kTileMarkers + bx * (r0 + u)] = tb[u];
        }
      }
    }
  }
  __syncthreads();
  if (!valid) return;
  double ox[5], oy[5], oz[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) ox[q] = oy[q] = oz[q] = 0.0;
  if (E1N) {
    const double nx_ = T.nrm[l], ny_ = T.nrm[nb + l], nz_ = T.nrm[2 * nb + l];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      ox[q] = nx_ * T.off[tslot(nb, t, 0, q, l)];
      oy[q] = ny_ * T.off[tslot(nb, t, 1, q, l)];
      oz[q] = nz_ * T.off[tslot(nb, t, 2, q, l)];
    }
  }
  double acc = 0.0;
  if (staged) {
    int offx[5], offy[5], offz[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {        // zero-weight points read the box's first point
      offx[q] = wx[q] != 0.0 ? ix[q] - bx0 : 0;
      offy[q] = wy[q] != 0.0 ? bx * (iy[q] - by0) : 0;
      offz[q] = wz[q] != 0.0 ? bx * by * (iz[q] - bz0) : 0;
    }
#pragma unroll
    for (int qk = 0; qk < 5; ++qk) {
#pragma unroll
      for (int qj = 0; qj < 5; ++qj) {
        const double* row = box + offy[qj] + offz[qk];
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int qi = 0; qi < 5; ++qi) {
          const double wv = wx[qi] * row[offx[qi]];
          s0 += wv;
          if (E1N) s1 = fma(wv, ox[qi], s1);
        }
        const double wjk = T.scale * wy[qj] * wz[qk];
        acc = fma(wjk, E1N ? fma(oy[qj] + oz[qk], s0, s1) : s0, acc);
      }
    }
  } else {
#pragma unroll 1
    for (int r = 0; r < 25; ++r) {
      const int qj = r % 5, qk = r / 5;
      double wyq = 0.0, wzq = 0.0, oyz = 0.0;
      int jy = 0, kz = 0;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        if (q == qj) { wyq = wy[q]; jy = iy[q]; oyz += oy[q]; }
        if (q == qk) { wzq = wz[q]; kz = iz[q]; oyz += oz[q]; }
      }
      if (wyq == 0.0 || wzq == 0.0) continue;
      double s0 = 0.0, s1 = 0.0;
#pragma unroll
      for (int qi = 0; qi < 5; ++qi) {
        if (wx[qi] == 0.0) continue;
        const double wv = wx[qi] * field(ix[qi], jy, kz);
        s0 += wv;
        if (E1N) s1 = fma(wv, ox[qi], s1);
      }
      acc = fma(T.scale * wyq * wzq, E1N ? fma(oyz, s0, s1) : s0, acc);
    }
  }
  double r = cp.sign * (acc * g.mul);
  const int i = c * nb + l;
  if (cp.sub) r -= cp.sub[i] * cp.subv[i];
  if (cp.addv) r += cp.addv[i];
  a.out[i] = r;
}

__global__ void __launch_bounds__(kTileMarkers) k_ib_gather_tile(GatherArgs a) {
  __shared__ double box[kTileBox];
  __shared__ int s_ref[2], s_lo[3], s_hi[3];
  const int c = blockIdx.y;
  const GComp& cp = a.comp[c];
  if (cp.mode == G_E1N) gather_tile<true>(a, cp, c, box, s_ref, s_lo, s_hi);
  else gather_tile<false>(a, cp, c, box, s_ref, s_lo, s_hi);
}

static void launch_gather_tile(const GatherArgs& a, cudaStream_t st) {
  const dim3 grid((a.T.nb + kTileMarkers - 1) / kTileMarkers, a.ncomp);
  k_ib_gather_tile<<<grid, kTileMarkers, 0, st>>>(a);
}

enum SpreadMode { S_RAW = 0, S_JUMP = 1, S_NORMAL = 2 };

// ---- spreading R f as a gather over an inverse map of the stencils ------
// The reference adds each marker's 125 stencil contributions to the field
// (local_reg, src/immersed_boundary_operators.f90:544-603).  Here every grid
// point sums the contributions that reach it, in increasing (marker, stencil
// point) order -- the order in which the markers are visited -- so R f is
// bitwise reproducible (no atomics, no order that depends on scheduling).
// Per component the map is CSR over the field's points: cnt[p] entries from
// off[p] in ent (marker << 7 | stencil point q = qi + 5 qj + 25 qk) with the
// tensor weight w = wx (wy wz) beside each entry.  It is rebuilt whenever the
// operators are (every RK stage for moving bodies).

// Stencil points whose one-dimensional weight is exactly zero along some
// axis (the five-point tables hold the delta function's support of four
// cells plus one point at distance >= 2) contribute exactly nothing and get
// no entry.

// count the entries of each grid point: one thread per (marker, qj, qk)
__global__ void k_sp_count(OpTables T, int c, int n1, int n2, int* __restrict__ cnt) {
  const int nb = T.nb;
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= 25 * (int64_t)nb) return;
  const int l = (int)(gid % nb);
  const int r = (int)(gid / nb);
  const int qj = r % 5, qk = r / 5;
  if (T.w1[tslot(nb, c, 1, qj, l)] == 0.0 || T.w1[tslot(nb, c, 2, qk, l)] == 0.0) return;
  const int iy = T.idx[tslot(nb, c, 1, qj, l)], iz = T.idx[tslot(nb, c, 2, qk, l)];
#pragma unroll
  for (int qi = 0; qi < 5; ++qi)
    if (T.w1[tslot(nb, c, 0, qi, l)] != 0.0)
      atomicAdd(cnt + lin(n1, n2, T.idx[tslot(nb, c, 0, qi, l)], iy, iz, 0), 1);
}

// place the entries (arbitrary order within a point; sorted next)
__global__ void k_sp_fill(OpTables T, int c, int n1, int n2, const int* __restrict__ off, int* __restrict__ cur,
                          uint32_t* __restrict__ ent) {
  const int nb = T.nb;
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= 25 * (int64_t)nb) return;
  const int l = (int)(gid % nb);
  const int r = (int)(gid / nb);
  const int qj = r % 5, qk = r / 5;
  if (T.w1[tslot(nb, c, 1, qj, l)] == 0.0 || T.w1[tslot(nb, c, 2, qk, l)] == 0.0) return;
  const int iy = T.idx[tslot(nb, c, 1, qj, l)], iz = T.idx[tslot(nb, c, 2, qk, l)];
#pragma unroll
  for (int qi = 0; qi < 5; ++qi) {
    if (T.w1[tslot(nb, c, 0, qi, l)] == 0.0) continue;
    const int64_t p = lin(n1, n2, T.idx[tslot(nb, c, 0, qi, l)], iy, iz, 0);
    const int slot = off[p] + atomicAdd(cur + p, 1);
    ent[slot] = ((uint32_t)l << 7) | (uint32_t)(qi + 5 * qj + 25 * qk);
  }
}

// sort each point's entries (insertion sort: a point has at most a few
// dozen) and attach the tensor weights
__global__ void k_sp_sort(OpTables T, int c, int64_t npts, const int* __restrict__ cnt, const int* __restrict__ off,
                          uint32_t* __restrict__ ent, double* __restrict__ w) {
  const int nb = T.nb;
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int n = cnt[p];
  if (n == 0) return;
  uint32_t* e = ent + off[p];
  constexpr int kSortLocal = 64;
  if (n <= kSortLocal) {
    // a thread-local copy (registers / L1), sorted there, written back once
    uint32_t t[kSortLocal];
    for (int a = 0; a < n; ++a) t[a] = e[a];
    for (int a = 1; a < n; ++a) {
      const uint32_t v = t[a];
      int b = a - 1;
      while (b >= 0 && t[b] > v) { t[b + 1] = t[b]; --b; }
      t[b + 1] = v;
    }
    for (int a = 0; a < n; ++a) e[a] = t[a];
  } else {
    for (int a = 1; a < n; ++a) {
      const uint32_t v = e[a];
      int b = a - 1;
      while (b >= 0 && e[b] > v) { e[b + 1] = e[b]; --b; }
      e[b + 1] = v;
    }
  }
  double* wp = w + off[p];
  for (int a = 0; a < n; ++a) {
    const int l = (int)(e[a] >> 7), q = (int)(e[a] & 127u);
    const int qi = q % 5, qj = (q / 5) % 5, qk = q / 25;
    wp[a] = T.w1[tslot(nb, c, 0, qi, l)] * (T.w1[tslot(nb, c, 1, qj, l)] * T.w1[tslot(nb, c, 2, qk, l)]);
  }
}

// per (component, marker) amplitude scale*factor*sb*f_c of the spread
__global__ void k_sp_amp(OpTables T, int comp0, int ncomp, int mode, const double* __restrict__ f, double dtnu,
                         double dt, double* __restrict__ amp) {
  const int nb = T.nb;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nb * ncomp) return;
  const int cc = gid / nb, l = gid - cc * nb;
  const int c = comp0 + cc;
  double fl;
  if (mode == S_RAW) fl = f[l];
  else if (mode == S_NORMAL) fl = T.nrm[c * nb + l];
  else fl = dtnu * f[c * nb + l] - dt * f[3 * nb + l] * T.nrm[c * nb + l];
  amp[c * nb + l] = T.scale * T.factor * T.sb[l] * fl;
}

struct SpGather {
  const int* cnt;
  const int* off;
  const uint32_t* ent;
  const double* w;
  double* F;
  int n1, n2, n3;
  int jlo, jhi;       // Fortran rows written (every point of them)
};

// F(i, j, k) = sum over the point's entries of w * amp(marker), for the
// rows jlo..jhi of up to three fields; points without entries get 0.
// A warp takes 32 consecutive points, whose entries are one contiguous run
// of the map: the run streams through shared memory in chunks (weights and
// marker amplitudes loaded by consecutive lanes), and each lane then adds
// its own point's terms in entry order.
constexpr int kSpChunk = 128;
__global__ void __launch_bounds__(256) k_sp_gather(SpGather g0, SpGather g1, SpGather g2, int ncomp,
                                                   const double* __restrict__ amp, int nb) {
  __shared__ double sw[8][kSpChunk], sa[8][kSpChunk];
  if ((int)blockIdx.y >= ncomp) return;
  // field description of this component, picked member by member (a
  // reference to one of the parameters would copy them to local memory)
  const int by = blockIdx.y;
#define SP_PICK(m) (by == 0 ? g0.m : (by == 1 ? g1.m : g2.m))
  SpGather g;
  g.cnt = SP_PICK(cnt); g.off = SP_PICK(off); g.ent = SP_PICK(ent); g.w = SP_PICK(w); g.F = SP_PICK(F);
  g.n1 = SP_PICK(n1); g.n2 = SP_PICK(n2); g.n3 = SP_PICK(n3); g.jlo = SP_PICK(jlo); g.jhi = SP_PICK(jhi);
#undef SP_PICK
  const int nrow = g.jhi - g.jlo + 1;
  const int64_t tot = (int64_t)g.n1 * nrow * g.n3;
  const double* a = amp + (int64_t)blockIdx.y * nb;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* ws = sw[warp];
  double* as = sa[warp];
  for (int64_t t0 = (blockIdx.x * (int64_t)blockDim.x + warp * 32); t0 < tot;
       t0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = t0 + lane;
    const bool valid = t < tot;
    int64_t p = 0;
    int n = 0, o = 0;
    if (valid) {
      const int i = (int)(t % g.n1);
      const int64_t r = t / g.n1;
      const int j = g.jlo + (int)(r % nrow);
      const int k = (int)(r / nrow);
      p = (int64_t)i + (int64_t)g.n1 * ((j - 1) + (int64_t)g.n2 * k);
      n = g.cnt[p];
      o = g.off[p];
    }
    // the warp's run of entries [lo, hi)
    int lo = n ? o : INT_MAX, hi = n ? o + n : INT_MIN;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, s));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, s));
    }
    double acc = 0.0;
    for (int cb = lo; cb < hi; cb += kSpChunk) {
      const int m = min(kSpChunk, hi - cb);
      // all loads of the chunk in flight before the marker amplitudes they
      // index, then the stores
      double wv[kSpChunk / 32], av[kSpChunk / 32];
      uint32_t ev[kSpChunk / 32];
#pragma unroll
      for (int u = 0; u < kSpChunk / 32; ++u) {
        const int e = lane + 32 * u;
        wv[u] = e < m ? g.w[cb + e] : 0.0;
        ev[u] = e < m ? g.ent[cb + e] : 0u;
      }
#pragma unroll
      for (int u = 0; u < kSpChunk / 32; ++u) av[u] = lane + 32 * u < m ? a[ev[u] >> 7] : 0.0;
#pragma unroll
      for (int u = 0; u < kSpChunk / 32; ++u) {
        ws[lane + 32 * u] = wv[u];
        as[lane + 32 * u] = av[u];
      }
      __syncwarp();
      const int e1 = min(o + n, cb + m);
      for (int e = max(o, cb); e < e1; ++e) acc += ws[e - cb] * as[e - cb];
      __syncwarp();
    }
    if (valid) g.F[p] = acc;
  }
}

// exclusive prefix sum of n ints (three passes: chunk sums, their scan,
// chunk scans)
constexpr int kScanChunk = 4096;
__global__ void __launch_bounds__(1024) k_scan_sums(const int* __restrict__ in, int64_t n, int* __restrict__ sums) {
  __shared__ int ws[32];
  const int64_t base = (int64_t)blockIdx.x * kScanChunk;
  int v = 0;
  for (int k = threadIdx.x; k < kScanChunk; k += blockDim.x)
    if (base + k < n) v += in[base + k];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    int u = ws[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = u;
  }
}

// block-wide exclusive scan of one value per thread (1024 threads); returns
// the thread's prefix and the block total in *total
__device__ int block_excl_scan(int v, int* ws, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = ws[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    ws[lane] = t;   // inclusive warp totals
  }
  __syncthreads();
  const int before = (wid > 0 ? ws[wid - 1] : 0) + x - v;
  *total = ws[31];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(1024) k_scan_top(int* __restrict__ sums, int nsums) {
  __shared__ int ws[32];
  int carry = 0;
  for (int base = 0; base < nsums; base += 1024) {
    const int k = base + threadIdx.x;
    const int v = k < nsums ? sums[k] : 0;
    int tot;
    const int ex = block_excl_scan(v, ws, &tot);
    if (k < nsums) sums[k] = carry + ex;
    carry += tot;
  }
}

__global__ void __launch_bounds__(1024) k_scan_chunks(const int* __restrict__ in, int64_t n,
                                                      const int* __restrict__ sums, int* __restrict__ out) {
  __shared__ int ws[32];
  const int64_t base = (int64_t)blockIdx.x * kScanChunk;
  constexpr int kPer = kScanChunk / 1024;
  int v[kPer];
  int loc = 0;
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int64_t k = base + (int64_t)threadIdx.x * kPer + u;
    v[u] = k < n ? in[k] : 0;
    loc += v[u];
  }
  int tot;
  int run = sums[blockIdx.x] + block_excl_scan(loc, ws, &tot);
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int64_t k = base + (int64_t)threadIdx.x * kPer + u;
    if (k < n) out[k] = run;
    run += v[u];
  }
}

// ---------------------------------------------------------------------------
// marker-vector kernels: mean removal, dot products, BiCGSTAB updates
// ---------------------------------------------------------------------------
static const int kIbRedBlocks = 256;

__global__ void k_body_sums(const double* __restrict__ v, const int* __restrict__ body, int nb,
                            int nbodies, double* __restrict__ out) {
  // one block per body, fixed order
  const int b = blockIdx.x;
  double acc = 0.0;
  for (int l = threadIdx.x; l < nb; l += blockDim.x)
    if (body[l] == b) acc += v[l];
  __shared__ double sm[256];
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = sm[0];
  (void)nbodies;
}

// Same sums for up to kMaxBodies bodies over the whole grid: per-thread
// per-body accumulators, block partials, and the last block to finish
// (ticket) adds the partials in block order.
constexpr int kMaxBodies = 8;
constexpr int kBodyBlocks = 64;
__global__ void __launch_bounds__(256) k_body_sums_grid(const double* __restrict__ v, const int* __restrict__ body,
                                                       int nb, int nbodies, double* __restrict__ part,
                                                       unsigned* __restrict__ ticket, double* __restrict__ out) {
  double acc[kMaxBodies];
#pragma unroll
  for (int q = 0; q < kMaxBodies; ++q) acc[q] = 0.0;
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nb; l += gridDim.x * blockDim.x) {
    const int b = body[l];
    const double x = v[l];
#pragma unroll
    for (int q = 0; q < kMaxBodies; ++q)
      if (q == b) acc[q] += x;
  }
  __shared__ double sm[8][kMaxBodies];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kMaxBodies; ++q) {
    double x = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sm[w][q] = x;
  }
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x < kMaxBodies) {
    double x = 0.0;
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) x += sm[ww][threadIdx.x];
    part[blockIdx.x * kMaxBodies + threadIdx.x] = x;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < nbodies) {
    double x = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) x += __ldcg(part + b * kMaxBodies + threadIdx.x);
    out[threadIdx.x] = x;
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

// v(p rows) = v - mean_body; then v -= E1nHc * pj (optional)
__global__ void k_remove_mean(double* __restrict__ v, const int* __restrict__ body,
                              const double* __restrict__ sums, const double* __restrict__ binv, int nb,
                              const double* __restrict__ e1nhc, const double* __restrict__ pj) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nb) return;
  double x = v[l] - sums[body[l]] * binv[body[l]];
  if (e1nhc) x = x - e1nhc[l] * pj[l];
  v[l] = x;
}

// partial dot products: up to 2 pairs
__global__ void __launch_bounds__(256) k_dot2(const double* __restrict__ a, const double* __restrict__ b,
                                             const double* __restrict__ c, const double* __restrict__ e,
                                             int64_t n, double* __restrict__ part) {
  double s0 = 0.0, s1 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    s0 += a[i] * b[i];
    if (c) s1 += c[i] * e[i];
  }
  __shared__ double sa[256], sb_[256];
  sa[threadIdx.x] = s0;
  sb_[threadIdx.x] = s1;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) { sa[threadIdx.x] += sa[threadIdx.x + s]; sb_[threadIdx.x] += sb_[threadIdx.x + s]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = sa[0]; part[2 * blockIdx.x + 1] = sb_[0]; }
}

// BiCGSTAB scalars on the device: sc[0] rho_o, [1] alpha, [2] om, [3] rho_n,
// [4] bta, [5] err, [6] dot1, [7] dot2
__global__ void k_dot_final(const double* __restrict__ part, int np, double* sc, int slot0, int op) {
  __shared__ double sa[256], sb_[256];
  double s0 = 0.0, s1 = 0.0;
  for (int t = threadIdx.x; t < np; t += blockDim.x) { s0 += part[2 * t]; s1 += part[2 * t + 1]; }
  sa[threadIdx.x] = s0;
  sb_[threadIdx.x] = s1;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) { sa[threadIdx.x] += sa[threadIdx.x + s]; sb_[threadIdx.x] += sb_[threadIdx.x + s]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double d0 = sa[0], d1 = sb_[0];
    if (op == 0) {            // rho_n = <rhat, r>; bta; rho_o = rho_n
      sc[3] = d0;
      sc[4] = (d0 / sc[0]) * (sc[1] / sc[2]);
      sc[0] = d0;
    } else if (op == 1) {     // alpha = rho_n / <rhat, nu>
      sc[1] = sc[3] / d0;
    } else if (op == 2) {     // om = <t, s>/<t, t>
      sc[2] = d0 / d1;
    } else if (op == 3) {     // err = <r, r>
      sc[5] = d0;
    } else {
      sc[slot0] = d0;
      sc[slot0 + 1] = d1;
    }
  }
}

// p = r + bta*(p - om*nu);  ph = M p
__global__ void k_bcg_p(int64_t n, const double* __restrict__ r, double* __restrict__ p,
                        const double* __restrict__ nu, double* __restrict__ ph,
                        const double* __restrict__ minv, const double* __restrict__ sc) {
  const double bta = sc[4], om = sc[2];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = r[i] + bta * (p[i] - om * nu[i]);
    p[i] = v;
    ph[i] = minv ? minv[i] * v : v;
  }
}

// h = x + alpha*ph (kept in x via later update); s = r - alpha*nu; sh = M s
__global__ void k_bcg_s(int64_t n, const double* __restrict__ r, const double* __restrict__ nu,
                        double* __restrict__ s, double* __restrict__ sh, double* __restrict__ x,
                        const double* __restrict__ ph, const double* __restrict__ minv,
                        const double* __restrict__ sc) {
  const double alpha = sc[1];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = r[i] - alpha * nu[i];
    s[i] = v;
    sh[i] = minv ? minv[i] * v : v;
    x[i] = x[i] + alpha * ph[i];       // h
  }
}

// x = h + om*sh; r = s - om*t; partial <r, r>
__global__ void __launch_bounds__(256) k_bcg_x(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                              const double* __restrict__ s, const double* __restrict__ sh,
                                              const double* __restrict__ t, const double* __restrict__ sc,
                                              double* __restrict__ part) {
  const double om = sc[2];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = x[i] + om * sh[i];
    const double v = s[i] - om * t[i];
    r[i] = v;
    acc += v * v;
  }
  __shared__ double sa[256];
  sa[threadIdx.x] = acc;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sa[threadIdx.x] += sa[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = sa[0]; part[2 * blockIdx.x + 1] = 0.0; }
}

__global__ void k_axpby(int64_t n, double a, const double* __restrict__ x, double b,
                        const double* __restrict__ y, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = a * x[i] + b * y[i];
}

__global__ void k_bcg_init(double* sc) {
  sc[0] = 1.0; sc[1] = 1.0; sc[2] = 1.0; sc[5] = 1.0;
}

// out_b = B_b in_b for every marker b, with in_b = (in[b], in[nb+b],
// in[2nb+b], in[3nb+b]) and B_b the 4x4 block blk[16*b ..] (row-major)
__global__ void k_apply_blocks(int nb, const double* __restrict__ blk, const double* __restrict__ in,
                               double* __restrict__ out) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    double v[4], B[16];
#pragma unroll
    for (int c = 0; c < 4; ++c) v[c] = in[(int64_t)c * nb + b];
#pragma unroll
    for (int q = 0; q < 16; ++q) B[q] = blk[16 * (int64_t)b + q];
#pragma unroll
    for (int c = 0; c < 4; ++c)
      out[(int64_t)c * nb + b] = B[4 * c] * v[0] + B[4 * c + 1] * v[1] + B[4 * c + 2] * v[2] + B[4 * c + 3] * v[3];
  }
}

// probe vector of one colour class: unit entries in block `blk` on the
// markers with (ix mod px, iz mod pz) = (cx, cz), ix = l mod lat_nx, iz = l / lat_nx
__global__ void k_probe_mask(int nb, int lat_nx, int blk, int px, int pz, int cx, int cz,
                             double* __restrict__ e) {
  const int64_t n = 4 * (int64_t)nb;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i / nb), l = (int)(i - (int64_t)c * nb);
    const int ix = l % lat_nx, iz = l / lat_nx;
    e[i] = (c == blk && ix % px == cx && iz % pz == cz) ? 1.0 : 0.0;
  }
}

// Per marker of the probed colour class, from the responses R_c = S e_c of
// the four component probes: the column block C_b of S restricted to the
// lattice neighbourhood N(b) (|dix| <= 2, |diz| <= 2, periodic, all four
// components), G_b = C_b^T C_b and the diagonal block S_bb.  Outputs the
// Jacobi block diag(1/S_bb,cc), the block sparse approximate inverse
// M_b = G_b^-1 S_bb^T (minimiser of ||e_b - C_b M_b||_F, the marker's block
// column of min ||I - S M||_F), and optionally the moments Crr = G_b,
// Cer = S_bb, Cee = 1 (36 floats) for training.
__global__ void k_probe_spai(int nb, int lat, int nrow, int px, int pz, int cx, int cz,
                             const double* __restrict__ R, double* __restrict__ jac,
                             double* __restrict__ spai, float* __restrict__ mom) {
  const int64_t n = 4 * (int64_t)nb;
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nb; l += gridDim.x * blockDim.x) {
    const int ix = l % lat, iz = l / lat;
    if (ix % px != cx || iz % pz != cz) continue;
    double G[16] = {0}, S[16];
    for (int dz = -2; dz <= 2; ++dz)
      for (int dx = -2; dx <= 2; ++dx) {
        const int jx = (ix + dx + lat) % lat, jz = (iz + dz + nrow) % nrow;
        const int lp = jx + lat * jz;
        if (lp >= nb) continue;
        for (int cr = 0; cr < 4; ++cr) {
          const int64_t row = (int64_t)cr * nb + lp;
          double v[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) v[c] = R[(int64_t)c * n + row];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) G[4 * a + b] += v[a] * v[b];
        }
      }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) S[4 * a + c] = R[(int64_t)c * n + (int64_t)a * nb + l];
    for (int c = 0; c < 4; ++c) {
      const double dg = S[5 * c];
      jac[16 * (int64_t)l + 5 * c] = (fabs(dg) > 1e-300) ? 1.0 / dg : 1.0;
    }
    // M = G^-1 S^T by Gauss-Jordan with partial pivoting on [G | S^T]
    double Aug[4][8];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) { Aug[a][b] = G[4 * a + b]; Aug[a][4 + b] = S[4 * b + a]; }
    bool sing = false;
    for (int c = 0; c < 4; ++c) {
      int piv = c;
      for (int r = c + 1; r < 4; ++r) if (fabs(Aug[r][c]) > fabs(Aug[piv][c])) piv = r;
      if (!(fabs(Aug[piv][c]) > 1e-300)) { sing = true; break; }
      if (piv != c)
        for (int q = 0; q < 8; ++q) { const double t = Aug[c][q]; Aug[c][q] = Aug[piv][q]; Aug[piv][q] = t; }
      const double inv = 1.0 / Aug[c][c];
      for (int q = 0; q < 8; ++q) Aug[c][q] *= inv;
      for (int r = 0; r < 4; ++r)
        if (r != c) {
          const double f = Aug[r][c];
          for (int q = 0; q < 8; ++q) Aug[r][q] -= f * Aug[c][q];
        }
    }
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b)
        spai[16 * (int64_t)l + 4 * a + b] = sing ? (a == b ? jac[16 * (int64_t)l + 5 * a] : 0.0) : Aug[a][4 + b];
    if (mom) {
      float* m = mom + 36 * (int64_t)l;
      for (int q = 0; q < 16; ++q) { m[q] = (float)G[q]; m[16 + q] = (float)S[q]; }
      for (int q = 0; q < 4; ++q) m[32 + q] = 1.f;
    }
  }
}

// ---------------------------------------------------------------------------
// IB projection final update: U = Ui - Ureg - G(dt*Pint - phi2)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_ib_final(Dims d, Metric m, const double* __restrict__ Ui,
                                                  const double* __restrict__ Vi, const double* __restrict__ Wi,
                                                  const double* __restrict__ Ur, const double* __restrict__ Vr,
                                                  const double* __restrict__ Wr, const double* __restrict__ Pint,
                                                  const double* __restrict__ phi2, double dt,
                                                  double* __restrict__ Uo, double* __restrict__ Vo,
                                                  double* __restrict__ Wo) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 2 + blockIdx.z * blockDim.z + threadIdx.z;
  if (i > d.Nx + 1 || j > d.Ny + 1 || k > d.Nz + 1) return;
  auto pe = [&](int a, int b, int c) {
    const int64_t r = idxR(d, a, b, c);
    return dt * (Pint[r] - phi2[r] / dt);
  };
  const double p0 = pe(i, j, k);
  const int64_t iu = idxU(d, i, j, k), iw = idxW(d, i, j, k);
  Uo[iu] = Ui[iu] - Ur[iu] - (pe(i + 1, j, k) - p0) * m.rdxg[i];
  Wo[iw] = Wi[iw] - Wr[iw] - (pe(i, j, k + 1) - p0) * m.rdzg[k];
  if (j <= d.Ny) {
    const int64_t iv = idxV(d, i, j, k);
    Vo[iv] = Vi[iv] - Vr[iv] - (pe(i, j + 1, k) - p0) * m.rdyg[j];
  }
}

// Heaviside: Hu_ext etc. by midpoint interpolation of Hc_ext (src/heaviside.f90:40-42)
__global__ void k_heaviside_interp(Dims d, const double* __restrict__ Hce, double* __restrict__ Hue,
                                   double* __restrict__ Hve, double* __restrict__ Hwe) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 2 + blockIdx.z * blockDim.z + threadIdx.z;
  if (i > d.Nx + 1 || j > d.Ny + 1 || k > d.Nz + 1) return;
  const double c0 = Hce[idxR(d, i, j, k)];
  Hue[idxU(d, i, j, k)] = 0.5 * (c0 + Hce[idxR(d, i + 1, j, k)]);
  Hwe[idxW(d, i, j, k)] = 0.5 * (c0 + Hce[idxR(d, i, j, k + 1)]);
  if (j <= d.Ny) Hve[idxV(d, i, j, k)] = 0.5 * (c0 + Hce[idxR(d, i, j + 1, k)]);
}

__global__ void k_one_minus(int64_t n, const double* __restrict__ a, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = 1.0 - a[i];
}

__global__ void k_negate(int64_t n, double* __restrict__ a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = -a[i];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static OpTables tables(Handle* h) {
  IbState* s = h->ib;
  OpTables T{};
  T.nb = s->nb;
  T.idx = s->idx_d;
  T.w1 = s->w1_d;
  T.off = s->off_d;
  T.nrm = s->nrm_d;
  T.sb = s->sb_d;
  T.scale = h->dx * h->dymin * h->dz;
  T.factor = 1.0 / (h->dx * h->dymin * h->dz);
  return T;
}

static unsigned thread_blocks(int64_t n) { return (unsigned)((n + 127) / 128); }

static int upload_geometry(Handle* h) {
  IbState* s = h->ib;
  cudaStream_t st = h->stream;
  const size_t nb = (size_t)s->nb;
  std::vector<double> binv(s->nbodies);
  for (int b = 0; b < s->nbodies; ++b) binv[b] = 1.0 / (double)s->body_count[b];
  struct Part { void* dst; const void* src; size_t bytes; };
  const Part parts[] = {
      {s->xb_d, s->xb.data(), 8 * nb},          {s->yb_d, s->yb.data(), 8 * nb},
      {s->zb_d, s->zb.data(), 8 * nb},          {s->ub_d, s->ub.data(), 24 * nb},
      {s->nrm_d, s->nrm.data(), 24 * nb},       {s->sb_d, s->sb.data(), 8 * nb},
      {s->yref_d, s->yref.data(), 4 * nb},      {s->body_d, s->body.data(), 4 * nb},
      {s->binv_d, binv.data(), 8 * binv.size()}};
  size_t total = 0;
  for (const Part& q : parts) total += (q.bytes + 15) & ~size_t(15);
  if (s->stage_bytes < total) {
    if (s->stage_h) {
      C3D_CUDA_TRY(h, cudaEventSynchronize(s->stage_ev));
      cudaFreeHost(s->stage_h);
      s->stage_h = nullptr;
    }
    C3D_CUDA_TRY(h, cudaMallocHost(reinterpret_cast<void**>(&s->stage_h), total));
    s->stage_bytes = total;
  }
  if (!s->stage_ev) C3D_CUDA_TRY(h, cudaEventCreateWithFlags(&s->stage_ev, cudaEventDisableTiming));
  else C3D_CUDA_TRY(h, cudaEventSynchronize(s->stage_ev));   // the last upload has left the staging
  // the host vectors go to page-locked staging, and from there
  // asynchronously to the device (the host may change them at once)
  size_t o = 0;
  for (const Part& q : parts) {
    std::memcpy(s->stage_h + o, q.src, q.bytes);
    C3D_CUDA_TRY(h, cudaMemcpyAsync(q.dst, s->stage_h + o, q.bytes, cudaMemcpyHostToDevice, st));
    o += (q.bytes + 15) & ~size_t(15);
  }
  C3D_CUDA_TRY(h, cudaEventRecord(s->stage_ev, st));
  return 0;
}

static int upload_grids(Handle* h) {
  IbState* s = h->ib;
  cudaStream_t st = h->stream;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->x_d, h->x.data(), 8 * h->x.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->y_d, h->y.data(), 8 * h->y.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->z_d, h->z.data(), 8 * h->z.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->xm_d, h->xm.data(), 8 * h->xm.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->ym_d, h->ym.data(), 8 * h->ym.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->zm_d, h->zm.data(), 8 * h->zm.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(st));
  s->grids_current = true;
  return 0;
}

void ib_grids_changed(Handle* h) {
  if (h->ib) h->ib->grids_current = false;
}

int ib_create(Handle* h) {
  IbState* s = new IbState();
  h->ib = s;
  s->kind = h->p.body_type;
  s->moving = (s->kind == "standing_wave" || s->kind == "traveling_wave_x" ||
               s->kind == "wall_standing_wave" || s->kind == "wall_plates");
  std::string err;
  int rc = geometry_host(h, s, h->t, err);
  if (rc) { h->last_error = err; return rc; }
  const int nb = s->nb;
  const Dims& d = h->d;
  if ((rc = dev_alloc(h, &s->xb_d, nb))) return rc;
  if ((rc = dev_alloc(h, &s->yb_d, nb))) return rc;
  if ((rc = dev_alloc(h, &s->zb_d, nb))) return rc;
  if ((rc = dev_alloc(h, &s->ub_d, 3 * nb))) return rc;
  if ((rc = dev_alloc(h, &s->nrm_d, 3 * nb))) return rc;
  if ((rc = dev_alloc(h, &s->sb_d, nb))) return rc;
  if ((rc = dev_alloc(h, &s->yref_d, nb))) return rc;
  if ((rc = dev_alloc(h, &s->body_d, nb))) return rc;
  if ((rc = dev_alloc(h, &s->binv_d, 8))) return rc;
  if ((rc = dev_alloc(h, &s->x_d, (int64_t)h->x.size()))) return rc;
  if ((rc = dev_alloc(h, &s->y_d, (int64_t)h->y.size()))) return rc;
  if ((rc = dev_alloc(h, &s->z_d, (int64_t)h->z.size()))) return rc;
  if ((rc = dev_alloc(h, &s->xm_d, (int64_t)h->xm.size()))) return rc;
  if ((rc = dev_alloc(h, &s->ym_d, (int64_t)h->ym.size()))) return rc;
  if ((rc = dev_alloc(h, &s->zm_d, (int64_t)h->zm.size()))) return rc;
  const int64_t nt = (int64_t)4 * 3 * 5 * nb;
  if ((rc = dev_alloc(h, &s->idx_d, nt))) return rc;
  if ((rc = dev_alloc(h, &s->w1_d, nt))) return rc;
  if ((rc = dev_alloc(h, &s->off_d, nt))) return rc;
  if ((rc = dev_alloc(h, &s->flag_d, 4))) return rc;
  if ((rc = dev_alloc(h, &s->Ureg, sizeU(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Vreg, sizeV(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Wreg, sizeW(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Hu, sizeU(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Hv, sizeV(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Hw, sizeW(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Hce, sizeR(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Ut, sizeU(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Vt, sizeV(d)))) return rc;
  if ((rc = dev_alloc(h, &s->Wt, sizeW(d)))) return rc;
  double** vecs[] = {&s->fb, &s->E1nHc, &s->E1nH, &s->rhs, &s->scr0, &s->scr1, &s->scr2, &s->r,
                     &s->rhat, &s->p, &s->nu, &s->ph, &s->s, &s->sh, &s->t};
  for (auto v : vecs)
    if ((rc = dev_alloc(h, v, 4 * (int64_t)nb))) return rc;
  if ((rc = dev_alloc(h, &s->jac_blk, 16 * (int64_t)nb))) return rc;
  if ((rc = dev_alloc(h, &s->spai_blk, 16 * (int64_t)nb))) return rc;
  if ((rc = dev_alloc(h, &s->red, 2 * kIbRedBlocks + 16))) return rc;
  if ((rc = dev_alloc(h, &s->ticket, 1))) return rc;
  if ((rc = dev_alloc(h, &s->sc, 16))) return rc;
  // H = 1 (interior) until compute_heaviside runs (app/main.f90:80-85)
  std::vector<double> ones(std::max(sizeU(d), std::max(sizeV(d), sizeW(d))), 1.0);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->Hu, ones.data(), 8 * sizeU(d), cudaMemcpyHostToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->Hv, ones.data(), 8 * sizeV(d), cudaMemcpyHostToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->Hw, ones.data(), 8 * sizeW(d), cudaMemcpyHostToDevice, h->stream));
  if ((rc = upload_grids(h))) return rc;
  if ((rc = upload_geometry(h))) return rc;
  return ib_setup_operators(h);
}

void ib_free(Handle* h) {
  if (h->ib) {
    band_free(h->ib);
    if (h->ib->stage_ev) {
      cudaEventSynchronize(h->ib->stage_ev);
      cudaEventDestroy(h->ib->stage_ev);
    }
    if (h->ib->stage_h) cudaFreeHost(h->ib->stage_h);
  }
  delete h->ib;
  h->ib = nullptr;
}

int ib_setup_geometry(Handle* h, double t) {
  IbState* s = h->ib;
  if (!s) return C3D_ERR_UNSUPPORTED;
  std::string err;
  const int nb0 = s->nb;
  int rc = geometry_host(h, s, t, err);
  if (rc) { h->last_error = err; return rc; }
  if (s->nb != nb0) { h->last_error = "marker count changed"; return C3D_ERR_PARAM; }
  return upload_geometry(h);
}

// smallest and largest y index of any stencil (all four locations)
__global__ void k_iy_range(const int* __restrict__ idx, int nb, int* __restrict__ range) {
  int lo = 1 << 30, hi = -(1 << 30);
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nb; l += gridDim.x * blockDim.x)
    for (int t = 0; t < 4; ++t)
      for (int q = 0; q < 5; ++q) {
        const int iy = idx[tslot(nb, t, 1, q, l)];
        lo = min(lo, iy);
        hi = max(hi, iy);
      }
  atomicMin(range, lo);
  atomicMax(range + 1, hi);
}

static int build_spread_maps(Handle* h);

int ib_setup_operators(Handle* h) {
  IbState* s = h->ib;
  if (!s) return C3D_ERR_UNSUPPORTED;
  if (s->x_d == nullptr) return 0;
  int rc = s->grids_current ? 0 : upload_grids(h);
  if (rc) return rc;
  IbGeomArgs a{};
  a.d = h->d; a.nb = s->nb;
  a.xb = s->xb_d; a.yb = s->yb_d; a.zb = s->zb_d; a.yref = s->yref_d;
  a.x = s->x_d; a.y = s->y_d; a.z = s->z_d; a.xm = s->xm_d; a.ym = s->ym_d; a.zm = s->zm_d;
  a.dx = h->dx; a.dz = h->dz; a.dymin = h->dymin; a.Lxp = h->Lxp; a.Lzp = h->Lzp;
  a.idx = s->idx_d; a.w1 = s->w1_d; a.off = s->off_d; a.flag = s->flag_d;
  // flag_d[0]: a stencil left the grid; flag_d[1..2]: the y rows the
  // stencils touch (the Schur complement's spread field and the rows of its
  // potential read by the gathers lie in [iy_lo - 1, iy_hi + 1]); one
  // read-back for both
  int fr[3] = {0, 1 << 30, -(1 << 30)};
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->flag_d, fr, sizeof(fr), cudaMemcpyHostToDevice, h->stream));
  k_ib_weights<<<(s->nb + 127) / 128, 128, 0, h->stream>>>(a);
  C3D_LAUNCH_CHECK(h);
  k_iy_range<<<std::min(148, (s->nb + 255) / 256), 256, 0, h->stream>>>(s->idx_d, s->nb, s->flag_d + 1);
  C3D_LAUNCH_CHECK(h);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(fr, s->flag_d, sizeof(fr), cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (fr[0]) { h->last_error = "Error: zi_supp out of range (marker stencil outside the grid)"; return C3D_ERR_PARAM; }
  s->iy_lo = fr[1];
  s->iy_hi = fr[2];
  return build_spread_maps(h);
}

// G phi - U_reg at the x-z interior points of the stencil rows [jlo, jhi]
// (src/projection.f90:135-139: the gradient of the potential, its boundary
// values, minus the spread field), into fields of the u, v, w shapes; v is
// zero on the wall faces.  Rows, columns and planes are those the stencil
// tables index (x and z interior, y rows [iy_lo, iy_hi]).
__global__ void __launch_bounds__(256) k_grad_minus_reg(Dims d, Metric m, const double* __restrict__ P,
                                                       const double* __restrict__ Ur,
                                                       const double* __restrict__ Vr,
                                                       const double* __restrict__ Wr, double* __restrict__ Gu,
                                                       double* __restrict__ Gv, double* __restrict__ Gw, int jlo,
                                                       int jhi) {
  const int nxi = d.Nx, nzi = d.Nz, nr = jhi - jlo + 1;
  const int64_t tot = (int64_t)nxi * nr * nzi;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 2 + (int)(t % nxi);
    const int64_t r = t / nxi;
    const int j = jlo + (int)(r % nr);
    const int k = 2 + (int)(r / nr);
    const bool centre = j >= 2 && j <= d.ny;       // u and w rows
    const double p0 = centre ? P[idxR(d, i, j, k)] : 0.0;
    if (centre) {
      const int64_t iu = idxU(d, i, j, k), iw = idxW(d, i, j, k);
      Gu[iu] = (P[idxR(d, i + 1, j, k)] - p0) * m.rdxg[i] - Ur[iu];
      Gw[iw] = (P[idxR(d, i, j, k + 1)] - p0) * m.rdzg[k] - Wr[iw];
    }
    if (j >= 1 && j <= d.ny) {                     // v faces
      const double gv = (j >= 2 && j <= d.ny - 1) ? (P[idxR(d, i, j + 1, k)] - p0) * m.rdyg[j] : 0.0;
      const int64_t iv = idxV(d, i, j, k);
      Gv[iv] = gv - Vr[iv];
    }
  }
}

// gather helpers
static GField gf_u(const Dims& d, const double* F) { return GField{F, d.nx, d.nyg, 0, 1.0}; }
static GField gf_v(const Dims& d, const double* F) { return GField{F, d.nxg, d.ny, 0, 1.0}; }
static GField gf_w(const Dims& d, const double* F) { return GField{F, d.nxg, d.nyg, 0, 1.0}; }

static int gather3(Handle* h, int mode, const double* U, const double* V, const double* W, double* out,
                   double sign = 1.0, const double* sub = nullptr, const double* subv = nullptr,
                   const double* addv = nullptr) {
  GatherArgs a{};
  a.T = tables(h); a.d = h->d;
  const GField fs[3] = {gf_u(h->d, U), gf_v(h->d, V), gf_w(h->d, W)};
  for (int c = 0; c < 3; ++c) a.comp[c] = GComp{fs[c], c, mode, sign, sub, subv, addv};
  a.ncomp = 3; a.out = out;
  launch_gather_tile(a, h->stream);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

static int gather_c(Handle* h, const double* P, double mul, double* out, double sign = 1.0) {
  GatherArgs a{};
  a.T = tables(h); a.d = h->d;
  a.comp[0] = GComp{GField{P, h->d.nxg - 2, h->d.nyg - 2, 1, mul}, 3, G_E1N, sign, nullptr, nullptr, nullptr};
  a.ncomp = 1; a.out = out;
  launch_gather_tile(a, h->stream);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// build the inverse maps of the u, v, w stencils (after the weights)
static int build_spread_maps(Handle* h) {
  IbState* s = h->ib;
  const Dims& d = h->d;
  const OpTables T = tables(h);
  const int64_t ne = 125 * (int64_t)s->nb;
  const int n1s[3] = {d.nx, d.nxg, d.nxg}, n2s[3] = {d.nyg, d.ny, d.nyg};
  const int64_t npts[3] = {sizeU(d), sizeV(d), sizeW(d)};
  int rc;
  for (int c = 0; c < 3; ++c) {
    if (!s->sp_cnt[c]) {
      if ((rc = dev_alloc(h, &s->sp_cnt[c], npts[c]))) return rc;
      if ((rc = dev_alloc(h, &s->sp_off[c], npts[c]))) return rc;
      if ((rc = dev_alloc(h, &s->sp_ent[c], ne))) return rc;
      if ((rc = dev_alloc(h, &s->sp_w[c], ne))) return rc;
    }
  }
  const int64_t maxpts = std::max(npts[0], std::max(npts[1], npts[2]));
  const int nchunks = (int)((maxpts + kScanChunk - 1) / kScanChunk);
  if (!s->sp_sums && (rc = dev_alloc(h, &s->sp_sums, nchunks))) return rc;
  if (!s->amp && (rc = dev_alloc(h, &s->amp, 3 * (int64_t)s->nb))) return rc;
  const unsigned gq = (unsigned)((25 * (int64_t)s->nb + 255) / 256);
  for (int c = 0; c < 3; ++c) {
    const int64_t n = npts[c];
    const int nch = (int)((n + kScanChunk - 1) / kScanChunk);
    C3D_CUDA_TRY(h, cudaMemsetAsync(s->sp_cnt[c], 0, 4 * (size_t)n, h->stream));
    k_sp_count<<<gq, 256, 0, h->stream>>>(T, c, n1s[c], n2s[c], s->sp_cnt[c]);
    C3D_LAUNCH_CHECK(h);
    k_scan_sums<<<nch, 1024, 0, h->stream>>>(s->sp_cnt[c], n, s->sp_sums);
    C3D_LAUNCH_CHECK(h);
    k_scan_top<<<1, 1024, 0, h->stream>>>(s->sp_sums, nch);
    C3D_LAUNCH_CHECK(h);
    k_scan_chunks<<<nch, 1024, 0, h->stream>>>(s->sp_cnt[c], n, s->sp_sums, s->sp_off[c]);
    C3D_LAUNCH_CHECK(h);
    // the counts become the fill cursors and are counts again afterwards
    C3D_CUDA_TRY(h, cudaMemsetAsync(s->sp_cnt[c], 0, 4 * (size_t)n, h->stream));
    k_sp_fill<<<gq, 256, 0, h->stream>>>(T, c, n1s[c], n2s[c], s->sp_off[c], s->sp_cnt[c], s->sp_ent[c]);
    C3D_LAUNCH_CHECK(h);
    k_sp_sort<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(T, c, n, s->sp_cnt[c], s->sp_off[c], s->sp_ent[c],
                                                                  s->sp_w[c]);
    C3D_LAUNCH_CHECK(h);
  }
  return 0;
}

// R f of components comp0 .. comp0+ncomp-1 into F0.. over the Fortran rows
// jlo..jhi of each field (every point of those rows is written)
static int spread(Handle* h, int mode, int comp0, int ncomp, const double* f, double dt,
                  double* F0, double* F1, double* F2, int jlo = 1, int jhi = 1 << 30) {
  IbState* s = h->ib;
  const Dims& d = h->d;
  const OpTables T = tables(h);
  k_sp_amp<<<thread_blocks((int64_t)ncomp * s->nb), 128, 0, h->stream>>>(T, comp0, ncomp, mode, f, dt * h->p.nu, dt,
                                                                         s->amp);
  C3D_LAUNCH_CHECK(h);
  double* Fs[3] = {F0, F1, F2};
  const int n1s[3] = {d.nx, d.nxg, d.nxg}, n2s[3] = {d.nyg, d.ny, d.nyg}, n3s[3] = {d.nzg, d.nzg, d.nz};
  SpGather g[3]{};
  int64_t most = 0;
  for (int cc = 0; cc < ncomp; ++cc) {
    const int c = comp0 + cc;
    g[cc].cnt = s->sp_cnt[c]; g[cc].off = s->sp_off[c]; g[cc].ent = s->sp_ent[c]; g[cc].w = s->sp_w[c];
    g[cc].F = Fs[cc]; g[cc].n1 = n1s[c]; g[cc].n2 = n2s[c]; g[cc].n3 = n3s[c];
    g[cc].jlo = std::max(jlo, 1);
    g[cc].jhi = std::min(jhi, n2s[c]);
    if (g[cc].jhi < g[cc].jlo) { g[cc].jlo = 1; g[cc].jhi = 0; }
    most = std::max(most, (int64_t)g[cc].n1 * (g[cc].jhi - g[cc].jlo + 1) * g[cc].n3);
  }
  if (most == 0) return 0;
  dim3 grid((unsigned)std::min<int64_t>((most + 255) / 256, 148 * 8), (unsigned)ncomp);
  k_sp_gather<<<grid, 256, 0, h->stream>>>(g[0], g[1], g[2], ncomp, s->amp + (int64_t)comp0 * s->nb, s->nb);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// zero U_reg, V_reg, W_reg and spread; then boundary conditions
// R f for the Schur complement: only the rows [jlo, jhi] of the spread
// fields are cleared (the banded solve reads nothing else; rows outside keep
// zeros or values of earlier geometries that no banded reader touches)
static int reg_all_band(Handle* h, int mode, const double* f, double dt, int jlo, int jhi) {
  IbState* s = h->ib;
  // no ghost fill: the band divergence (k_xfft_fwd) folds the periodic x and
  // z images and the wall faces itself, and the gathers read x-z interior
  // points only
  return spread(h, mode, 0, 3, f, dt, s->Ureg, s->Vreg, s->Wreg, jlo, jhi);
}

static int reg_all(Handle* h, int mode, const double* f, double dt) {
  IbState* s = h->ib;
  const Dims& d = h->d;
  C3D_CUDA_TRY(h, cudaMemsetAsync(s->Ureg, 0, 8 * sizeU(d), h->stream));
  C3D_CUDA_TRY(h, cudaMemsetAsync(s->Vreg, 0, 8 * sizeV(d), h->stream));
  C3D_CUDA_TRY(h, cudaMemsetAsync(s->Wreg, 0, 8 * sizeW(d), h->stream));
  int rc = spread(h, mode, 0, 3, f, dt, s->Ureg, s->Vreg, s->Wreg, s->iy_lo, s->iy_hi);
  if (rc) return rc;
  return launch_fill_ghosts3(h, s->Ureg, s->Vreg, s->Wreg);
}

static int remove_mean(Handle* h, double* v, const double* pj_for_e1nhc) {
  IbState* s = h->ib;
  if (s->nbodies <= kMaxBodies) {
    k_body_sums_grid<<<kBodyBlocks, 256, 0, h->stream>>>(v, s->body_d, s->nb, s->nbodies, s->red + 16,
                                                         s->ticket, s->red);
  } else {
    k_body_sums<<<s->nbodies, 256, 0, h->stream>>>(v, s->body_d, s->nb, s->nbodies, s->red);
  }
  C3D_LAUNCH_CHECK(h);
  k_remove_mean<<<(s->nb + 255) / 256, 256, 0, h->stream>>>(v, s->body_d, s->red, s->binv_d, s->nb,
                                                            pj_for_e1nhc ? s->E1nHc : nullptr,
                                                            pj_for_e1nhc);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

int ib_regT(Handle* h, const double* U, const double* V, const double* W, double* Eu) {
  return gather3(h, G_E, U, V, W, Eu);
}
int ib_regT_1n(Handle* h, const double* U, const double* V, const double* W, double* E) {
  return gather3(h, G_E1N, U, V, W, E);
}
int ib_regTc_1n(Handle* h, const double* P, double* E) { return gather_c(h, P, 1.0, E); }

int ib_reg(Handle* h, int comp, const double* f, double* F) {
  IbState* s = h->ib;
  const Dims& d = h->d;
  const int64_t n = comp == 1 ? sizeU(d) : (comp == 2 ? sizeV(d) : sizeW(d));
  C3D_CUDA_TRY(h, cudaMemsetAsync(F, 0, 8 * n, h->stream));
  (void)s;
  return spread(h, S_RAW, comp - 1, 1, f, 0.0, F, nullptr, nullptr, s->iy_lo, s->iy_hi);
}

// schur(Sf, f), src/projection.f90:98-144
int ib_schur(Handle* h, const double* f, double* Sf, double dt) {
  IbState* s = h->ib;
  const int nb = s->nb;
  int rc;
  // :106-120 on the band of y rows the markers' stencils reach
  const int jlo = s->iy_lo - 1, jhi = s->iy_hi + 1;
  if ((rc = reg_all_band(h, S_JUMP, f, dt, jlo - 1, jhi + 1))) return rc;
  if ((rc = launch_poisson_of_div_band(h, s->Ureg, s->Vreg, s->Wreg, h->rhs_p, jlo, jhi))) return rc;
  // Sf(u) = E(G phi - U_reg) - E1nH_ext*dudn                          :129-140
  // (G phi - U_reg formed once on the stencil rows, then gathered) and
  // Sf(p) = -E1n_c(phi/dt), gathered in the same launch;
  // then the mean removal and -E1nHc_ext*p_jump                       :123-126
  const Dims& d = h->d;
  const int64_t npts = (int64_t)d.Nx * (s->iy_hi - s->iy_lo + 1) * d.Nz;
  k_grad_minus_reg<<<(unsigned)std::min<int64_t>((npts + 255) / 256, 148 * 8), 256, 0, h->stream>>>(
      d, h->m, h->rhs_p, s->Ureg, s->Vreg, s->Wreg, s->Ut, s->Vt, s->Wt, s->iy_lo, s->iy_hi);
  C3D_LAUNCH_CHECK(h);
  GatherArgs a{};
  a.T = tables(h); a.d = d;
  const GField fs[3] = {gf_u(d, s->Ut), gf_v(d, s->Vt), gf_w(d, s->Wt)};
  for (int c = 0; c < 3; ++c) a.comp[c] = GComp{fs[c], c, G_E, 1.0, s->E1nH, f, nullptr};
  a.comp[3] = GComp{GField{h->rhs_p, d.nxg - 2, d.nyg - 2, 1, 1.0 / dt}, 3, G_E1N, -1.0, nullptr, nullptr, nullptr};
  a.ncomp = 4; a.out = Sf;
  launch_gather_tile(a, h->stream);
  C3D_LAUNCH_CHECK(h);
  return remove_mean(h, Sf + 3 * nb, f + 3 * nb);
}

static int dot(Handle* h, const double* a, const double* b, const double* c, const double* e, int op,
               int slot0 = 6) {
  IbState* s = h->ib;
  const int64_t n = 4 * (int64_t)s->nb;
  k_dot2<<<kIbRedBlocks, 256, 0, h->stream>>>(a, b, c, e, n, s->red);
  C3D_LAUNCH_CHECK(h);
  k_dot_final<<<1, 256, 0, h->stream>>>(s->red, kIbRedBlocks, s->sc, slot0, op);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// diagonal (Jacobi) preconditioner: diag(S) estimated by probing with
// well-separated unit vectors per unknown block
static int build_jacobi(Handle* h, double dt);
static bool jacobi_stale(Handle* h, double dt);

// bicgstab(x, b), src/projection.f90:146-186, right-preconditioned when a
// preconditioner is selected.  Modes: NONE (the reference's unpreconditioned
// solver), JACOBI (per-marker 4x4 diagonal blocks from lattice probing), SPAI
// (probed 4x4 block sparse approximate inverse), BAND (the banded z-Fourier
// inverse of the probed lattice band of S) and LEARNED (the same banded
// inverse with the band predicted by the network, plus a warm start: the
// extrapolated solution history, then x0 += M r0).  In LEARNED mode the
// probed band takes over, restarting from the current iterate, when the
// residual stalls (the best residual of the last kStallWindow iterations is
// not 1 % below the best before them), when the solve is slow (twice the
// iterations of the recent probed-band solves, and 20 more) or when it
// breaks down (non-finite scalars; restart from the entry guess); after
// kSlowLimit slow solves in a row the probed band serves LEARNED until the
// network is trained again.  The iterations run as one CUDA graph launch
// per solve (per kBcgChunk iterations in LEARNED mode, which checks between
// launches).
static const int kStallWindow = 20;
static const int kBcgChunk = 10;       // LEARNED: iterations per graph launch between stall checks
static const int kSlowLimit = 2;       // consecutive slow LEARNED solves before the probed band serves
static int learned_warm_start(Handle* h, double* x);
static int push_history(Handle* h, const double* x);

static int bcg_restart(Handle* h, const double* b, double* x, double dt, unsigned gb) {
  IbState* s = h->ib;
  const int64_t n = 4 * (int64_t)s->nb;
  int rc;
  if ((rc = ib_schur(h, x, s->r, dt))) return rc;                    // r = b - S x
  k_axpby<<<gb, 256, 0, h->stream>>>(n, 1.0, b, -1.0, s->r, s->r);
  C3D_LAUNCH_CHECK(h);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->rhat, s->r, 8 * n, cudaMemcpyDeviceToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaMemsetAsync(s->nu, 0, 8 * n, h->stream));
  C3D_CUDA_TRY(h, cudaMemsetAsync(s->p, 0, 8 * n, h->stream));
  k_bcg_init<<<1, 1, 0, h->stream>>>(s->sc);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// One BiCGSTAB iteration (src/projection.f90:160-184): the launches only,
// no host synchronisation, so that it can be captured into a graph.
static int bcg_iteration(Handle* h, double* x, double dt, const double* blk, bool band) {
  IbState* s = h->ib;
  const int nb = s->nb;
  const int64_t n = 4 * (int64_t)nb;
  const unsigned gb = 148 * 4;
  const unsigned gm = (unsigned)((nb + 255) / 256);
  int rc;
  if ((rc = dot(h, s->rhat, s->r, nullptr, nullptr, 0))) return rc;           // rho_n, bta
  k_bcg_p<<<gb, 256, 0, h->stream>>>(n, s->r, s->p, s->nu, s->ph, nullptr, s->sc);
  C3D_LAUNCH_CHECK(h);
  if (band) {
    if ((rc = band_apply(h, s->p, s->ph))) return rc;
  } else if (blk) {
    k_apply_blocks<<<gm, 256, 0, h->stream>>>(nb, blk, s->p, s->ph);
    C3D_LAUNCH_CHECK(h);
  }
  if ((rc = ib_schur(h, s->ph, s->nu, dt))) return rc;
  if ((rc = dot(h, s->rhat, s->nu, nullptr, nullptr, 1))) return rc;          // alpha
  k_bcg_s<<<gb, 256, 0, h->stream>>>(n, s->r, s->nu, s->s, s->sh, x, s->ph, nullptr, s->sc);
  C3D_LAUNCH_CHECK(h);
  if (band) {
    if ((rc = band_apply(h, s->s, s->sh))) return rc;
  } else if (blk) {
    k_apply_blocks<<<gm, 256, 0, h->stream>>>(nb, blk, s->s, s->sh);
    C3D_LAUNCH_CHECK(h);
  }
  if ((rc = ib_schur(h, s->sh, s->t, dt))) return rc;
  if ((rc = dot(h, s->t, s->s, s->t, s->t, 2))) return rc;                    // om
  k_bcg_x<<<kIbRedBlocks, 256, 0, h->stream>>>(n, x, s->r, s->s, s->sh, s->t, s->sc, s->red);
  C3D_LAUNCH_CHECK(h);
  k_dot_final<<<1, 256, 0, h->stream>>>(s->red, kIbRedBlocks, s->sc, 0, 3);   // err
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// End of a captured iteration: count it, record its squared residual and
// keep the WHILE node looping while the residual is finite and at or above
// the tolerance and the launch's iteration limit is not reached.
__global__ void k_bcg_loop(cudaGraphConditionalHandle cond, const double* __restrict__ sc, int* __restrict__ loop,
                           double* __restrict__ hist, double eps) {
  const double err = sc[5];
  const int it = loop[0] + 1;
  loop[0] = it;
  hist[it - 1] = err;
  const bool go = isfinite(err) && err >= eps && it < loop[1];
  cudaGraphSetConditional(cond, go ? 1u : 0u);
}

// The iteration loop as one executable graph: a conditional WHILE node
// whose body (one iteration and k_bcg_loop) runs until k_bcg_loop stops it,
// so a solve costs one graph launch and one host synchronisation instead of
// one per iteration.  What the body bakes in (mode, factors, operand
// pointers, dt, tolerance, the band of stencil rows) is the graph's key;
// the graph is re-captured when it changes.  Sets bcg_graph_off, and
// leaves the loop to the host, when conditional nodes are unavailable.
static int bcg_graph_ready(Handle* h, double* x, double dt, const double* blk, bool band, int mode, double eps) {
  IbState* s = h->ib;
  const bool block = band && s->band ? band_is_block(h) : false;
  const std::vector<double> key = {(double)mode, (double)block, (double)(uintptr_t)blk, (double)(uintptr_t)x,
                                   dt, eps, (double)s->iy_lo, (double)s->iy_hi, (double)h->p.cg_max_iter,
                                   (double)s->nb};
  if (s->bcg_exec && key == s->bcg_key) return 0;
  if (s->bcg_exec) { cudaGraphExecDestroy(s->bcg_exec); s->bcg_exec = nullptr; }
  if (s->bcg_graph) { cudaGraphDestroy(s->bcg_graph); s->bcg_graph = nullptr; }
  cudaGraph_t g = nullptr;
  C3D_CUDA_TRY(h, cudaGraphCreate(&g, 0));
  s->bcg_graph = g;
  cudaGraphConditionalHandle cond;
  cudaGraphNodeParams np{};
  cudaGraphNode_t node;
  if (cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault) != cudaSuccess ||
      (np.type = cudaGraphNodeTypeConditional, np.conditional.handle = cond,
       np.conditional.type = cudaGraphCondTypeWhile, np.conditional.size = 1,
       cudaGraphAddNode(&node, g, nullptr, 0, &np) != cudaSuccess)) {
    cudaGetLastError();
    s->bcg_graph_off = true;
    return 0;
  }
  cudaGraph_t body = np.conditional.phGraph_out[0];
  const bool pdl = h->use_pdl;
  h->use_pdl = false;                 // plain kernel nodes in the body
  const int64_t l0 = h->launches;
  C3D_CUDA_TRY(h, cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  int rc = bcg_iteration(h, x, dt, blk, band);
  if (rc == 0) {
    k_bcg_loop<<<1, 1, 0, h->stream>>>(cond, s->sc, s->loop_d, s->hist_d, eps);
    if (cudaGetLastError() != cudaSuccess) rc = C3D_ERR_CUDA;
    else h->launches++;
  }
  cudaGraph_t captured = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(h->stream, &captured);
  h->use_pdl = pdl;
  s->bcg_body_launches = h->launches - l0;
  h->launches = l0;
  if (rc) return rc;
  if (ec != cudaSuccess) { h->last_error = std::string("BiCGSTAB graph capture: ") + cudaGetErrorString(ec); return C3D_ERR_CUDA; }
  cudaGraphExec_t ex = nullptr;
  C3D_CUDA_TRY(h, cudaGraphInstantiate(&ex, g, 0));
  s->bcg_exec = ex;
  s->bcg_key = key;
  return 0;
}

// the predicted band is redone when dt changed or a marker moved by more
// than 0.03 dymin since the prediction (the probed band's rule)
bool learned_stale(Handle* h, double dt) {
  IbState* s = h->ib;
  if (s->dt_at_lrn != dt || s->yb_at_lrn.size() != s->yb.size()) return true;
  double mx = 0.0;
  for (size_t k = 0; k < s->yb.size(); ++k) {
    mx = std::max(mx, std::fabs(s->yb[k] - s->yb_at_lrn[k]));
    mx = std::max(mx, std::fabs(s->xb[k] - s->xb_at_lrn[k]));
  }
  return mx > 0.03 * h->dymin;
}

void ib_rows(const Handle* h, int32_t rows[2]) {
  rows[0] = h->ib ? h->ib->iy_lo : 0;
  rows[1] = h->ib ? h->ib->iy_hi : 0;
}

int ib_bicgstab(Handle* h, const double* b, double dt) {
  IbState* s = h->ib;
  const int64_t n = 4 * (int64_t)s->nb;
  const unsigned gb = 148 * 4;
  int rc;
  int mode = h->precond_mode;
  if (mode == C3D_PRECOND_LEARNED && s->lrn_slow >= kSlowLimit) {
    // the network's band was slow on consecutive solves: the probed band
    // serves until the network is trained again
    h->stats.precond_fallbacks++;
    mode = C3D_PRECOND_BAND;
  }
  const bool pure_band = mode == C3D_PRECOND_BAND;
  if (!s->ev_a) {
    C3D_CUDA_TRY(h, cudaEventCreate(&s->ev_a));
    C3D_CUDA_TRY(h, cudaEventCreate(&s->ev_b));
  }
  // band factors: probed (BAND) when stale, or predicted by the network
  // (LEARNED) at every new geometry; timed as preconditioner builds
  const bool need_probe = mode == C3D_PRECOND_BAND && band_stale(h, dt);
  const bool need_learn = mode == C3D_PRECOND_LEARNED && (!s->have_lrn || learned_stale(h, dt));
  // allocations out of the timed build
  if (need_learn && (rc = mlp_prepare_band(h))) return rc;
  if (need_probe && !s->prb && (rc = dev_alloc(h, &s->prb, 16 * (int64_t)s->nb))) return rc;
  if (need_probe || need_learn) {
    C3D_CUDA_TRY(h, cudaEventRecord(s->ev_a, h->stream));
    if (need_probe) {
      if ((rc = band_build(h, dt))) return rc;
      if (mlp_collecting(h) && (rc = mlp_add_probe_set(h))) return rc;
    } else if ((rc = mlp_build_band(h, dt))) {
      if (rc != C3D_ERR_NAN) return rc;
      // the predicted band is singular: the probed band takes over
      h->stats.precond_fallbacks++;
      mode = C3D_PRECOND_BAND;
      if ((rc = band_build(h, dt))) return rc;
    }
    C3D_CUDA_TRY(h, cudaEventRecord(s->ev_b, h->stream));
    C3D_CUDA_TRY(h, cudaEventSynchronize(s->ev_b));
    float bms = 0.f;
    C3D_CUDA_TRY(h, cudaEventElapsedTime(&bms, s->ev_a, s->ev_b));
    h->stats.precond_build_ms += bms;
    h->stats.precond_builds += need_learn ? 1 : 0;
  }
  if ((mode == C3D_PRECOND_JACOBI || mode == C3D_PRECOND_SPAI) && jacobi_stale(h, dt)) {
    if ((rc = build_jacobi(h, dt))) return rc;
  }
  const double* blk = mode == C3D_PRECOND_JACOBI ? s->jac_blk
                      : mode == C3D_PRECOND_SPAI ? s->spai_blk : nullptr;
  bool band = mode == C3D_PRECOND_BAND || mode == C3D_PRECOND_LEARNED;
  double* x = s->fb;
  C3D_CUDA_TRY(h, cudaEventRecord(s->ev_a, h->stream));
  if (mode == C3D_PRECOND_LEARNED && (rc = learned_warm_start(h, x))) return rc;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->scr1, x, 8 * n, cudaMemcpyDeviceToDevice, h->stream));
  if ((rc = bcg_restart(h, b, x, dt, gb))) return rc;
  if (mode == C3D_PRECOND_LEARNED) {
    // warm start x0 += M r0
    if ((rc = band_apply(h, s->r, s->scr2))) return rc;
    k_axpby<<<gb, 256, 0, h->stream>>>(n, 1.0, x, 1.0, s->scr2, x);
    C3D_LAUNCH_CHECK(h);
    if ((rc = bcg_restart(h, b, x, dt, gb))) return rc;
  }
  const double eps = h->p.cg_tol * h->p.cg_tol;
  double err = 1.0;
  int it = 0;
  std::vector<double> hist;
  const int maxit = h->p.cg_max_iter;
  if (s->hist_cap < maxit) {
    if ((rc = dev_alloc(h, &s->hist_d, maxit))) return rc;
    s->hist_cap = maxit;
  }
  if (!s->loop_d && (rc = dev_alloc(h, &s->loop_d, 2))) return rc;
  while (it < maxit && err >= eps) {
    // LEARNED checks for stalls every kBcgChunk iterations; the other modes
    // run the whole solve in one launch
    const int lim = mode == C3D_PRECOND_LEARNED ? std::min(maxit, it + kBcgChunk) : maxit;
    int done = it;
    if (!s->bcg_graph_off && (rc = bcg_graph_ready(h, x, dt, blk, band, mode, eps)) == 0 && !s->bcg_graph_off) {
      const int lc[2] = {it, lim};
      C3D_CUDA_TRY(h, cudaMemcpyAsync(s->loop_d, lc, sizeof(lc), cudaMemcpyHostToDevice, h->stream));
      C3D_CUDA_TRY(h, cudaGraphLaunch(s->bcg_exec, h->stream));
      C3D_CUDA_TRY(h, cudaMemcpyAsync(&done, s->loop_d, 4, cudaMemcpyDeviceToHost, h->stream));
      C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
      if (done <= it || done > lim) { h->last_error = "BiCGSTAB graph: bad iteration count"; return C3D_ERR_CUDA; }
      h->launches += s->bcg_body_launches * (done - it);
    } else {
      if (rc) return rc;
      // host-driven iteration (conditional graphs unavailable)
      if ((rc = bcg_iteration(h, x, dt, blk, band))) return rc;
      done = it + 1;
      C3D_CUDA_TRY(h, cudaMemcpyAsync(s->hist_d + it, s->sc + 5, 8, cudaMemcpyDeviceToDevice, h->stream));
    }
    const size_t h0 = hist.size();
    hist.resize(h0 + (done - it));
    C3D_CUDA_TRY(h, cudaMemcpyAsync(hist.data() + h0, s->hist_d + it, 8 * (size_t)(done - it),
                                    cudaMemcpyDeviceToHost, h->stream));
    C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    it = done;
    err = hist.back();
    if (mode == C3D_PRECOND_LEARNED) {
      const bool broke = !(err == err) || std::isinf(err);
      // stall: the best residual of the last kStallWindow iterations is not
      // 1 % below the best one before them
      bool stalled = false;
      if ((int)hist.size() > kStallWindow) {
        const size_t cut = hist.size() - kStallWindow;
        const double before = *std::min_element(hist.begin(), hist.begin() + cut);
        const double recent = *std::min_element(hist.begin() + cut, hist.end());
        stalled = recent > 0.98 * before;   // squared norms: |r| down < 1 %
      }
      // slow: the probed band's recent solves needed fewer than half as many
      // iterations (and 20 fewer): the predicted band fits this geometry badly
      const double ref = s->band_iters_ref;
      const bool slow = ref > 0.0 && it >= std::max(2.0 * ref, ref + 20.0);
      if (slow) s->lrn_slow++;
      if (broke || stalled || slow) {
        // the probed band of the current geometry takes over
        h->stats.precond_fallbacks++;
        mode = C3D_PRECOND_BAND;
        if ((rc = band_build(h, dt))) return rc;
        s->have_lrn = false;
        if (broke)   // the iterate may be polluted: restart from the entry guess
          C3D_CUDA_TRY(h, cudaMemcpyAsync(x, s->scr1, 8 * n, cudaMemcpyDeviceToDevice, h->stream));
        if ((rc = bcg_restart(h, b, x, dt, gb))) return rc;
        hist.clear();
        err = 1.0;
      }
    }
  }
  if (err == err && (rc = push_history(h, x))) return rc;
  if (pure_band && err < eps)
    s->band_iters_ref = s->band_iters_ref > 0.0 ? 0.5 * (s->band_iters_ref + it) : (double)it;
  if (h->precond_mode == C3D_PRECOND_LEARNED && mode == C3D_PRECOND_LEARNED && err < eps) s->lrn_slow = 0;
  C3D_CUDA_TRY(h, cudaEventRecord(s->ev_b, h->stream));
  C3D_CUDA_TRY(h, cudaEventSynchronize(s->ev_b));
  float ms = 0.f;
  C3D_CUDA_TRY(h, cudaEventElapsedTime(&ms, s->ev_a, s->ev_b));
  h->stats.last_bicgstab_ms = ms;
  h->stats.bicgstab_ms += ms;
  h->stats.precond_mode = mode;
  h->stats.bicgstab_solves++;
  h->stats.bicgstab_iters += it;
  h->stats.last_bicgstab_iters = it;
  h->stats.last_residual = std::sqrt(err);
  if (!(err == err)) { h->last_error = "BiCGSTAB produced a non-finite residual"; return C3D_ERR_NAN; }
  if (it == h->p.cg_max_iter && err >= eps) return C3D_WARN_NOT_CONVERGED;
  return 0;
}

// squared errors of the order-0, -1 and -2 extrapolations of the newest
// solution h0 from the three before it: |h0 - h1|^2, |h0 - (2 h1 - h2)|^2,
// |h0 - (3 h1 - 3 h2 + h3)|^2, block partials
__global__ void __launch_bounds__(256) k_extrap_err(const double* __restrict__ h0, const double* __restrict__ h1,
                                                   const double* __restrict__ h2, const double* __restrict__ h3,
                                                   int64_t n, double* __restrict__ part) {
  double e0 = 0.0, e1 = 0.0, e2 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a = h0[i] - h1[i];
    const double b = h0[i] - (2.0 * h1[i] - h2[i]);
    const double c = h0[i] - (3.0 * h1[i] - 3.0 * h2[i] + h3[i]);
    e0 += a * a;
    e1 += b * b;
    e2 += c * c;
  }
  __shared__ double sa[3][256];
  sa[0][threadIdx.x] = e0;
  sa[1][threadIdx.x] = e1;
  sa[2][threadIdx.x] = e2;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int q = 0; q < 3; ++q) sa[q][threadIdx.x] += sa[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; ++q) part[3 * blockIdx.x + q] = sa[q][0];
}

// x = extrapolation of order 0, 1 or 2 from h0 (newest), h1, h2
__global__ void k_extrap(int64_t n, int order, const double* __restrict__ h0, const double* __restrict__ h1,
                         const double* __restrict__ h2, double* __restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = order == 0 ? h0[i] : order == 1 ? 2.0 * h0[i] - h1[i] : 3.0 * h0[i] - 3.0 * h1[i] + h2[i];
}

// Warm start of the learned mode: the surface unknowns are smooth in time at
// a fixed RK stage, so the solution of this stage is extrapolated from the
// same stage of the previous steps.  The order (0, 1 or 2) is the one that
// best predicted the newest stored solution from those before it (chosen
// on the solver's own past solutions).  Without two stored solutions of the
// stage the current fb (the reference's warm start) is kept.
static int learned_warm_start(Handle* h, double* x) {
  IbState* s = h->ib;
  const int st = s->stage;
  s->warm_order = -1;
  if (st < 0 || s->nhist[st] < 2) return 0;
  const int64_t n = 4 * (int64_t)s->nb;
  double** H = s->hist[st];
  int order = 1;
  if (s->nhist[st] >= IbState::kHist) {
    int rc;
    if (!s->ext_part && (rc = dev_alloc(h, &s->ext_part, 3 * kIbRedBlocks))) return rc;
    k_extrap_err<<<kIbRedBlocks, 256, 0, h->stream>>>(H[0], H[1], H[2], H[3], n, s->ext_part);
    C3D_LAUNCH_CHECK(h);
    std::vector<double> part(3 * kIbRedBlocks);
    C3D_CUDA_TRY(h, cudaMemcpyAsync(part.data(), s->ext_part, 8 * part.size(), cudaMemcpyDeviceToHost, h->stream));
    C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    double e[3] = {0, 0, 0};
    for (int b = 0; b < kIbRedBlocks; ++b)
      for (int q = 0; q < 3; ++q) e[q] += part[3 * b + q];
    order = 0;
    for (int q = 1; q < 3; ++q)
      if (e[q] < e[order]) order = q;
  } else if (s->nhist[st] == 2) {
    order = 1;
  }
  if (order == 2 && s->nhist[st] < 3) order = 1;
  k_extrap<<<148 * 4, 256, 0, h->stream>>>(n, order, H[0], H[1], H[2], x);
  C3D_LAUNCH_CHECK(h);
  s->warm_order = order;
  return 0;
}

// keep the converged solution of this RK stage (newest first)
static int push_history(Handle* h, const double* x) {
  IbState* s = h->ib;
  const int st = s->stage;
  if (st < 0) return 0;
  const int64_t n = 4 * (int64_t)s->nb;
  int rc;
  double** H = s->hist[st];
  if (!H[IbState::kHist - 1]) {
    for (int k = 0; k < IbState::kHist; ++k)
      if ((rc = dev_alloc(h, &H[k], n))) return rc;
  }
  double* oldest = H[IbState::kHist - 1];
  for (int k = IbState::kHist - 1; k > 0; --k) H[k] = H[k - 1];
  H[0] = oldest;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(H[0], x, 8 * n, cudaMemcpyDeviceToDevice, h->stream));
  s->nhist[st] = std::min(s->nhist[st] + 1, IbState::kHist);
  return 0;
}

// out = M in for the preconditioner of the current mode (built when missing
// or stale); the identity without one
int ib_precond_apply(Handle* h, const double* in, double* out, double dt) {
  IbState* s = h->ib;
  const int nb = s->nb;
  const int64_t n = 4 * (int64_t)nb;
  const int mode = h->precond_mode;
  int rc;
  if (mode == C3D_PRECOND_BAND) {
    if (band_stale(h, dt) && (rc = band_build(h, dt))) return rc;
    return band_apply(h, in, out);
  }
  if (mode == C3D_PRECOND_LEARNED) {
    if ((!s->have_lrn || learned_stale(h, dt)) && (rc = mlp_build_band(h, dt))) return rc;
    return band_apply(h, in, out);
  }
  if (mode == C3D_PRECOND_NONE) {
    C3D_CUDA_TRY(h, cudaMemcpyAsync(out, in, 8 * n, cudaMemcpyDeviceToDevice, h->stream));
    return 0;
  }
  if (jacobi_stale(h, dt) && (rc = build_jacobi(h, dt))) return rc;
  const double* blk = mode == C3D_PRECOND_JACOBI ? s->jac_blk : s->spai_blk;
  k_apply_blocks<<<(unsigned)((nb + 255) / 256), 256, 0, h->stream>>>(nb, blk, in, out);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// Probe pass: lattice colour classes (ix = cx mod px, iz = cz mod pz, px =
// pz = 5, beyond the 5-point delta support), one unit probe per component and
// class, 4*px*pz Schur applications in all.  Fills the Jacobi and SPAI
// blocks; with mom != null also the SPAI training moments.
int ib_probe(Handle* h, double dt, float* mom) {
  IbState* s = h->ib;
  const int nb = s->nb;
  const int64_t n = 4 * (int64_t)nb;
  const int lat = s->lat_nx > 0 ? s->lat_nx : nb;
  const int nrow = (nb + lat - 1) / lat;
  const int px = std::min(5, lat), pz = std::min(5, nrow);
  const unsigned gb = 148 * 4;
  int rc;
  if (s->prb == nullptr && (rc = dev_alloc(h, &s->prb, 4 * n))) return rc;
  C3D_CUDA_TRY(h, cudaMemsetAsync(s->jac_blk, 0, 16 * 8 * (size_t)nb, h->stream));
  for (int cz = 0; cz < pz; ++cz)
    for (int cx = 0; cx < px; ++cx) {
      for (int blk = 0; blk < 4; ++blk) {
        k_probe_mask<<<gb, 256, 0, h->stream>>>(nb, lat, blk, px, pz, cx, cz, s->scr0);
        C3D_LAUNCH_CHECK(h);
        if ((rc = ib_schur(h, s->scr0, s->prb + (size_t)blk * n, dt))) return rc;
      }
      k_probe_spai<<<(nb + 127) / 128, 128, 0, h->stream>>>(nb, lat, nrow, px, pz, cx, cz, s->prb, s->jac_blk,
                                                            s->spai_blk, mom);
      C3D_LAUNCH_CHECK(h);
    }
  // safeguard: the diagonal of S can be small or change sign on some markers
  // (a moving plane crossing the stretched y cells); entries below 0.2 of the
  // component's median magnitude, or of the other sign, take the median
  std::vector<double> jb((size_t)16 * nb);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(jb.data(), s->jac_blk, 8 * jb.size(), cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int c = 0; c < 4; ++c) {
    std::vector<double> dg(nb);
    for (int l = 0; l < nb; ++l) dg[l] = 1.0 / jb[16 * (size_t)l + 5 * c];
    std::vector<double> tmp(dg);
    std::nth_element(tmp.begin(), tmp.begin() + nb / 2, tmp.end());
    const double med = tmp[nb / 2];
    int clipped = 0;
    for (int l = 0; l < nb; ++l) {
      const double d = dg[l];
      if (!(std::fabs(d) >= 0.2 * std::fabs(med)) || (d > 0) != (med > 0)) {
        jb[16 * (size_t)l + 5 * c] = 1.0 / med;
        ++clipped;
      }
    }
    s->jac_clipped[c] = clipped;
  }
  C3D_CUDA_TRY(h, cudaMemcpyAsync(s->jac_blk, jb.data(), 8 * jb.size(), cudaMemcpyHostToDevice, h->stream));
  s->have_jac = true;
  s->yb_at_jac = s->yb;
  s->dt_at_jac = dt;
  return 0;
}

static int build_jacobi(Handle* h, double dt) { return ib_probe(h, dt, nullptr); }

// the Jacobi blocks are re-probed when dt changed or a marker moved by more
// than a tenth of the smallest wall-normal spacing since the last probe
static bool jacobi_stale(Handle* h, double dt) {
  IbState* s = h->ib;
  if (!s->have_jac || s->dt_at_jac != dt || s->yb_at_jac.size() != s->yb.size()) return true;
  double mx = 0.0;
  for (size_t k = 0; k < s->yb.size(); ++k) mx = std::max(mx, std::fabs(s->yb[k] - s->yb_at_jac[k]));
  return mx > 0.1 * h->dymin;
}

// compute_heaviside, src/heaviside.f90:20-54
int ib_heaviside(Handle* h) {
  IbState* s = h->ib;
  const Dims& d = h->d;
  int rc;
  if ((rc = reg_all(h, S_NORMAL, nullptr, 0.0))) return rc;                       // :30-33
  if ((rc = launch_divergence(h, s->Ureg, s->Vreg, s->Wreg, s->Hce))) return rc;  // :35
  k_negate<<<148 * 8, 256, 0, h->stream>>>(sizeR(d), s->Hce);                   // :36
  C3D_LAUNCH_CHECK(h);
  if ((rc = launch_poisson_solve(h, s->Hce, 0, h->dt))) return rc;               // :37
  k_one_minus<<<148 * 8, 256, 0, h->stream>>>(sizeR(d), s->Hce, s->Hce);         // :38 Hc_ext
  C3D_LAUNCH_CHECK(h);
  dim3 b(32, 4, 2), g((d.Nx + 31) / 32, (d.Ny + 3) / 4, (d.Nz + 1) / 2);
  k_heaviside_interp<<<g, b, 0, h->stream>>>(d, s->Hce, s->Ut, s->Vt, s->Wt);     // :40-42
  C3D_LAUNCH_CHECK(h);
  if ((rc = launch_fill_ghosts3(h, s->Ut, s->Vt, s->Wt))) return rc;              // :43
  k_one_minus<<<148 * 8, 256, 0, h->stream>>>(sizeU(d), s->Ut, s->Hu);           // :45-47
  k_one_minus<<<148 * 8, 256, 0, h->stream>>>(sizeV(d), s->Vt, s->Hv);
  k_one_minus<<<148 * 8, 256, 0, h->stream>>>(sizeW(d), s->Wt, s->Hw);
  C3D_LAUNCH_CHECK(h);
  if ((rc = launch_fill_ghosts3(h, s->Hu, s->Hv, s->Hw))) return rc;              // :49
  if ((rc = gather_c(h, s->Hce, 1.0, s->E1nHc))) return rc;                       // :51
  if ((rc = gather3(h, G_E1N, s->Ut, s->Vt, s->Wt, s->E1nH))) return rc;          // :52
  return 0;
}

// compute_IB_projection, src/projection.f90:48-96.  On entry U,V,W hold the
// non-IB projected field, Us,Vs,Ws the field before it (U_interim), and
// P_interim the non-IB pseudo-pressure / dt.
int ib_projection(Handle* h, double dt, int rk_step) {
  IbState* s = h->ib;
  const int nb = s->nb;
  int rc;
  // rhs(u) = -E u + ub;  rhs(p) = -E1n_c(P_interim), mean removed   :51-57
  if ((rc = gather3(h, G_E, h->U, h->V, h->W, s->rhs, -1.0, nullptr, nullptr, s->ub_d))) return rc;
  if ((rc = gather_c(h, h->P_interim, 1.0, s->rhs + 3 * nb, -1.0))) return rc;
  if ((rc = remove_mean(h, s->rhs + 3 * nb, nullptr))) return rc;
  s->stage = (rk_step >= 1 && rk_step <= 3) ? rk_step - 1 : -1;
  rc = ib_bicgstab(h, s->rhs, dt);                                              // :60
  s->stage = -1;
  if (rc < 0) return rc;
  const int warn = rc;
  // R f, divergence, Poisson (P side effect at rk_step 1), final update   :63-94
  if ((rc = reg_all(h, S_JUMP, s->fb, dt))) return rc;
  if ((rc = launch_poisson_of_div(h, s->Ureg, s->Vreg, s->Wreg, h->rhs_p, rk_step, dt))) return rc;
  const Dims& d = h->d;
  dim3 b(32, 4, 2), g((d.Nx + 31) / 32, (d.Ny + 3) / 4, (d.Nz + 1) / 2);
  k_ib_final<<<g, b, 0, h->stream>>>(d, h->m, h->Us, h->Vs, h->Ws, s->Ureg, s->Vreg, s->Wreg,
                                     h->P_interim, h->rhs_p, dt, h->U, h->V, h->W);
  C3D_LAUNCH_CHECK(h);
  if ((rc = launch_fill_ghosts3(h, h->U, h->V, h->W))) return rc;
  return warn;
}

double* ib_marker_ptr(Handle* h, int id, int64_t* len) {
  IbState* s = h->ib;
  if (!s) return nullptr;
  const int nb = s->nb;
  switch (id) {
    case C3D_MARKER_FB: *len = 4 * (int64_t)nb; return s->fb;
    case C3D_MARKER_UB: *len = 3 * (int64_t)nb; return s->ub_d;
    case C3D_MARKER_XB: *len = nb; return s->xb_d;
    case C3D_MARKER_YB: *len = nb; return s->yb_d;
    case C3D_MARKER_ZB: *len = nb; return s->zb_d;
    case C3D_MARKER_NORMALS: *len = 3 * (int64_t)nb; return s->nrm_d;
    case C3D_MARKER_SB: *len = nb; return s->sb_d;
    case C3D_MARKER_E1NH_EXT: *len = 3 * (int64_t)nb; return s->E1nH;
    case C3D_MARKER_E1NHC_EXT: *len = nb; return s->E1nHc;
    default: return nullptr;
  }
}

double* ib_field_ptr(Handle* h, int id) {
  IbState* s = h->ib;
  if (!s) return nullptr;
  switch (id) {
    case C3D_FIELD_U_REG: return s->Ureg;
    case C3D_FIELD_V_REG: return s->Vreg;
    case C3D_FIELD_W_REG: return s->Wreg;
    case C3D_FIELD_HU_INTERIOR: return s->Hu;
    case C3D_FIELD_HV_INTERIOR: return s->Hv;
    case C3D_FIELD_HW_INTERIOR: return s->Hw;
    case C3D_FIELD_HC_EXTERIOR: return s->Hce;
    default: return nullptr;
  }
}

double* ib_scratch(Handle* h, int which) {
  IbState* s = h->ib;
  if (!s) return nullptr;
  return which == 0 ? s->scr0 : (which == 1 ? s->scr1 : s->scr2);
}

int ib_nb(Handle* h) { return h->ib ? h->ib->nb : 0; }
const double* ib_hu(Handle* h) { return h->ib ? h->ib->Hu : nullptr; }
const double* ib_hv(Handle* h) { return h->ib ? h->ib->Hv : nullptr; }
const double* ib_hw(Handle* h) { return h->ib ? h->ib->Hw : nullptr; }
bool ib_moving(Handle* h) { return h->ib && h->ib->moving; }

}  // namespace c3d
