/*
 * fl_mm_oracle.c -- CPU oracle for the ghost-fluid steps of the two-material
 * path: the Riemann ghost-fluid method (star states written beside the
 * interface), the ghost-cell extrapolation into the band outside each
 * material, state initialisation inside a level set and the final merge.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement used by tests/ as the
 * checker; the product never links it.  2-D grids, x fastest, SoA states
 * (rho, E, m_x, m_y) with `pitch`, held as doubles; with f32 != 0 every value
 * written back is rounded to float, as the FP32 kernels store it.  Level sets
 * are FP64.  Reads outside the domain mirror it (ghost[-1-g] = cell[g]).
 *
 * Defined semantics (the reference's versions do not run as shipped: debug
 * printf in every thread, a 2-D interpolation that forms arrays of
 * references, unsynchronised neighbour reads):
 *  - the GFM reads the states as they were before the pass; when several
 *    sources write one target cell, the source with the highest flat index
 *    wins (a sequential raster loop);
 *  - a source whose level-set gradient vanishes is skipped, and a target
 *    outside the domain is not written;
 *  - the probe states use the arithmetic of the reference's 2-D math::interp
 *    (math/interp.hpp:120-167) as it computes, which is not the bilinear form
 *    its comment documents: with X0, X1 the cells offset by off_x and
 *    off_x + sign along x from the source and Y0, Y1 those offset along y,
 *    close = X0(1-fx) + X1 fx, far = Y0(1-fx) + Y1 fx, r = close(1-fy) + far fy,
 *    in double (pinned to the reference's function, tests/test_levelset_pinned.py);
 *  - the extrapolation is a Jacobi iteration over the band cells, stopped
 *    when no cell changes by 1e-8 or more (L1 over the components, the
 *    reference's per-cell tolerance) or after max_iters sweeps.
 * Parity pin: the reference's multimaterial driver does not run, but the
 * per-source body of RiemannGFM::invoke (steps 1-4: normal, probe
 * interpolation, rotation, two-material HLLC star state, rotation back) runs
 * on the host with the reference's own functors (oracle/ref_driver_ls.cpp);
 * flo_mm_gfm_star is pinned to it bit for bit.  The CUDA kernels are checked
 * against this file.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline int64_t mir(int64_t i, int64_t n) {
  if (i < 0) i = -1 - i;
  else if (i >= n) i = 2 * n - 1 - i;
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

static inline int64_t idx(int64_t nx, int64_t ny, int64_t x, int64_t y) {
  return mir(y, ny) * nx + mir(x, nx);
}

static inline int isgn(double v) { return (0.0 < v) - (v < 0.0); }
static inline double dmaxr(double a, double b) { return (a < b) ? b : a; }  /* std::max */
static inline double st(double v, int f32) { return f32 ? (double)(float)v : v; }

/* ideal gas (state/state_impl.hpp:117-128, material/ideal_gas.hpp:75-78) */
static double pressure2(const double* u, double g) {
  const double r = u[0];
  const double vx = u[2] / r, vy = u[3] / r;
  return (g - 1.0) * (u[1] - 0.5 * r * (vx * vx + vy * vy));
}

/* sound speed with the material's p_inf (stiff_fluid.hpp:92-96; 0 for the
 * ideal gas, ideal_gas.hpp:75-78: p + 0 = p) */
static double sound2(const double* u, double g, double pinf) {
  return sqrt(g * (pressure2(u, g) + pinf) / u[0]);
}

/* Hllc::wavespeed_slr (flux_method/flux_hllc.hpp:447-462) */
static double wavespeed_slr(const double* u, double pstar, double a, double q, double g) {
  const double p = pressure2(u, g);
  const double vel = u[2] / u[0];
  if (pstar <= p) return vel + a;
  return vel + a * sqrt(1.0 + q * (pstar / p - 1.0));
}

/* Hllc::solve_star_conservative_left (flux_method/flux_hllc.hpp:330-361)
 * with q_k (:425-430), wavespeed_star (:490-513) and star_state_cons
 * (:532-568), normal direction x. */
static void star_left(const double* ul, const double* ur, double gl, double gr, double il,
                      double ir, double* out) {
  const double al = sound2(ul, gl, il), ar = sound2(ur, gr, ir);
  const double pl = pressure2(ul, gl), pr = pressure2(ur, gr);
  const double vl = ul[2] / ul[0], vr = ur[2] / ur[0];
  const double p_pvrs = 0.5 * ((pl + pr) - (0.25 * (vr - vl) * (ur[0] + ul[0]) * (al + ar)));
  const double p_star = dmaxr(0.0, p_pvrs);
  const double ql = (gl + 1.0) / (2.0 * gl), qr = (gr + 1.0) / (2.0 * gr);
  const double wsl = wavespeed_slr(ul, p_star, -al, ql, gl);
  const double wsr = wavespeed_slr(ur, p_star, ar, qr, gr);
  const double fl = ul[0] * (wsl - vl), fr = ur[0] * (wsr - vr);
  const double s_star = (pr - pl + vl * fl - vr * fr) / (fl - fr);
  const double sf = wsl - vl;
  const double scale = sf / (wsl - s_star);
  for (int c = 0; c < 4; ++c) out[c] = scale * ul[c];
  out[2] = s_star * ul[0] * scale;
  out[1] = scale * (ul[1] + ul[0] * (s_star - vl) * (s_star + pl / (ul[0] * sf)));
}

/* star_left for the pin against the reference's function */
void flo_mm_star_left(const double* ul, const double* ur, double gl, double il, double gr,
                      double ir, double* out) {
  star_left(ul, ur, gl, gr, il, ir, out);
}

static void load4(const double* u, int64_t pitch, int64_t i, double* o) {
  for (int c = 0; c < 4; ++c) o[c] = u[c * pitch + i];
}

/* probe of the state around (x, y) with offsets w (in cells), with the
 * arithmetic of the reference's 2-D math::interp (math/interp.hpp:120-167). */
static void interp2(const double* u, int64_t pitch, int64_t nx, int64_t ny, int64_t x, int64_t y,
                    const double* w, double* out) {
  int64_t off[2];
  int sg[2];
  double f[2];
  for (int d = 0; d < 2; ++d) {
    sg[d] = isgn(w[d]);
    const double aw = fabs(w[d]);
    const double ao = floor(aw);
    off[d] = (int64_t)((double)sg[d] * ao);
    f[d] = aw - ao;
  }
  double X0[4], X1[4], Y0[4], Y1[4];
  load4(u, pitch, idx(nx, ny, x + off[0], y), X0);
  load4(u, pitch, idx(nx, ny, x + off[0] + sg[0], y), X1);
  load4(u, pitch, idx(nx, ny, x, y + off[1]), Y0);
  load4(u, pitch, idx(nx, ny, x, y + off[1] + sg[1]), Y1);
  const double factor = 1.0 - f[0];
  for (int c = 0; c < 4; ++c) {
    const double close = X0[c] * factor + X1[c] * f[0];
    const double far = Y0[c] * factor + Y1[c] * f[0];
    out[c] = close * (1.0 - f[1]) + far * f[1];
  }
}

/* Is (x, y) a GFM source of material A (level set pa) against B (pb)?
 * (ghost_fluid/riemann_ghost_fluid.hpp:59-71,204-231, levelset/levelset.hpp
 * :166-219).  On success n receives grad(pa)/|grad(pa)| (norm() with dh = 1,
 * iterator/multidim_iterator.hpp:291-306). */
static int gfm_source(const double* pa, const double* pb, int64_t nx, int64_t ny, int64_t x,
                      int64_t y, double h, double* n) {
  const double phi = pa[y * nx + x];
  if (!((phi <= 0.0 || phi <= -0.0) && phi >= -h)) return 0;
  const double xm = pa[idx(nx, ny, x - 1, y)], xp = pa[idx(nx, ny, x + 1, y)];
  const double ym = pa[idx(nx, ny, x, y - 1)], yp = pa[idx(nx, ny, x, y + 1)];
  if (xm == 0.0 || xp == 0.0 || ym == 0.0 || yp == 0.0) return 0;
  const double ob = pb[y * nx + x];
  if (!((ob > 0.0 && ob < fabs(h)) || ob == 0.0)) return 0;
  const double g0 = 0.5 * (xp - xm), g1 = 0.5 * (yp - ym);
  const double mag = g0 * g0 + g1 * g1;
  const double s = sqrt(mag);
  if (!(s > 0.0)) return 0;
  n[0] = g0 / s;
  n[1] = g1 / s;
  return 1;
}

/* star state of source (x, y) of material A (riemann_ghost_fluid.hpp:70-176) */
static void gfm_star(const double* ua, const double* ub, int64_t pitch, int64_t nx, int64_t ny,
                     const double* pa, int64_t x, int64_t y, double h, const double* n, double ga,
                     double gb, double ia, double ib, double* star) {
  const double abs_phi = fabs(pa[y * nx + x]);
  const double h32 = 1.5 * h;
  double w[2], wl[4], wr[4];
  for (int d = 0; d < 2; ++d) w[d] = n[d] * (abs_phi - h32) / h;
  interp2(ua, pitch, nx, ny, x, y, w, wl);
  for (int d = 0; d < 2; ++d) w[d] = n[d] * (abs_phi + h32) / h;
  interp2(ub, pitch, nx, ny, x, y, w, wr);
  const double vl[2] = {wl[2] / wl[0], wl[3] / wl[0]};
  const double vr[2] = {wr[2] / wr[0], wr[3] / wr[0]};
  const double vl_n = vl[0] * n[0] + vl[1] * n[1];
  const double vr_n = vr[0] * n[0] + vr[1] * n[1];
  /* set_velocity on a conservative state: m = v * rho, energy untouched
   * (state/state.hpp:435-441) */
  wl[2] = vl_n * wl[0];
  wr[2] = vr_n * wr[0];
  wl[3] = 0.0 * wl[0];
  wr[3] = 0.0 * wr[0];
  star_left(wl, wr, ga, gb, ia, ib, star);
  /* rotate back, dimension by dimension on the updated star state */
  for (int d = 0; d < 2; ++d) {
    const double sv = star[2 + d] / star[0];
    const double v = vl[d] + (sv - vl_n) * n[d];
    star[2 + d] = v * star[0];
  }
}

/* Star states of listed source cells of material A (the per-source body of
 * the GFM), with the target offsets sign(n); cells that are not GFM sources
 * (gfm_source) get NaN and a zero offset. */
void flo_mm_gfm_star(int64_t nx, int64_t ny, int64_t pitch, double h, const double* ua,
                     const double* ub, const double* pa, const double* pb, double ga, double ia,
                     double gb, double ib, int64_t ncells, const int64_t* xs, const int64_t* ys,
                     double* stars, int* tx, int* ty) {
  for (int64_t k = 0; k < ncells; ++k) {
    double n[2];
    if (!gfm_source(pa, pb, nx, ny, xs[k], ys[k], h, n)) {
      for (int c = 0; c < 4; ++c) stars[4 * k + c] = NAN;
      tx[k] = ty[k] = 0;
      continue;
    }
    gfm_star(ua, ub, pitch, nx, ny, pa, xs[k], ys[k], h, n, ga, gb, ia, ib, stars + 4 * k);
    tx[k] = isgn(n[0]);
    ty[k] = isgn(n[1]);
  }
}

/* GFM for both materials from the pre-pass states; u0/u1 updated in place.
 * Returns the number of target cells written. */
int64_t flo_mm_gfm_mat(int64_t nx, int64_t ny, int64_t pitch, double h, double g0, double i0,
                       double g1, double i1, double* u0, double* u1, const double* p0,
                       const double* p1, int f32) {
  const int64_t n = nx * ny;
  double* snap0 = (double*)malloc(sizeof(double) * 4 * pitch);
  double* snap1 = (double*)malloc(sizeof(double) * 4 * pitch);
  memcpy(snap0, u0, sizeof(double) * 4 * pitch);
  memcpy(snap1, u1, sizeof(double) * 4 * pitch);
  int64_t written = 0;
  for (int m = 0; m < 2; ++m) {
    const double* pa = m == 0 ? p0 : p1;
    const double* pb = m == 0 ? p1 : p0;
    const double* ua = m == 0 ? snap0 : snap1;
    const double* ub = m == 0 ? snap1 : snap0;
    double* dst = m == 0 ? u0 : u1;
    const double ga = m == 0 ? g0 : g1, gb = m == 0 ? g1 : g0;
    const double ia = m == 0 ? i0 : i1, ib = m == 0 ? i1 : i0;
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t x = 0; x < nx; ++x) {
        double nrm[2], star[4];
        if (!gfm_source(pa, pb, nx, ny, x, y, h, nrm)) continue;
        const int64_t tx = x + isgn(nrm[0]), ty = y + isgn(nrm[1]);
        if (tx < 0 || tx >= nx || ty < 0 || ty >= ny) continue;
        gfm_star(ua, ub, pitch, nx, ny, pa, x, y, h, nrm, ga, gb, ia, ib, star);
        const int64_t t = ty * nx + tx;
        for (int c = 0; c < 4; ++c) dst[c * pitch + t] = st(star[c], f32);
        ++written;
      }
  }
  free(snap0);
  free(snap1);
  (void)n;
  return written;
}

int64_t flo_mm_gfm(int64_t nx, int64_t ny, int64_t pitch, double h, double g0, double g1,
                   double* u0, double* u1, const double* p0, const double* p1, int f32) {
  return flo_mm_gfm_mat(nx, ny, pitch, h, g0, 0.0, g1, 0.0, u0, u1, p0, p1, f32);
}

/* band of the extrapolation: dh <= phi <= 6 dh / sqrt(2), phi > 0
 * (ghost_fluid/ghost_fluid_extrapolator.hpp:104-127, band_width 3 + 3) */
static int in_band(double phi, double h) {
  const double upper = (6.0 * h) * 0.70710678118654752440;
  return phi > 0.0 && phi <= upper && phi >= h;
}

/* Ghost-cell extrapolation of one material (ghost_fluid_extrapolator.hpp
 * :54-202) as a Jacobi iteration.  Returns the number of sweeps. */
int flo_mm_extrapolate(int64_t nx, int64_t ny, int64_t pitch, double h, double* u,
                       const double* phi, int f32, int max_iters) {
  const int64_t n = nx * ny;
  double* cur = (double*)malloc(sizeof(double) * 4 * pitch);
  double* nxt = (double*)malloc(sizeof(double) * 4 * pitch);
  memcpy(cur, u, sizeof(double) * 4 * pitch);
  memcpy(nxt, u, sizeof(double) * 4 * pitch);
  int it = 0;
  for (; it < max_iters;) {
    double worst = 0.0;
    int nan_seen = 0;
#pragma omp parallel for schedule(static) reduction(max : worst) reduction(| : nan_seen)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t x = 0; x < nx; ++x) {
        const int64_t i = y * nx + x;
        if (!in_band(phi[i], h)) continue;
        const double fact = 0.5 / h;
        double g[2];
        g[0] = fact * (phi[idx(nx, ny, x + 1, y)] - phi[idx(nx, ny, x - 1, y)]);
        g[1] = fact * (phi[idx(nx, ny, x, y + 1)] - phi[idx(nx, ny, x, y - 1)]);
        const double s = sqrt(g[0] * g[0] + g[1] * g[1]);
        const double sign = (double)isgn(phi[i]);
        double nrm[2], l1 = 0.0;
        for (int d = 0; d < 2; ++d) {
          nrm[d] = -sign * (g[d] / s);
          l1 += fabs(nrm[d]);
        }
        const int use_n = l1 > 1e-2;
        double p[4] = {0.0, 0.0, 0.0, 0.0};
        for (int d = 0; d < 2; ++d) {
          const int64_t mx = d == 0 ? x - 1 : x, my = d == 0 ? y : y - 1;
          const int64_t px = d == 0 ? x + 1 : x, py = d == 0 ? y : y + 1;
          const int64_t qm = idx(nx, ny, mx, my), qp = idx(nx, ny, px, py);
          const int64_t q = phi[qm] < phi[qp] ? qm : qp;
          const double w = use_n ? fabs(nrm[d]) : 0.5;
          for (int c = 0; c < 4; ++c) p[c] += cur[c * pitch + q] * w;
        }
        if (use_n)
          for (int c = 0; c < 4; ++c) p[c] = p[c] / l1;
        int has_nan = 0;
        for (int c = 0; c < 4; ++c) has_nan |= isnan(p[c]);
        double err = 0.0;
        if (has_nan) {
          nan_seen = 1;
          for (int c = 0; c < 4; ++c) nxt[c * pitch + i] = cur[c * pitch + i];
        } else {
          for (int c = 0; c < 4; ++c) {
            const double v = st(p[c], f32);
            err += fabs(v - cur[c * pitch + i]);
            nxt[c * pitch + i] = v;
          }
        }
        if (err > worst) worst = err;
      }
    ++it;
    double* t = cur;
    cur = nxt;
    nxt = t;
    /* band cells of both buffers must agree before the next sweep reads */
    if (!(worst >= 1e-8) && !nan_seen) break;
  }
  for (int64_t i = 0; i < n; ++i)
    if (in_band(phi[i], h))
      for (int c = 0; c < 4; ++c) u[c * pitch + i] = cur[c * pitch + i];
  free(cur);
  free(nxt);
  return it;
}

/* set_states (state/cuda/state_initialization.cuh:72-86): cells inside the
 * level set (phi <= 0) take the conservative form of prim (rho, p, vx, vy). */
void flo_mm_set_states_mat(int64_t n, int64_t pitch, double* u, const double* phi,
                           const double* prim, double g, double pinf, int f32) {
  /* prim -> cons in the state's precision (state/state_impl.hpp:390-406) */
  double cons[4];
  if (f32) {
    const float r = (float)prim[0], p = (float)prim[1], vx = (float)prim[2], vy = (float)prim[3];
    const float gf = (float)g, pf = (float)pinf;
    float v2 = 0.0f;
    v2 += vx * vx;
    v2 += vy * vy;
    /* e from the eos (ideal_gas.hpp:59-63; stiff_fluid.hpp:76-80) */
    const float e = (p + gf * pf) / ((gf - 1.0f) * r);
    cons[0] = r;
    cons[1] = r * (0.5f * v2 + e);
    cons[2] = vx * r;
    cons[3] = vy * r;
  } else {
    const double r = prim[0], p = prim[1], vx = prim[2], vy = prim[3];
    double v2 = 0.0;
    v2 += vx * vx;
    v2 += vy * vy;
    const double e = (p + g * pinf) / ((g - 1.0) * r);
    cons[0] = r;
    cons[1] = r * (0.5 * v2 + e);
    cons[2] = vx * r;
    cons[3] = vy * r;
  }
  for (int64_t i = 0; i < n; ++i) {
    if (!(phi[i] <= 0.0 || phi[i] <= -0.0)) continue;
    for (int c = 0; c < 4; ++c) u[c * pitch + i] = cons[c];
  }
}

void flo_mm_set_states(int64_t n, int64_t pitch, double* u, const double* phi, const double* prim,
                       double g, int f32) {
  flo_mm_set_states_mat(n, pitch, u, phi, prim, g, 0.0, f32);
}

/* combine_into_first (material/cuda/combine_materials.cuh:39-66): cells
 * inside material 1 take its state in material 0's buffer. */
void flo_mm_combine(int64_t n, int64_t pitch, double* u0, const double* u1, const double* phi1) {
  for (int64_t i = 0; i < n; ++i)
    if (phi1[i] <= 0.0 || phi1[i] <= -0.0)
      for (int c = 0; c < 4; ++c) u0[c * pitch + i] = u1[c * pitch + i];
}
