// fl_walk3.cuh -- 3-D sweeps as register-streaming walks.
//
// Same arithmetic as sweep_kernel (fl_sweep.cuh) for D = 3: one dimensional
// sweep of SplitSolver::invoke (solver/split_solver.hpp:138-162) with
// MUSCL-Hancock, flattening (reconstruction/muscl_reconstructor.hpp:59-172),
// one Riemann solve per face, the conservative update and the optional fused
// max wavespeed.  The walk reuses the 2-D walker's mapping (fl_walk.cuh) on
// planes of the grid:
//   sweep x (S = 0): lanes along x (the stencil across lanes), rows along y,
//                    one launch plane per z;
//   sweep y (S = 1): lanes along x, rows along y (the stencil down the
//                    strip), one plane per z;
//   sweep z (S = 2): lanes along x, rows along z (the stencil down the
//                    strip), one plane per y.
// The flattening coefficient chi is the minimum over all three dimensions.
// The walk computes the x part across lanes and the row part down the strip.
// The third dimension's part (z for S = 0, 1; y for S = 2) comes from a plane
// that chi_dim_kernel fills in a first pass over the sweep's input.  At ghost
// positions of the walk (mirrored lanes or rows), that plane is read at the
// mirrored cell without the ghost's reflective flip.  That flip changes the
// momentum only by rounding ((-(m / rho)) * rho), so the value differs from
// the tile kernel's by rounding at most.
#pragma once

#include <cfloat>
#include <type_traits>

#include "fl_internal.cuh"
#include "fl_numerics.cuh"
#include "fl_sweep.cuh"
#include "fl_walk.cuh"

namespace fl {

#ifndef FL_WALK3_CTAS_F64
#define FL_WALK3_CTAS_F64 3
#endif
#ifndef FL_WALK3_CTAS_F32
#define FL_WALK3_CTAS_F32 4
#endif

template <typename T, int S>
struct Walk3Cfg {
  static constexpr int HX = (S == 0) ? 4 : 3;  // halo lanes on each side
  static constexpr int OWN = 32 - 2 * HX;      // owned columns per warp
  static constexpr int RY = FL_WALK_RY;        // rows per warp strip
  static constexpr int WARPS = FL_WALK_WARPS;  // warps per CTA (stacked strips)
  static constexpr int THREADS = 32 * WARPS;
  static constexpr int DR = (S == 2) ? 2 : 1;  // row dimension
  static constexpr int DT = (S == 2) ? 1 : 2;  // third dimension (chi from the plane)
  static constexpr int MIN_CTAS = sizeof(T) == 8 ? FL_WALK3_CTAS_F64 : FL_WALK3_CTAS_F32;
};

// One warp's strip of plane `pl` (index along DT): columns of group bx, rows
// [y0, y0 + ry) along DR.  xc: the DT part of chi for every cell (nullptr
// when flattening is off).
template <typename T, int S, int FLUX>
__device__ __forceinline__ void walk_strip_3d(const SweepParams& p, const T* __restrict__ xc,
                                              T dtdh, int64_t bx, int64_t y0, int ry, int64_t pl,
                                              double& ws_local, bool want_ws) {
  using W = Walk3Cfg<T, S>;
  constexpr int D = 3;
  constexpr int NC = 5;
  constexpr int DR = W::DR;
  constexpr int SW = (S == 0) ? 0 : 1;  // 0: stencil across lanes, 1: down the strip
  constexpr bool STIFF = (FLUX & kStiffEos) != 0;
  const T gamma = (T)p.gamma;
  const T pinf = (T)p.pinf;
  const T gm1 = gamma - T(1);
  const T adi = (gamma + T(1)) / (T(2) * gamma);
  const T hd = T(0.5) * dtdh;
  const bool muscl = !p.basic;
  const bool flatten = muscl && p.flatten;
  const T chi_init = (sizeof(T) == 8) ? (T)DBL_MAX : (T)FLT_MAX;

  const T* __restrict__ in = static_cast<const T*>(p.in);
  T* __restrict__ out = static_cast<T*>(p.out);
  const int64_t pitch = p.pitch;
  const int64_t n0 = p.n[0];
  const int64_t nr = p.n[DR];
  const int64_t rs = (DR == 1) ? n0 : n0 * p.n[1];       // cells between rows
  const int64_t base = pl * ((DR == 1) ? n0 * p.n[1] : n0);  // first cell of the plane
  const int lane = threadIdx.x & 31;

  const int64_t x = bx * W::OWN - W::HX + lane;
  bool fx = false;
  const int64_t gx = mirror_index(x, n0, fx);
  const bool flip_x = fx && (p.reflect & 1u);
  const bool flip_r_on = (p.reflect & (1u << DR)) != 0;
  const bool owned = lane >= W::HX && lane < 32 - W::HX && x < n0;

  if (y0 >= nr) return;
  const int64_t y_end = (y0 + ry < nr) ? y0 + ry : nr;
  // windows, index 4 = newest row k; row k - i at index 4 - i
  Cons<T, D> U[5];
  // FP64 re-derives the velocities the flattening needs from U (two more
  // reciprocals per row, 16 fewer live registers, fewer spills: +7%); FP32
  // keeps them in windows (re-deriving measured 1.5% slower there)
  constexpr bool kRederive = sizeof(T) == 8;
  T P[5], VX[5], VY[5];
  T CHY[3];  // row-direction chi bases of rows k-4, k-3, k-2
  Cons<T, D> er_prev, f_prev;
  const int64_t k_first = y0 - 3 - SW;
  const int64_t k_last = y_end + 2 + SW;
  Cons<T, D> pre;
  bool pre_fy = false;
  {
    const int64_t gy = mirror_index(k_first, nr, pre_fy);
#pragma unroll
    for (int c = 0; c < NC; ++c) pre.v[c] = __ldg(in + c * pitch + base + gy * rs + gx);
  }
  // the third dimension's chi part of evolve row k - 3, loaded one row ahead
  // like the state
  T ct_pre = T(0);
  if (flatten) {
    bool f = false;
    ct_pre = __ldg(xc + base + mirror_index(k_first - 3, nr, f) * rs + gx);
  }
  // the walk; its common form (FAST: no reflective end in the walk's two
  // dimensions, MUSCL with flattening and the van Leer limiter, the
  // wavespeed in the z sweep only) has the reflective flips and the
  // reconstruction, limiter and wavespeed tests compiled out
  auto walk = [&](auto fast) {
  constexpr bool FAST = decltype(fast)::value;
  constexpr bool RF = !FAST;
  const bool flat = FAST || flatten;
  const bool mus = FAST || muscl;
  for (int64_t k = k_first; k <= k_last; ++k) {
    const T ct = ct_pre;
    if (flat && k < k_last) {
      bool f = false;
      ct_pre = __ldg(xc + base + mirror_index(k - 2, nr, f) * rs + gx);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      U[i] = U[i + 1];
      P[i] = P[i + 1];
      if constexpr (!kRederive) {
        VX[i] = VX[i + 1];
        VY[i] = VY[i + 1];
      }
    }
    {
      Cons<T, D> u = pre;
      const bool fy = pre_fy;
      if (k < k_last) {
        const int64_t gy = mirror_index(k + 1, nr, pre_fy);
#pragma unroll
        for (int c = 0; c < NC; ++c) pre.v[c] = __ldg(in + c * pitch + base + gy * rs + gx);
      }
      if (RF && flip_x) u.v[2] = (-(u.v[2] / u.v[0])) * u.v[0];
      if (RF && fy && flip_r_on) u.v[2 + DR] = (-(u.v[2 + DR] / u.v[0])) * u.v[0];
      const Derived<T, D> q = derive(u, gm1);
      U[4] = u;
      P[4] = q.p;
      if constexpr (!kRederive) {
        VX[4] = q.v[0];
        VY[4] = q.v[DR];
      }
    }
    CHY[0] = CHY[1];
    CHY[1] = CHY[2];
    // re-derived: the same products derive() formed when the rows were loaded
    const T rinv1 = kRederive ? fl_rcp<T>(U[1].v[0]) : T(0);
    if (flat) {
      if constexpr (kRederive)
        CHY[2] = (T)chi_base<T>(P[3], P[1], P[4], P[0], U[1].v[2 + DR] * rinv1,
                                U[3].v[2 + DR] * fl_rcp<T>(U[3].v[0]));
      else
        CHY[2] = (T)chi_base<T>(P[3], P[1], P[4], P[0], VY[1], VY[3]);
    }
    const int64_t j = k - 3;  // evolve row
    const bool evolve_row = (SW == 0) ? (j >= y0) : (j >= y0 - 1);
    if (!evolve_row) continue;

    // ---- x flattening base of row j on this lane --------------------------
    const T pj = P[1], vxj = kRederive ? U[1].v[2] * rinv1 : VX[1];
    const T p_r1 = shfl_dn(pj, 1), p_l1 = shfl_up(pj, 1);
    const T p_r2 = shfl_dn(pj, 2), p_l2 = shfl_up(pj, 2);
    T chx = T(1);
    if (flat) chx = (T)chi_base<T>(p_r1, p_l1, p_r2, p_l2, shfl_up(vxj, 1), shfl_dn(vxj, 1));
    const T chx_r = shfl_dn(chx, 1), chx_l = shfl_up(chx, 1);

    const Cons<T, D>& u = U[1];
    Cons<T, D> er, el;
    if (!mus) {
      er = u;
      el = u;
    } else {
      T chi_v = T(1);
      if (flat) {
        const T dx = p_r1 - p_l1;
        const int sx = (T(0) < dx) - (dx < T(0));
        const T cx = std_min(chx, sx > 0 ? chx_r : (sx < 0 ? chx_l : chx));
        const T dy = P[2] - P[0];
        const int sy = (T(0) < dy) - (dy < T(0));
        const T cr = std_min(CHY[1], sy > 0 ? CHY[2] : (sy < 0 ? CHY[0] : CHY[1]));
        // minimum over dimensions 0, 1, 2 in order
        chi_v = (DR == 1) ? std_min(std_min(std_min(chi_init, cx), cr), ct)
                          : std_min(std_min(std_min(chi_init, cx), ct), cr);
      }
      const T ch = chi_v * T(0.5);
      Cons<T, D> a, b;
      // the limiter kind tested once per position, not per component
      auto slopes = [&](auto lim) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          T um, up;
          if (SW == 0) {
            um = shfl_up(u.v[c], 1);
            up = shfl_dn(u.v[c], 1);
          } else {
            um = U[0].v[c];
            up = U[2].v[c];
          }
          const T delta =
              ch * limited_slope<T>(decltype(lim)::value, u.v[c] - um, up - u.v[c]);
          a.v[c] = u.v[c] - delta;
          b.v[c] = u.v[c] + delta;
        }
      };
      if (!FAST && p.limiter == kSuperbee)
        slopes(std::integral_constant<int, kSuperbee>{});
      else
        slopes(std::integral_constant<int, kVanLeer>{});
      Cons<T, D> fa, fb;
      flux_q(a, derive(a, gm1), S, fa);
      flux_q(b, derive(b, gm1), S, fb);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const T df = fa.v[c] - fb.v[c];
        er.v[c] = b.v[c] + hd * df;
        el.v[c] = a.v[c] + hd * df;
      }
    }

    if (SW == 0) {
      Cons<T, D> ul, fx_l;
#pragma unroll
      for (int c = 0; c < NC; ++c) ul.v[c] = shfl_up(er.v[c], 1);
      riemann_q<FLUX>(ul, derive(ul, gm1), el, derive(el, gm1), 0, gamma, gm1, adi, dtdh, fx_l,
                      pinf);
      Cons<T, D> r;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const T fr = shfl_dn(fx_l.v[c], 1);
        r.v[c] = u.v[c] + dtdh * (fx_l.v[c] - fr);
      }
      if (owned && j < y_end) {
        const int64_t gi = base + j * rs + x;
#pragma unroll
        for (int c = 0; c < NC; ++c) out[c * pitch + gi] = r.v[c];
        if (FAST ? S == 2 : want_ws)
          ws_max(ws_local, (double)max_wavespeed_q<STIFF>(derive(r, gm1), gamma, pinf));
      }
    } else {
      if (j >= y0) {
        Cons<T, D> fxy;
        riemann_q<FLUX>(er_prev, derive(er_prev, gm1), el, derive(el, gm1), S, gamma, gm1, adi,
                        dtdh, fxy, pinf);
        if (j >= y0 + 1 && owned) {
          const Cons<T, D>& uo = U[0];
          Cons<T, D> r;
#pragma unroll
          for (int c = 0; c < NC; ++c) r.v[c] = uo.v[c] + dtdh * (f_prev.v[c] - fxy.v[c]);
          const int64_t gi = base + (j - 1) * rs + x;
#pragma unroll
          for (int c = 0; c < NC; ++c) out[c * pitch + gi] = r.v[c];
          if (FAST ? S == 2 : want_ws)
            ws_max(ws_local, (double)max_wavespeed_q<STIFF>(derive(r, gm1), gamma, pinf));
        }
        f_prev = fxy;
      }
      er_prev = er;
    }
  }
  };
  if ((p.reflect & (1u | (1u << DR))) == 0 && flatten && p.limiter == kVanLeer &&
      want_ws == (S == 2))
    walk(std::true_type{});
  else
    walk(std::false_type{});
}

template <typename T, int S, int FLUX>
__global__ void __launch_bounds__(Walk3Cfg<T, S>::THREADS, Walk3Cfg<T, S>::MIN_CTAS)
walk_kernel_3d(SweepParams p, const T* __restrict__ xc) {
  using W = Walk3Cfg<T, S>;
  if (p.walk_next != nullptr && blockIdx.x == 0 && threadIdx.x == 0)
    p.walk_next[1 - p.walk_slot] = 0u;
  if (p.ctrl != nullptr && *(volatile int*)&p.ctrl->done) return;
  const T dtdh = (p.ctrl != nullptr) ? (T)p.ctrl->dtdh : (T)p.dtdh;
  __shared__ double s_red[W::WARPS];
  const int warp = threadIdx.x >> 5;
  double ws_local = 0.0;
  const bool want_ws = (p.ws_accum != nullptr);
  if (p.walk_next == nullptr) {
    const int64_t y0 = ((int64_t)blockIdx.y * W::WARPS + warp) * W::RY;
    for (int64_t pl = blockIdx.z; pl < p.n[W::DT]; pl += gridDim.z)
      walk_strip_3d<T, S, FLUX>(p, xc, dtdh, (int64_t)blockIdx.x, y0, W::RY, pl, ws_local,
                                want_ws);
  } else {
    // strips taken dynamically, column group fastest, then the strip along
    // the row dimension, then the plane
    const int64_t ncol = (p.n[0] + W::OWN - 1) / W::OWN;
    const int64_t nrow = (p.n[W::DR] + W::RY - 1) / W::RY;
    const int64_t items = ncol * nrow * p.n[W::DT];
    unsigned int* next = &p.walk_next[p.walk_slot];
    for (;;) {
      unsigned int item = 0u;
      if ((threadIdx.x & 31) == 0) item = atomicAdd(next, 1u);
      item = __shfl_sync(0xffffffffu, item, 0);
      if ((int64_t)item >= items) break;
      const int64_t cr = (int64_t)item % (ncol * nrow);
      walk_strip_3d<T, S, FLUX>(p, xc, dtdh, cr % ncol, (cr / ncol) * W::RY, W::RY,
                                (int64_t)item / (ncol * nrow), ws_local, want_ws);
    }
  }
  if (want_ws) {
    const double m = cta_max<W::WARPS>(ws_local, s_red);
    if (threadIdx.x == 0) {
      atomicMax(p.ws_accum, (unsigned long long)__double_as_longlong(m));
      if (p.finalize && p.ctrl) {
        __threadfence();
        const unsigned int total = gridDim.x * gridDim.y * gridDim.z;
        const unsigned int prev = atomicAdd(&p.ctrl->arrive, 1u);
        if (prev == total - 1) {
          __threadfence();
          finalize_control(p.ctrl, true);
        }
      }
    }
  }
}

// The DT part of chi for every cell of the sweep's input: min(base(i),
// base(i + s)) along DT, s the sign of p(i + 1) - p(i - 1), with the bases of
// the flattening test (muscl_reconstructor.hpp:59-87).  Lanes along x (all
// own a column), a strip along DT per warp, one plane per index of the
// remaining dimension (DR of the walk).  Positions beyond the domain along
// DT are mirror ghosts with the reflective flip.
template <typename T, int S>
__global__ void __launch_bounds__(Walk3Cfg<T, S>::THREADS)
chi_dim_kernel(SweepParams p, T* __restrict__ xc) {
  using W = Walk3Cfg<T, S>;
  constexpr int D = 3;
  constexpr int NC = 5;
  constexpr int DT = W::DT, DR = W::DR;
  if (p.ctrl != nullptr && *(volatile int*)&p.ctrl->done) return;
  const T gm1 = (T)p.gamma - T(1);
  const T* __restrict__ in = static_cast<const T*>(p.in);
  const int64_t pitch = p.pitch;
  const int64_t n0 = p.n[0], nt = p.n[DT];
  const int64_t ts = (DT == 1) ? n0 : n0 * p.n[1];           // cells between DT rows
  const int64_t ps = (DR == 1) ? n0 : n0 * p.n[1];           // cells between planes
  const bool flip_t_on = (p.reflect & (1u << DT)) != 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t x = (int64_t)blockIdx.x * 32 + lane;
  const int64_t gx = x < n0 ? x : n0 - 1;
  const int64_t j0 = ((int64_t)blockIdx.y * W::WARPS + warp) * W::RY;
  if (j0 >= nt) return;
  const int64_t j_end = (j0 + W::RY < nt) ? j0 + W::RY : nt;
  for (int64_t pl = blockIdx.z; pl < p.n[DR]; pl += gridDim.z) {
    const int64_t base = pl * ps;
    T P[5], V[5], CH[3];
    for (int64_t k = j0 - 3; k <= j_end + 2; ++k) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        P[i] = P[i + 1];
        V[i] = V[i + 1];
      }
      bool ft = false;
      const int64_t gk = mirror_index(k, nt, ft);
      Cons<T, D> u;
#pragma unroll
      for (int c = 0; c < NC; ++c) u.v[c] = __ldg(in + c * pitch + base + gk * ts + gx);
      if (ft && flip_t_on) u.v[2 + DT] = (-(u.v[2 + DT] / u.v[0])) * u.v[0];
      const Derived<T, D> q = derive(u, gm1);
      P[4] = q.p;
      V[4] = q.v[DT];
      CH[0] = CH[1];
      CH[1] = CH[2];
      CH[2] = (T)chi_base<T>(P[3], P[1], P[4], P[0], V[1], V[3]);  // base of row k - 2
      const int64_t j = k - 3;
      if (j < j0 || x >= n0) continue;
      const T dt = P[2] - P[0];
      const int st = (T(0) < dt) - (dt < T(0));
      xc[base + j * ts + x] = std_min(CH[1], st > 0 ? CH[2] : (st < 0 ? CH[0] : CH[1]));
    }
  }
}

}  // namespace fl
