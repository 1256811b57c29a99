// fl_walk.cuh -- register-streaming 2-D sweep kernel ("walker").
//
// Same arithmetic as sweep_kernel (fl_sweep.cuh): one dimensional sweep of
// SplitSolver::invoke (solver/split_solver.hpp:138-162), MUSCL-Hancock with
// flattening (reconstruction/muscl_reconstructor.hpp:59-172), one Riemann
// solve per face, conservative update, optional fused max wavespeed.
//
// Mapping.  A warp owns 32 consecutive x columns and streams down a strip of
// RY rows.  Every lane loads its column's state once per row (coalesced),
// derives pressure and velocities once, and keeps sliding register windows
// of the rows it still needs.  Neighbours along x come from warp shuffles;
// neighbours along y come from the windows.  No shared-memory staging and no
// block barriers.
//   x sweep (S = 0): the stencil runs across lanes.  Lanes 0..31 hold columns
//     x0-4 .. x0+27; flattening along x is valid on lanes 2..29, evolved faces
//     on lanes 3..28, Riemann faces on lanes 4..28, updates on lanes 4..27
//     (24 owned columns).  The y flattening bases come from the row windows.
//   y sweep (S = 1): the stencil runs down the strip.  Lanes hold columns
//     x0-3 .. x0+28; the x flattening needs lanes +-3, so lanes 3..28 (26)
//     are owned.  Evolved faces, Riemann solves and updates follow the walk.
// Rows and columns outside the domain are mirror ghosts, as in stage A of
// sweep_kernel.
#pragma once

#include <cfloat>
#include <type_traits>

#include "fl_internal.cuh"
#include "fl_numerics.cuh"
#include "fl_sweep.cuh"

#ifndef FL_WALK_RY
#define FL_WALK_RY 64
#endif
#ifndef FL_WALK_WARPS
#define FL_WALK_WARPS 4
#endif
#ifndef FL_WALK_CTAS_F64_X
#define FL_WALK_CTAS_F64_X 4
#endif
#ifndef FL_WALK_CTAS_F64_Y
#define FL_WALK_CTAS_F64_Y 3
#endif
#ifndef FL_WALK_CTAS_F32_X
#define FL_WALK_CTAS_F32_X 6
#endif
#ifndef FL_WALK_CTAS_F32_Y
#define FL_WALK_CTAS_F32_Y 5
#endif

namespace fl {

template <typename T, int S>
struct WalkCfg {
  static constexpr int HX = (S == 0) ? 4 : 3;  // halo lanes on each side
  static constexpr int OWN = 32 - 2 * HX;      // owned columns per warp
  static constexpr int RY = FL_WALK_RY;        // rows per warp strip
  static constexpr int WARPS = FL_WALK_WARPS;  // warps per CTA (stacked strips)
  static constexpr int THREADS = 32 * WARPS;
  // resident CTAs per SM the register allocation is held to: 65536 /
  // (128 threads * MIN_CTAS) registers per thread.  Measured choice; the
  // FL_WALK_CTAS_* macros override it for tuning builds.
  static constexpr int MIN_CTAS = sizeof(T) == 8 ? (S == 0 ? FL_WALK_CTAS_F64_X : FL_WALK_CTAS_F64_Y)
                                                 : (S == 0 ? FL_WALK_CTAS_F32_X : FL_WALK_CTAS_F32_Y);
};

template <typename T>
__device__ __forceinline__ T shfl_up(T v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
template <typename T>
__device__ __forceinline__ T shfl_dn(T v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

// One warp's strip: columns of column group bx, rows [y0, y0 + ry).  Stores
// the updated rows and folds the wavespeed of each stored cell into
// ws_local.  p.in / p.out / p.n / p.pitch describe the grid; dtdh is taken
// from the caller.
template <typename T, int S, int FLUX>
__device__ __forceinline__ void walk_strip_2d(const SweepParams& p, T dtdh, int64_t bx,
                                              int64_t y0, int ry, double& ws_local,
                                              bool want_ws) {
  using W = WalkCfg<T, S>;
  constexpr int D = 2;
  constexpr int NC = 4;
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
  const int64_t n0 = p.n[0], n1 = p.n[1];
  const int lane = threadIdx.x & 31;

  const int64_t x = bx * W::OWN - W::HX + lane;
  bool fx = false;
  const int64_t gx = mirror_index(x, n0, fx);
  const bool flip_x = fx && (p.reflect & 1u);
  const bool flip_y_on = (p.reflect & 2u) != 0;
  const bool owned = lane >= W::HX && lane < 32 - W::HX && x < n0;

  if (y0 < n1) {
    const int64_t y_end = (y0 + ry < n1) ? y0 + ry : n1;
    // windows, index 4 = newest row k; row k - i at index 4 - i
    Cons<T, D> U[5];
    T P[5], VX[5], VY[5];
    T CHY[3];  // chi_y of rows k-4, k-3, k-2
    Cons<T, D> er_prev, f_prev;
    const int64_t k_first = y0 - 3 - (S == 1 ? 1 : 0);
    const int64_t k_last = y_end + (S == 1 ? 3 : 2);
    // row k + 1 is loaded while row k is processed (global-load latency
    // overlaps the arithmetic)
    Cons<T, D> pre;
    bool pre_fy = false;
    {
      const int64_t gy = mirror_index(k_first, n1, pre_fy);
#pragma unroll
      for (int c = 0; c < NC; ++c) pre.v[c] = __ldg(in + c * pitch + gy * n0 + gx);
    }
    // the walk; its common form (FAST: no reflective end in x or y, MUSCL
    // with flattening and the van Leer limiter, the wavespeed in the y sweep
    // only) has the reflective flips and the reconstruction, limiter and
    // wavespeed tests compiled out.  A slab's row window for the wavespeed
    // stays a runtime test, so that slabs take the same code as the
    // undivided grid and match it bit for bit.
    auto walk = [&](auto fast) {
    constexpr bool FAST = decltype(fast)::value;
    const bool flat = FAST || flatten;
    const bool mus = FAST || muscl;
    for (int64_t k = k_first; k <= k_last; ++k) {
      // ---- shift windows and take row k ----------------------------------
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        U[i] = U[i + 1];
        P[i] = P[i + 1];
        VX[i] = VX[i + 1];
        VY[i] = VY[i + 1];
      }
      {
        Cons<T, D> u = pre;
        const bool fy = pre_fy;
        if (k < k_last) {
          const int64_t gy = mirror_index(k + 1, n1, pre_fy);
#pragma unroll
          for (int c = 0; c < NC; ++c) pre.v[c] = __ldg(in + c * pitch + gy * n0 + gx);
        }
        if (!FAST && flip_x) u.v[2] = (-(u.v[2] / u.v[0])) * u.v[0];
        if (!FAST && fy && flip_y_on) u.v[3] = (-(u.v[3] / u.v[0])) * u.v[0];
        const Derived<T, D> q = derive(u, gm1);
        U[4] = u;
        P[4] = q.p;
        VX[4] = q.v[0];
        VY[4] = q.v[1];
      }
      // ---- y flattening base of row k - 2 (needs rows k-4..k) -----------
      CHY[0] = CHY[1];
      CHY[1] = CHY[2];
      if (flat) CHY[2] = (T)chi_base<T>(P[3], P[1], P[4], P[0], VY[1], VY[3]);
      const int64_t j = k - 3;  // evolve row
      const bool evolve_row = (S == 0) ? (j >= y0) : (j >= y0 - 1);
      if (!evolve_row) continue;

      // ---- x flattening base of row j on this lane ----------------------
      const T pj = P[1], vxj = VX[1];
      const T p_r1 = shfl_dn(pj, 1), p_l1 = shfl_up(pj, 1);
      const T p_r2 = shfl_dn(pj, 2), p_l2 = shfl_up(pj, 2);
      T chx = T(1);
      if (flat) chx = (T)chi_base<T>(p_r1, p_l1, p_r2, p_l2, shfl_up(vxj, 1), shfl_dn(vxj, 1));
      const T chx_r = shfl_dn(chx, 1), chx_l = shfl_up(chx, 1);

      // ---- evolved face states of (lane, j) -------------------------------
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
          const T cy = std_min(CHY[1], sy > 0 ? CHY[2] : (sy < 0 ? CHY[0] : CHY[1]));
          chi_v = std_min(std_min(chi_init, cx), cy);
        }
        const T ch = chi_v * T(0.5);
        Cons<T, D> a, b;
        // the limiter kind tested once per position, not per component
        auto slopes = [&](auto lim) {
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            T um, up;
            if (S == 0) {
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

      if (S == 0) {
        // face between lanes (lane-1, lane), then update of (lane, j)
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
          const int64_t gi = j * n0 + x;
#pragma unroll
          for (int c = 0; c < NC; ++c) out[c * pitch + gi] = r.v[c];
          if ((FAST ? S == 1 : want_ws) && ws_row_counts(p, j))
            ws_max(ws_local, (double)max_wavespeed_q<STIFF>(derive(r, gm1), gamma, pinf));
        }
      } else {
        if (j >= y0) {
          // face (j-1, j) along y, then update of row j - 1
          Cons<T, D> fxy;
          riemann_q<FLUX>(er_prev, derive(er_prev, gm1), el, derive(el, gm1), 1, gamma, gm1,
                          adi, dtdh, fxy, pinf);
          if (j >= y0 + 1 && owned) {
            const Cons<T, D>& uo = U[0];
            Cons<T, D> r;
#pragma unroll
            for (int c = 0; c < NC; ++c) r.v[c] = uo.v[c] + dtdh * (f_prev.v[c] - fxy.v[c]);
            const int64_t gi = (j - 1) * n0 + x;
#pragma unroll
            for (int c = 0; c < NC; ++c) out[c * pitch + gi] = r.v[c];
            if ((FAST ? S == 1 : want_ws) && ws_row_counts(p, j - 1))
              ws_max(ws_local, (double)max_wavespeed_q<STIFF>(derive(r, gm1), gamma, pinf));
          }
          f_prev = fxy;
        }
        er_prev = er;
      }
    }
    };
    if ((p.reflect & 3u) == 0 && flatten && p.limiter == kVanLeer && want_ws == (S == 1))
      walk(std::true_type{});
    else
      walk(std::false_type{});
  }
}

// Warp max, then CTA max of the per-lane wavespeeds (all threads call).
template <int WARPS>
__device__ __forceinline__ double cta_max(double v, double* s_red) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) ws_max(v, __shfl_xor_sync(0xffffffffu, v, off));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = s_red[0];
#pragma unroll
  for (int w = 1; w < WARPS; ++w) ws_max(m, s_red[w]);
  return m;
}

// Strips are scheduled statically (blockIdx.x the column group, blockIdx.y
// and the warp the strip) or, given strip counters, dynamically: a grid of
// resident CTAs whose warps take strips, column group fastest, from
// walk_next[walk_slot] until none is left, so that no SM idles while a last
// partial wave of CTAs runs.  The sweep clears the other counter, which the
// next sweep of the stream uses.
template <typename T, int S, int FLUX>
__global__ void __launch_bounds__(WalkCfg<T, S>::THREADS, WalkCfg<T, S>::MIN_CTAS)
walk_kernel_2d(SweepParams p) {
  using W = WalkCfg<T, S>;
  // cleared before the early exit too, so that a finished run keeps both
  // counters ready for the next sweeps on the same control block
  if (p.walk_next != nullptr && blockIdx.x == 0 && threadIdx.x == 0)
    p.walk_next[1 - p.walk_slot] = 0u;
  if (p.ctrl != nullptr && *(volatile int*)&p.ctrl->done) return;
  const T dtdh = (p.ctrl != nullptr) ? (T)p.ctrl->dtdh : (T)p.dtdh;
  __shared__ double s_red[W::WARPS];
  const int warp = threadIdx.x >> 5;
  double ws_local = 0.0;
  const bool want_ws = (p.ws_accum != nullptr);
  // the rows to compute: [r_lo, r_hi)
  const bool win = p.row_hi > p.row_lo;
  const int64_t r_lo = win ? p.row_lo : 0, r_hi = win ? p.row_hi : p.n[1];
  if (p.walk_next == nullptr) {
    const int64_t y0 = r_lo + ((int64_t)blockIdx.y * W::WARPS + warp) * W::RY;
    if (y0 < r_hi)
      walk_strip_2d<T, S, FLUX>(p, dtdh, (int64_t)blockIdx.x, y0,
                                (int)(r_hi - y0 < W::RY ? r_hi - y0 : W::RY), ws_local, want_ws);
  } else {
    const int ry = (p.walk_ry > 0) ? p.walk_ry : W::RY;
    const int64_t ncol = (p.n[0] + W::OWN - 1) / W::OWN;
    const int64_t items = ncol * ((r_hi - r_lo + ry - 1) / ry);
    unsigned int* next = &p.walk_next[p.walk_slot];
    for (;;) {
      unsigned int item = 0u;
      if ((threadIdx.x & 31) == 0) item = atomicAdd(next, 1u);
      item = __shfl_sync(0xffffffffu, item, 0);
      if ((int64_t)item >= items) break;
      const int64_t y0 = r_lo + ((int64_t)item / ncol) * ry;
      walk_strip_2d<T, S, FLUX>(p, dtdh, (int64_t)item % ncol, y0,
                                (int)(r_hi - y0 < ry ? r_hi - y0 : ry), ws_local, want_ws);
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

}  // namespace fl
