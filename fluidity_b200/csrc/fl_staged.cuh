// fl_staged.cuh -- TMA-staged 2-D sweep kernel.
//
// Same arithmetic as walk_kernel_2d (fl_walk.cuh) and sweep_kernel
// (fl_sweep.cuh): one dimensional sweep of SplitSolver::invoke
// (solver/split_solver.hpp:138-162), MUSCL-Hancock with flattening
// (reconstruction/muscl_reconstructor.hpp:59-172), one Riemann solve per face,
// conservative update, optional fused max wavespeed.
//
// Mapping.  Both sweeps walk ALONG the sweep dimension; the 32 lanes of a
// warp lie ACROSS it, one cell each, and every lane's cell is an output cell.
//   y sweep (S = 1): lanes are 32 consecutive columns, the walk steps row by
//     row.  A stage is one row of 40 columns (the lanes' 32 plus 4 on each
//     side) of all four component planes, one TMA box.
//   x sweep (S = 0): lanes are 32 consecutive rows, the walk steps column by
//     column (a transposed walk).  A stage is 16 bytes of columns (2 in FP64,
//     4 in FP32) of 38 rows (the lanes' 32 plus 3 on each side), one TMA box.
//     Updated cells collect in a shared output tile of the same shape that a
//     TMA store writes back when its columns are complete.
// Each warp owns a ring of stages in shared memory, each with an mbarrier;
// lane 0 keeps the ring filled ahead of the walk.  The stencil along the
// sweep reads the ring (own lane only, no exchange).  The stencil across the
// sweep -- the flattening coefficient's pressure and velocity reach of 3 --
// goes through two small per-warp exchange rows (pressure and velocity);
// the 6 across-halo cells (3 on each side of the warp) are derived in one
// extra pass of all lanes, of which lanes 0-5 keep theirs (no divergent
// region), and each lane computes the flattening base of the neighbour its
// pressure rises towards itself, from those rows.
// The reference's halo of 4 along the sweep costs 7 extra derivations per
// strip of 64 and one extra evolve and Riemann solve at its start.
//
// Rows and columns outside the domain are mirror ghosts (ghost[-1-g] =
// cell[g], solver/boundary_loader.hpp:175-199), with the normal momentum
// negated as (-(m/rho))*rho at reflective ends.  Along the sweep the TMA
// boxes are taken at the mirrored coordinates; across it the lanes read the
// mirrored cell of their box.
#pragma once

#include <cfloat>
#include <type_traits>

#include "fl_internal.cuh"
#include "fl_numerics.cuh"
#include "fl_sweep.cuh"
#include "fl_tma.cuh"

#ifndef FL_STAGED_RY
#define FL_STAGED_RY 64
#endif


namespace fl {

// GEO = 1: the walk runs along the slow dimension of the input's layout and a
// stage is one row of 40 cells along its fast dimension (the lanes' 32 plus 4
// on each side).  GEO = 0: the walk runs along the fast dimension and a stage
// is 16 bytes of it (2 cells in FP64, 4 in FP32) over 38 rows (the lanes' 32
// plus 3 on each side).  TOUT: updated cells collect in a shared tile of 16
// bytes along the walk by 32 lanes, written back by a TMA store whose tensor
// map has the walk dimension fastest; otherwise each lane stores its cell,
// in the input's layout.
template <typename T, int GEO, bool TOUT>
struct StagedCfg {
  static constexpr int NC = 4;
  static constexpr int CB = 16 / (int)sizeof(T);  // cells per 16 bytes
  static constexpr int PPS = GEO ? 1 : CB;         // walk positions per stage
  static constexpr int BW = GEO ? 40 : 38;         // across extent of a box
  static constexpr int AOFF = GEO ? 4 : 3;         // box index of lane 0's cell
  static constexpr int STAGE = NC * BW * PPS;      // elements per stage
  static constexpr uint32_t STAGE_BYTES = STAGE * sizeof(T);
  // stages the walk reads at once (positions k-4 .. k), plus prefetch
  static constexpr int LIVE = GEO ? 5 : (CB == 2 ? 3 : 2);
  // FP64 rows with a tiled output: 7 stages, so that four CTAs stay resident
  static constexpr int NS = GEO ? ((TOUT && sizeof(T) == 8) ? 7 : 8) : (sizeof(T) == 8 ? 5 : 4);
  static constexpr int WARPS = (!GEO && sizeof(T) == 8) ? 2 : 4;
  static constexpr int THREADS = 32 * WARPS;
  static constexpr int RY = FL_STAGED_RY;
  // A tiled output collects 32 bytes along the walk per lane (one DRAM
  // sector: 4 cells in FP64, 8 in FP32) before its TMA store; 16-byte
  // stores left half-written sectors that L2 filled from DRAM, 55% more
  // reads than the sweep's own.
  static constexpr int OPS = 32 / (int)sizeof(T);      // walk positions per store
  static constexpr int OUT = TOUT ? NC * 32 * OPS : 0;  // output tile elements
  // output tiles: one for the row geometry (a second would cost a resident
  // CTA per SM in FP64), two otherwise
  static constexpr int NOUT = TOUT ? (GEO ? 1 : 2) : 0;
  static constexpr size_t RING_BYTES = (size_t)NS * STAGE_BYTES;
  static constexpr size_t OUT_BYTES = (size_t)NOUT * OUT * sizeof(T);
  static constexpr size_t X_BYTES = 2 * 40 * sizeof(T);
  static constexpr size_t BAR_BYTES = NS * 8;
  static constexpr size_t WARP_BYTES =
      (RING_BYTES + OUT_BYTES + X_BYTES + BAR_BYTES + 127) / 128 * 128;
  // plus 128 bytes to align the first warp's region (TMA boxes start on
  // 128-byte boundaries: every part size above is a multiple of 128)
  static constexpr size_t SMEM = WARPS * WARP_BYTES + 128;
  static_assert(STAGE_BYTES % 128 == 0 && (OUT * sizeof(T)) % 128 == 0, "128-byte boxes");
  // registers held to this many resident CTAs per SM
  // (FP32 rows: 5, as many as their shared memory allows; 6 held the
  // registers to 80 for no resident CTA more, 1.3% slower)
  static constexpr int MIN_CTAS = (sizeof(T) == 8) ? (GEO ? 4 : 7) : (GEO ? 5 : 4);
  static_assert(NS >= LIVE + 1, "the ring needs room to prefetch");
};

// Per-warp view of the shared-memory region.
template <typename T, int GEO, bool TOUT>
struct StagedSmem {
  using C = StagedCfg<T, GEO, TOUT>;
  T* ring;
  T* out;
  T* xp;   // pressure across the warp, by box index
  T* xv;   // velocity across the sweep, by box index
  uint64_t* bars;
  __device__ __forceinline__ explicit StagedSmem(unsigned char* base) {
    ring = reinterpret_cast<T*>(base);
    out = reinterpret_cast<T*>(base + C::RING_BYTES);
    xp = reinterpret_cast<T*>(base + C::RING_BYTES + C::OUT_BYTES);
    xv = xp + 40;
    bars = reinterpret_cast<uint64_t*>(base + C::RING_BYTES + C::OUT_BYTES + C::X_BYTES);
  }
};

// Box coordinate along the sweep of stage t's first position p0, and whether
// the stage is a mirror image (its positions map to columns in reverse).
template <typename T, int GEO, bool TOUT>
__device__ __forceinline__ int stage_along(int p0, int nl, bool& reversed) {
  using C = StagedCfg<T, GEO, TOUT>;
  reversed = false;
  if (GEO) {  // one row per stage: the mirrored row itself
    bool f;
    return (int)mirror_index((int64_t)p0, (int64_t)nl, f);
  }
  if (p0 < 0) {
    reversed = true;
    return -p0 - C::CB;
  }
  if (p0 >= nl) {
    reversed = true;
    return 2 * nl - p0 - C::CB;
  }
  return p0;
}

template <typename T, int GEO, bool TOUT>
__device__ __forceinline__ void stage_issue(const StagedSmem<T, GEO, TOUT>& sm,
                                            const CUtensorMap* tin, int slot, int p0, int nl,
                                            int a0) {
  using C = StagedCfg<T, GEO, TOUT>;
  bool rev;
  const int al = stage_along<T, GEO, TOUT>(p0, nl, rev);
  T* dst = sm.ring + (size_t)slot * C::STAGE;
  mbar_expect_tx(&sm.bars[slot], C::STAGE_BYTES);
  if (GEO)
    tma_load_3d(dst, tin, &sm.bars[slot], a0 - C::AOFF, al, 0);
  else
    tma_load_3d(dst, tin, &sm.bars[slot], al, a0 - C::AOFF, 0);
}

// One warp's strip: across block `ab` (cells a0 = 32 ab .. a0 + 31 across
// the sweep), positions [s0, s0 + ry) along it.  Stores the updated cells and
// folds the wavespeed of each stored cell into ws_local.  gstage counts the
// stages this warp has issued before (ring slot and barrier phase).  Grid
// extents are below 2^30 (checked by the launcher), so positions are ints.
template <typename T, int S, int FLUX, int GEO, bool TOUT>
__device__ __forceinline__ void staged_strip(const SweepParams& p, const CUtensorMap* tin,
                                             const CUtensorMap* tout,
                                             const StagedSmem<T, GEO, TOUT>& sm, T dtdh, T dhdt,
                                             int ab,
                                             int s0, int ry, double& ws_local, bool want_ws,
                                             uint32_t& gstage, int& fault) {
  using Cf = StagedCfg<T, GEO, TOUT>;
  constexpr int D = 2;
  constexpr int NC = 4;
  constexpr int PPS = Cf::PPS;
  constexpr int NS = Cf::NS;
  constexpr bool STIFF = (FLUX & kStiffEos) != 0;
  const T gamma = (T)p.gamma;
  const T pinf = (T)p.pinf;
  const T gm1 = gamma - T(1);
  const T adi = (gamma + T(1)) / (T(2) * gamma);
  const T hd = T(0.5) * dtdh;
  const bool muscl = !p.basic;
  const bool flatten = muscl && p.flatten;
  const T chi_init = (sizeof(T) == 8) ? (T)DBL_MAX : (T)FLT_MAX;
  const int lane = threadIdx.x & 31;

  const int nl = (int)p.n[S];      // cells along the sweep
  const int na = (int)p.n[1 - S];  // cells across it
  const int a0 = ab * 32;
  const bool flip_l_on = (p.reflect & (1u << S)) != 0;
  const bool flip_a_on = (p.reflect & (1u << (1 - S))) != 0;

  // this lane's cell across the sweep, and the box index it reads
  const int ai = a0 + lane;
  bool fa = false;
  const int gai = (int)mirror_index(ai, na, fa);
  int aoff = gai - (a0 - Cf::AOFF);
  aoff = aoff < 0 ? 0 : (aoff >= Cf::BW ? Cf::BW - 1 : aoff);
  const bool flip_a = fa && flip_a_on;
  const bool owned = ai < na;
  const int own = Cf::AOFF + lane;  // exchange index of this lane's cell
  // lanes 0-5: one across-halo cell each (3 on each side of the warp)
  const int hai = (lane < 3) ? a0 - 3 + lane : a0 + 29 + lane;
  bool fh = false;
  const int ghai = (int)mirror_index(hai, na, fh);
  int hoff = ghai - (a0 - Cf::AOFF);
  hoff = hoff < 0 ? 0 : (hoff >= Cf::BW ? Cf::BW - 1 : hoff);
  const bool flip_h = fh && flip_a_on;
  const int hx = (lane < 3) ? Cf::AOFF - 3 + lane : Cf::AOFF + 29 + lane;

  const int s_end = (s0 + ry < nl) ? s0 + ry : nl;
  const int k_first = s0 - 4;
  const int k_last = s_end + 3;
  const int nr = k_last - k_first + 1;
  const int nst = (nr + PPS - 1) / PPS;  // stages of this strip
  const uint32_t g0 = gstage;

  // fill the ring
  __syncwarp();
  int issued = (nst < NS) ? nst : NS;  // stages issued so far (warp-uniform)
  int waiting = 0;                     // the stage the walk waits for next
  if (lane == 0) {
    fence_proxy_async_smem();
    for (int t = 0; t < issued; ++t)
      stage_issue<T, GEO, TOUT>(sm, tin, (int)((g0 + t) % NS), k_first + t * PPS, nl, a0);
  }

  // the stage holding walk offset r, and r's column within it.  With one
  // position per stage the walk's own stage slot advances by one per row
  // (slot_r below), and the rows behind it are slots back from it.
  int slot_r = (int)(g0 % NS);   // ring slot of the stage of walk offset r
  auto stage_of = [&](int r, int& q) -> const T* {
    const int t = r / PPS;
    q = r - t * PPS;
    if (!GEO) {
      bool rev;
      (void)stage_along<T, GEO, TOUT>(k_first + t * PPS, nl, rev);
      if (rev) q = PPS - 1 - q;
    }
    return sm.ring + (size_t)((g0 + t) % NS) * Cf::STAGE;
  };
  auto stage_back = [&](int r, int back, int& q) -> const T* {
    if (GEO) {
      q = 0;
      int sl = slot_r - back;
      if (sl < 0) sl += NS;
      return sm.ring + (size_t)sl * Cf::STAGE;
    }
    return stage_of(r - back, q);
  };
  // the cell at box index a of a stage, with the ghost flips: gl along the
  // sweep (a mirrored position), fx across it (a mirrored lane)
  auto load = [&](const T* st, int q, int a, bool gl, bool fx) {
    Cons<T, D> u;
#pragma unroll
    for (int c = 0; c < NC; ++c)
      u.v[c] = GEO ? st[c * Cf::BW + a] : st[(c * Cf::BW + a) * Cf::CB + q];
    if (gl) u.v[2 + S] = (-(u.v[2 + S] / u.v[0])) * u.v[0];
    if (fx) u.v[3 - S] = (-(u.v[3 - S] / u.v[0])) * u.v[0];
    return u;
  };
  auto ghost_l = [&](int k) { return flip_l_on && (unsigned)k >= (unsigned)nl; };

  // windows along the sweep: index 4 = newest position k, k - i at 4 - i
  T P[5], VL[5];
  T CHA[3];   // flattening base along the sweep at k-4, k-3, k-2
  T CX[4];    // across part of chi at k-3 .. k
  Cons<T, D> er_prev, f_prev;
#pragma unroll
  for (int i = 0; i < 5; ++i) { P[i] = T(0); VL[i] = T(0); }
#pragma unroll
  for (int i = 0; i < 3; ++i) CHA[i] = T(1);
#pragma unroll
  for (int i = 0; i < 4; ++i) CX[i] = T(1);

  T* const out = static_cast<T*>(p.out);
  const int64_t pitch = p.pitch;

  // the walk, with the limiter kind fixed for the whole strip.  Its common
  // form (FAST: no end of either dimension reflects, MUSCL with flattening,
  // the wavespeed folded in the y sweep only and over every row) has the
  // reflective flips and the reconstruction and wavespeed tests compiled
  // out.
  auto walk = [&](auto lim, auto fast) {
  constexpr int LIM = decltype(lim)::value;
  constexpr bool FAST = decltype(fast)::value;
  constexpr bool RF = !FAST;
  const bool flat = FAST || flatten;
  const bool mus = FAST || muscl;
  for (int r = 0; r < nr; ++r) {
    const int k = k_first + r;
    // ---- ring: recycle the stage the walk no longer reads, wait for k ----
    if (r >= 5 && (r - 5) % PPS == PPS - 1) {
      const int td = (r - 5) / PPS;
      if (td + NS < nst) {
        __syncwarp();
        if (lane == 0) {
          fence_proxy_async_smem();
          stage_issue<T, GEO, TOUT>(sm, tin, (int)((g0 + td) % NS), k_first + (td + NS) * PPS,
                                    nl, a0);
        }
        ++issued;
      }
    }
    if (r % PPS == 0) {
      waiting = r / PPS;
      const uint32_t g = g0 + waiting;
      if (!mbar_wait_bounded(&sm.bars[g % NS], (g / NS) & 1u)) {
        fault = 1;
        break;
      }
    }
    // ---- derive position k: own cell, then the across halo ---------------
    if (GEO && r > 0) slot_r = (slot_r + 1 == NS) ? 0 : slot_r + 1;
    int qk;
    const T* stk = stage_back(r, 0, qk);
    const bool glk = RF && ghost_l(k);
    const Cons<T, D> u = load(stk, qk, aoff, glk, RF && flip_a);
    const Derived<T, D> q = derive(u, gm1);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      P[i] = P[i + 1];
      VL[i] = VL[i + 1];
    }
    P[4] = q.p;
    VL[4] = q.v[S];
    T cx = T(1);
    if (flat) {
      sm.xp[own] = q.p;
      sm.xv[own] = q.v[1 - S];
      {
        // every lane derives a halo cell (lanes 0-5 keep theirs): no
        // divergent region between the own and the halo derivations
        const Cons<T, D> uh = load(stk, qk, hoff, glk, RF && flip_h);
        const Derived<T, D> qh = derive(uh, gm1);
        if (lane < 6) {
          sm.xp[hx] = qh.p;
          sm.xv[hx] = qh.v[1 - S];
        }
      }
      __syncwarp();
      const T pr1 = sm.xp[own + 1], pl1 = sm.xp[own - 1];
      const T pr2 = sm.xp[own + 2], pl2 = sm.xp[own - 2];
      const T vr1 = sm.xv[own + 1], vl1 = sm.xv[own - 1];
      const T dx = pr1 - pl1;
      const int sx = (T(0) < dx) - (dx < T(0));
      // the two values the neighbour the pressure rises towards needs beyond
      // this lane's own reach
      const T p3 = sm.xp[own + 3 * sx], v2 = sm.xv[own + 2 * sx];
      __syncwarp();  // every lane has read the exchange rows
      const T chx = (T)chi_base<T>(pr1, pl1, pr2, pl2, vl1, vr1);
      const T qp = q.p, qv = q.v[1 - S];
      const bool upw = sx > 0;
      const T cn = (T)chi_base<T>(upw ? pr2 : qp, upw ? qp : pl2, upw ? p3 : pr1, upw ? pl1 : p3,
                                  upw ? qv : v2, upw ? v2 : qv);
      cx = std_min(chx, sx != 0 ? cn : chx);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) CX[i] = CX[i + 1];
    CX[3] = cx;
    // ---- flattening base along the sweep of position k - 2 ---------------
    CHA[0] = CHA[1];
    CHA[1] = CHA[2];
    if (flat) CHA[2] = (T)chi_base<T>(P[3], P[1], P[4], P[0], VL[1], VL[3]);

    const int j = k - 3;  // evolve position
    if (j < s0 - 1) continue;
    // ---- evolved face states of (lane, j) ----------------------------------
    int qj, qm;
    const T* stj = stage_back(r, 3, qj);
    const T* stm = stage_back(r, 4, qm);
    const Cons<T, D> uj = load(stj, qj, aoff, RF && ghost_l(j), RF && flip_a);
    const Cons<T, D> um = load(stm, qm, aoff, RF && ghost_l(j - 1), RF && flip_a);  // position j - 1
    Cons<T, D> er, el;
    if (!mus) {
      er = uj;
      el = uj;
    } else {
      int qp;
      const T* stp = stage_back(r, 2, qp);
      const Cons<T, D> up = load(stp, qp, aoff, RF && ghost_l(j + 1), RF && flip_a);
      T chi_v = T(1);
      if (flat) {
        const T dl = P[2] - P[0];
        const int sl = (T(0) < dl) - (dl < T(0));
        const T cl = std_min(CHA[1], sl > 0 ? CHA[2] : (sl < 0 ? CHA[0] : CHA[1]));
        chi_v = std_min(std_min(chi_init, CX[0]), cl);
      }
      const T ch = chi_v * T(0.5);
      Cons<T, D> a, b;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const T delta = ch * limited_slope<T>(LIM, uj.v[c] - um.v[c], up.v[c] - uj.v[c]);
        a.v[c] = uj.v[c] - delta;
        b.v[c] = uj.v[c] + delta;
      }
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
    if (j >= s0) {
      // face (j-1, j), then the update of position j - 1
      Cons<T, D> fj;
      riemann_qh<FLUX>(er_prev, derive(er_prev, gm1), el, derive(el, gm1), S, gamma, gm1, adi,
                       dtdh, dhdt, fj, pinf);
      if (j >= s0 + 1) {
        Cons<T, D> res;
#pragma unroll
        for (int c = 0; c < NC; ++c) res.v[c] = um.v[c] + dtdh * (f_prev.v[c] - fj.v[c]);
        const int jo = j - 1;  // the updated position
        if (!TOUT) {
          if (owned) {
            T* o = out + (int64_t)jo * na + ai;
#pragma unroll
            for (int c = 0; c < NC; ++c) o[c * pitch] = res.v[c];
          }
        } else {
          // collect the column in the output tile; store it when complete
          const int col = (jo - s0) % Cf::OPS;
          const int buf = (Cf::NOUT == 2) ? ((jo - s0) / Cf::OPS) & 1 : 0;
          T* ob = sm.out + (size_t)buf * Cf::OUT;
          if (col == 0) {
            // the store that last read this tile has finished reading it
            if (lane == 0) {
              if (Cf::NOUT == 2)
                bulk_wait_read<1>();
              else
                bulk_wait_read<0>();
            }
            __syncwarp();
          }
#pragma unroll
          for (int c = 0; c < NC; ++c) ob[(c * 32 + lane) * Cf::OPS + col] = res.v[c];
          // the group is complete, or the strip ends (a partial group only
          // at the domain's end, where the store is cut at the extent)
          if (col == Cf::OPS - 1 || jo == s_end - 1) {
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
              tma_store_3d(tout, ob, jo - col, a0, 0);
              bulk_commit();
            }
          }
        }
        if ((FAST ? S == 1 : want_ws) && owned && (FAST || ws_row_counts(p, S == 1 ? jo : ai)))
          ws_max(ws_local, (double)max_wavespeed_q<STIFF>(derive(res, gm1), gamma, pinf));
      }
      f_prev = fj;
    }
    er_prev = er;
  }
  };
  using SB = std::integral_constant<int, kSuperbee>;
  using VL_ = std::integral_constant<int, kVanLeer>;
  if (!flip_l_on && !flip_a_on && flatten && want_ws == (S == 1) && p.ws_hi <= p.ws_lo) {
    if (p.limiter == kSuperbee)
      walk(SB{}, std::true_type{});
    else
      walk(VL_{}, std::true_type{});
  } else {
    if (p.limiter == kSuperbee)
      walk(SB{}, std::false_type{});
    else
      walk(VL_{}, std::false_type{});
  }
  if (fault) {
    // stop issuing; let every copy already issued land before the shared
    // memory is released (each wait bounded again)
    for (int t = waiting; t < issued; ++t) {
      const uint32_t g = g0 + (uint32_t)t;
      (void)mbar_wait_bounded(&sm.bars[g % NS], (g / NS) & 1u, 100000000ull);
    }
  }
  gstage = g0 + (uint32_t)nst;
}

// Strips are scheduled statically (each warp of the grid takes one strip)
// or, given strip counters, dynamically: a grid of resident CTAs whose warps
// take strips, across block fastest, from walk_next[walk_slot] until none is
// left.  The sweep clears the other counter, which the next sweep of the
// stream uses.  Both schedules run the same strip code.
template <typename T, int S, int FLUX, int GEO, bool TOUT>
__global__ void __launch_bounds__(StagedCfg<T, GEO, TOUT>::THREADS,
                                  StagedCfg<T, GEO, TOUT>::MIN_CTAS)
    staged_walk_2d(SweepParams p, const __grid_constant__ CUtensorMap tin,
                   const __grid_constant__ CUtensorMap tout) {
  using Cf = StagedCfg<T, GEO, TOUT>;
  if (p.walk_next != nullptr && blockIdx.x == 0 && threadIdx.x == 0)
    p.walk_next[1 - p.walk_slot] = 0u;
  if (p.ctrl != nullptr && *(volatile int*)&p.ctrl->done) return;
  const T dtdh = (p.ctrl != nullptr) ? (T)p.ctrl->dtdh : (T)p.dtdh;
  const T dhdt = T(1.0) / dtdh;  // Lax-Friedrichs coefficient, once per launch
  extern __shared__ __align__(128) unsigned char staged_smem[];
  __shared__ double s_red[Cf::WARPS];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t mis = smem_addr(staged_smem) & 127u;
  unsigned char* base = staged_smem + (mis ? 128u - mis : 0u);
  StagedSmem<T, GEO, TOUT> sm(base + (size_t)warp * Cf::WARP_BYTES);
  if (lane == 0) {
    for (int s = 0; s < Cf::NS; ++s) mbar_init(&sm.bars[s], 1);
    mbar_init_fence();
  }
  __syncwarp();

  double ws_local = 0.0;
  const bool want_ws = (p.ws_accum != nullptr);
  const int ry = (p.walk_ry > 0) ? p.walk_ry : Cf::RY;
  const int64_t nab = (p.n[1 - S] + 31) / 32;
  // positions along the walk to compute: a row window when the walk runs
  // along the rows (the y sweep in the grid's own layout), else all
  const bool win = S == 1 && !p.transposed && p.row_hi > p.row_lo;
  const int64_t w_lo = win ? p.row_lo : 0, w_hi = win ? p.row_hi : p.n[S];
  const int64_t items = nab * ((w_hi - w_lo + ry - 1) / ry);
  uint32_t gstage = 0;
  int fault = 0;
  unsigned int* next = (p.walk_next != nullptr) ? &p.walk_next[p.walk_slot] : nullptr;
  int64_t item = (int64_t)blockIdx.x * Cf::WARPS + warp;
  if (next != nullptr) {
    unsigned int v = 0u;
    if (lane == 0) v = atomicAdd(next, 1u);
    item = (int64_t)__shfl_sync(0xffffffffu, v, 0);
  }
  while (item < items && !fault) {
    const int64_t s0 = w_lo + (item / nab) * ry;
    staged_strip<T, S, FLUX, GEO, TOUT>(p, &tin, &tout, sm, dtdh, dhdt, (int)(item % nab),
                                        (int)s0, (int)(w_hi - s0 < ry ? w_hi - s0 : ry),
                                        ws_local, want_ws, gstage, fault);
    if (next == nullptr) break;
    unsigned int v = 0u;
    if (lane == 0) v = atomicAdd(next, 1u);
    item = (int64_t)__shfl_sync(0xffffffffu, v, 0);
  }
  if (TOUT && lane == 0) bulk_wait<0>();
  if (fault && lane == 0 && p.status != nullptr) {
    atomicExch(p.status, kETimeout);
    if (p.ctrl != nullptr) atomicExch(&p.ctrl->done, 1);
  }
  if (want_ws) {
    // CTA max of the lanes' wavespeeds (warp shuffles, then the CTA)
    double v = ws_local;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ws_max(v, __shfl_xor_sync(0xffffffffu, v, off));
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = s_red[0];
#pragma unroll
      for (int w = 1; w < Cf::WARPS; ++w) ws_max(m, s_red[w]);
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
