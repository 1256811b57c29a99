// fl_batch.cuh -- batched solver for thousands of independent problems.
//
// No reference counterpart: the reference solves one grid per simulator.
// Each problem is the reference's split-solver time loop (simulator_impl.hpp
// :223-258) with its own CFL time step; the arithmetic per cell is that of
// sweep_kernel / walk_kernel_2d.
//
// * 1-D problems (n <= kBatch1dMax(T)) live in shared memory for the whole
//   launch: a persistent CTA pops a problem from an atomic work queue (largest
//   first), loads its state once, runs every time step in shared memory --
//   ghost refresh, one sweep with the MUSCL stencil streamed through
//   registers, the block-wide CFL reduction and the Parameters update -- and
//   writes the state and its time control back once.
// * 2-D problems run one batched launch per sweep: a CTA is one work item
//   (problem, column group, strip row) of the register-streaming walker; the
//   last item of a problem to finish its y sweep advances that problem's time
//   control.
#pragma once

#include <type_traits>

#include <cfloat>

#include "fl_internal.cuh"
#include "fl_numerics.cuh"
#include "fl_sweep.cuh"
#include "fl_walk.cuh"

namespace fl {

// Device descriptor of one problem of a batch.
struct BatchProblem {
  int64_t n0, n1;     // cells (n1 = 1 in 1-D)
  int64_t offset;     // element offset of component plane 0 in the arenas
  int64_t pitch;      // elements between component planes
  int dims;           // 1 or 2
  int ry;             // 2-D: rows per warp strip (autotuned)
  int items;          // 2-D: work items of the problem (CTAs per sweep)
  int pad_;
};

// One 2-D work item: WalkCfg::WARPS stacked strips of one column group.
struct BatchItem {
  int problem;
  int bx;
  int by;
  int pad_;
};

struct BatchArgs {
  const BatchProblem* problems;
  StepControl* ctrl;          // one per problem
  const BatchItem* items;     // 2-D work items
  const int* order;           // 1-D problems in queue order (largest first)
  int* queue;                 // 1-D work-queue head (reset before each launch)
  int count;                  // items (2-D launch) or 1-D problems in `order`
  void* arena_a;              // states; every problem's result ends here
  void* arena_b;              // 2-D ping-pong partner
  double gamma;
  double pinf;                // stiffened fluid's p_inf (0: ideal gas), every problem
  int limiter;
  int basic;
  int flatten;
  uint32_t reflect;
};

template <typename T>
constexpr int batch1d_max() {
  // two state copies of 3 planes with 4 ghosts per side in < 220 KB
  return (int)((220 * 1024) / (2 * 3 * sizeof(T))) - 8;
}

// Advance one problem's control after a step given the step's max wavespeed
// (Parameters::update_simulation_info / update_time_delta /
// continue_simulation, simulator/parameters.hpp:60-77).
__device__ __forceinline__ void advance_control(StepControl& c, double ws, bool advance) {
  if (advance) {
    if (c.is_f32) c.run_time = (double)((float)c.run_time + (float)c.dt);
    else c.run_time = c.run_time + c.dt;
    c.iters += 1;
  }
  if (c.is_f32) {
    c.dt = (double)(float)((double)(float)c.cfl * c.res / (double)(float)ws);
    c.dtdh = (double)(float)(c.dt / c.res);
  } else {
    c.dt = c.cfl * c.res / ws;
    c.dtdh = c.dt / c.res;
  }
  bool cont = (c.run_time < c.sim_time) && (c.iters < c.max_iters);
  if (!(ws > 0.0) || !(ws <= DBL_MAX)) {
    c.status = kENan;
    cont = false;
  }
  c.done = cont ? 0 : 1;
}

// ---- initial wavespeed of every problem (one CTA per problem) -------------

template <typename T>
__global__ void __launch_bounds__(256) batch_init_kernel(BatchArgs a, int nprob, double cfl,
                                                         double sim_time, long long max_iters,
                                                         const double* res) {
  __shared__ double s_red[8];
  const int pid = blockIdx.x;
  if (pid >= nprob) return;
  const BatchProblem pr = a.problems[pid];
  const T* in = static_cast<const T*>(a.arena_a) + pr.offset;
  const T gamma = (T)a.gamma, gm1 = gamma - T(1), pinf = (T)a.pinf;
  const bool stiff = a.pinf != 0.0;
  const int64_t cells = pr.n0 * pr.n1;
  double local = 0.0;
  for (int64_t i = threadIdx.x; i < cells; i += blockDim.x) {
    if (pr.dims == 1) {
      Cons<T, 1> u;
      for (int c = 0; c < 3; ++c) u.v[c] = in[c * pr.pitch + i];
      const Derived<T, 1> q = derive(u, gm1);
      ws_max(local, (double)(stiff ? max_wavespeed_q<true>(q, gamma, pinf)
                                   : max_wavespeed_q<false>(q, gamma)));
    } else {
      Cons<T, 2> u;
      for (int c = 0; c < 4; ++c) u.v[c] = in[c * pr.pitch + i];
      const Derived<T, 2> q = derive(u, gm1);
      ws_max(local, (double)(stiff ? max_wavespeed_q<true>(q, gamma, pinf)
                                   : max_wavespeed_q<false>(q, gamma)));
    }
  }
  const double m = cta_max<8>(local, s_red);
  if (threadIdx.x == 0) {
    StepControl c;
    c.dt = 0.0;
    c.dtdh = 0.0;
    c.run_time = 0.0;
    c.is_f32 = sizeof(T) == 4;
    c.sim_time = c.is_f32 ? (double)(float)sim_time : sim_time;
    c.cfl = c.is_f32 ? (double)(float)cfl : cfl;
    c.res = res[pid];
    c.iters = 0;
    c.max_iters = max_iters;
    c.ws_bits = 0ull;
    c.arrive = 0u;
    c.status = 0;
    c.walk_next[0] = 0u;
    c.walk_next[1] = 0u;
    advance_control(c, m, false);
    a.ctrl[pid] = c;
  }
}

__global__ void batch_reset_queue_kernel(int* queue) { *queue = 0; }

// ---- 1-D: one problem per CTA, resident in shared memory ------------------

// New states of cells [c0, c1) of a 1-D line held in shared memory with 4
// ghosts per side (cell i at index i + 4 of each plane, plane stride ld),
// written to the same positions of dst.  Same streaming scheme as the y sweep
// of walk_strip_2d, along x.
template <typename T, int FLUX>
__device__ __forceinline__ void walk_line_1d(const T* src, T* dst, int ld, int c0, int c1,
                                             T gamma, T gm1, T adi, T dtdh, int limiter,
                                             bool muscl, bool flatten, double& ws_local,
                                             T pinf) {
  constexpr int D = 1;
  constexpr int NC = 3;
  constexpr bool STIFF = (FLUX & kStiffEos) != 0;
  const T hd = T(0.5) * dtdh;
  const T chi_init = (sizeof(T) == 8) ? (T)DBL_MAX : (T)FLT_MAX;
  Cons<T, D> U[5];
  T P[5], V[5];
  T CH[3];
  Cons<T, D> er_prev, f_prev;
  // the walk, with the limiter kind fixed for the whole row
  auto walk = [&](auto lim) {
  for (int k = c0 - 4; k <= c1 + 3; ++k) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      U[i] = U[i + 1];
      P[i] = P[i + 1];
      V[i] = V[i + 1];
    }
    Cons<T, D> u;
#pragma unroll
    for (int c = 0; c < NC; ++c) u.v[c] = src[c * ld + 4 + k];
    const Derived<T, D> q = derive(u, gm1);
    U[4] = u;
    P[4] = q.p;
    V[4] = q.v[0];
    CH[0] = CH[1];
    CH[1] = CH[2];
    if (flatten) CH[2] = (T)chi_base<T>(P[3], P[1], P[4], P[0], V[1], V[3]);
    const int j = k - 3;
    if (j < c0 - 1) continue;
    const Cons<T, D>& uj = U[1];
    Cons<T, D> er, el;
    if (!muscl) {
      er = uj;
      el = uj;
    } else {
      T chi_v = T(1);
      if (flatten) {
        const T dx = P[2] - P[0];
        const int sx = (T(0) < dx) - (dx < T(0));
        chi_v = std_min(chi_init, std_min(CH[1], sx > 0 ? CH[2] : (sx < 0 ? CH[0] : CH[1])));
      }
      const T ch = chi_v * T(0.5);
      Cons<T, D> aa, bb;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const T delta = ch * limited_slope<T>(decltype(lim)::value, uj.v[c] - U[0].v[c],
                                                U[2].v[c] - uj.v[c]);
          aa.v[c] = uj.v[c] - delta;
          bb.v[c] = uj.v[c] + delta;
        }
      Cons<T, D> fa, fb;
      flux_q(aa, derive(aa, gm1), 0, fa);
      flux_q(bb, derive(bb, gm1), 0, fb);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const T df = fa.v[c] - fb.v[c];
        er.v[c] = bb.v[c] + hd * df;
        el.v[c] = aa.v[c] + hd * df;
      }
    }
    if (j >= c0) {
      Cons<T, D> fx;
      riemann_q<FLUX>(er_prev, derive(er_prev, gm1), el, derive(el, gm1), 0, gamma, gm1, adi,
                      dtdh, fx, pinf);
      if (j >= c0 + 1) {
        const Cons<T, D>& uo = U[0];
        Cons<T, D> r;
#pragma unroll
        for (int c = 0; c < NC; ++c) r.v[c] = uo.v[c] + dtdh * (f_prev.v[c] - fx.v[c]);
#pragma unroll
        for (int c = 0; c < NC; ++c) dst[c * ld + 4 + (j - 1)] = r.v[c];
        ws_max(ws_local, (double)max_wavespeed_q<STIFF>(derive(r, gm1), gamma, pinf));
      }
      f_prev = fx;
    }
    er_prev = er;
  }
  };
  if (limiter == kSuperbee)
    walk(std::integral_constant<int, kSuperbee>{});
  else
    walk(std::integral_constant<int, kVanLeer>{});
}

template <typename T>
__device__ __forceinline__ void fill_ghosts_1d(T* s, int ld, int n, bool reflect) {
  // ghost[-1-g] = cell[g], ghost[n+g] = cell[n-1-g]; reflective: m -> (-(m/rho))*rho
  const int t = threadIdx.x;
  if (t < 8) {
    const int g = t & 3;
    const int src = (t < 4) ? g : n - 1 - g;
    const int dst = (t < 4) ? -1 - g : n + g;
    const T rho = s[4 + src];
    T m = s[2 * ld + 4 + src];
    if (reflect) m = (-(m / rho)) * rho;
    s[4 + dst] = rho;
    s[ld + 4 + dst] = s[ld + 4 + src];
    s[2 * ld + 4 + dst] = m;
  }
}

template <typename T, int FLUX, int THREADS>
__global__ void __launch_bounds__(THREADS) batch1d_kernel(BatchArgs a, long long nsteps, int ld) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sA = reinterpret_cast<T*>(smem_raw);
  T* sB = sA + 3 * ld;
  __shared__ double s_red[THREADS / 32];
  __shared__ int s_pid;
  __shared__ StepControl s_ctrl;
  const T gamma = (T)a.gamma, gm1 = gamma - T(1);
  const T adi = (gamma + T(1)) / (T(2) * gamma);
  const T pinf = (T)a.pinf;
  const bool muscl = !a.basic;
  const bool flatten = muscl && a.flatten;
  const bool reflect = (a.reflect & 1u) != 0;
  while (true) {
    if (threadIdx.x == 0) s_pid = atomicAdd(a.queue, 1);
    __syncthreads();
    const int qi = s_pid;
    if (qi >= a.count) break;
    const int pid = a.order[qi];
    const BatchProblem pr = a.problems[pid];
    const int n = (int)pr.n0;
    T* g = static_cast<T*>(a.arena_a) + pr.offset;
    for (int i = threadIdx.x; i < n; i += THREADS)
      for (int c = 0; c < 3; ++c) sA[c * ld + 4 + i] = g[c * pr.pitch + i];
    if (threadIdx.x == 0) s_ctrl = a.ctrl[pid];
    __syncthreads();
    // contiguous segments of at least 4 cells per thread
    const int per = (n + THREADS - 1) / THREADS < 4 ? 4 : (n + THREADS - 1) / THREADS;
    const int c0 = threadIdx.x * per;
    const int c1 = (c0 + per < n) ? c0 + per : n;
    T* cur = sA;
    T* nxt = sB;
    for (long long s = 0; s < nsteps; ++s) {
      if (s_ctrl.done) break;                       // uniform: read after a barrier
      const T dtdh = (T)s_ctrl.dtdh;
      fill_ghosts_1d(cur, ld, n, reflect);
      __syncthreads();
      double ws = 0.0;
      if (c0 < n)
        walk_line_1d<T, FLUX>(cur, nxt, ld, c0, c1, gamma, gm1, adi, dtdh, a.limiter, muscl,
                              flatten, ws, pinf);
      const double m = cta_max<THREADS / 32>(ws, s_red);
      if (threadIdx.x == 0) advance_control(s_ctrl, m, true);
      __syncthreads();
      T* t = cur;
      cur = nxt;
      nxt = t;
    }
    for (int i = threadIdx.x; i < n; i += THREADS)
      for (int c = 0; c < 3; ++c) g[c * pr.pitch + i] = cur[c * ld + 4 + i];
    if (threadIdx.x == 0) a.ctrl[pid] = s_ctrl;
    __syncthreads();
  }
}

// ---- 2-D: one batched launch per sweep -------------------------------------

template <typename T, int S, int FLUX>
__global__ void __launch_bounds__(WalkCfg<T, S>::THREADS) batch2d_kernel(BatchArgs a) {
  using W = WalkCfg<T, S>;
  __shared__ double s_red[W::WARPS];
  const BatchItem it = a.items[blockIdx.x];
  const BatchProblem pr = a.problems[it.problem];
  StepControl* ctrl = a.ctrl + it.problem;
  if (*(volatile int*)&ctrl->done) return;           // uniform over the CTA
  const T dtdh = (T)ctrl->dtdh;
  SweepParams p;
  p.in = static_cast<const T*>(S == 0 ? a.arena_a : a.arena_b) + pr.offset;
  p.out = static_cast<T*>(S == 0 ? a.arena_b : a.arena_a) + pr.offset;
  p.pitch = pr.pitch;
  p.n[0] = pr.n0;
  p.n[1] = pr.n1;
  p.n[2] = 1;
  p.gamma = a.gamma;
  p.pinf = a.pinf;
  p.dtdh = 0.0;
  p.limiter = a.limiter;
  p.basic = a.basic;
  p.flatten = a.flatten;
  p.reflect = a.reflect;
  p.ctrl = nullptr;
  p.ws_accum = nullptr;
  p.ws_lo = 0;
  p.ws_hi = 0;
  p.finalize = 0;
  const int warp = threadIdx.x >> 5;
  const int64_t y0 = ((int64_t)it.by * W::WARPS + warp) * pr.ry;
  double ws_local = 0.0;
  walk_strip_2d<T, S, FLUX>(p, dtdh, (int64_t)it.bx, y0, pr.ry, ws_local, S == 1);
  if (S == 1) {
    const double m = cta_max<W::WARPS>(ws_local, s_red);
    if (threadIdx.x == 0) {
      atomicMax(&ctrl->ws_bits, (unsigned long long)__double_as_longlong(m));
      __threadfence();
      const unsigned int prev = atomicAdd(&ctrl->arrive, 1u);
      if (prev == (unsigned int)pr.items - 1) {
        __threadfence();
        finalize_control(ctrl, true);
      }
    }
  }
}

}  // namespace fl
