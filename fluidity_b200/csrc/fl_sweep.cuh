// fl_sweep.cuh -- the fused dimensional sweep kernel.
//
// One launch performs SplitSolver::invoke (solver/split_solver.hpp:138-162)
// for every cell of the grid in one dimension S:
//
//   out = U + dtdh * (F(i-1/2) - F(i+1/2))                 (split_solver.hpp:160)
//   F(i+1/2) = Riemann(evolve_R(i), evolve_L(i+1))         (flux_solver.hpp:92-98)
//
// Layout: structure-of-arrays component planes in HBM.  A CTA owns a tile of
// TX x TY x TZ output cells.  It stages the tile plus its halo -- 4 cells in
// the sweep dimension (MUSCL limiter + flattening reach i +- 4) and 3 across
// (the flattening coefficient reads +-3 in every dimension,
// reconstruction/muscl_reconstructor.hpp:104-111) -- in shared memory,
// computing each cell's pressure once on load.  Then, all in shared memory and
// registers:
//   stage C: per cell, the flattening chi, the limited slope and BOTH evolved
//            face states (each cell's two faces share one flux pair);
//   stage D: per face, one Riemann solve (the reference solves each face twice);
//   stage E: per cell, the conservative update, stored back to HBM, and when
//            asked the max wavespeed of the new state (fused CFL reduction:
//            warp shuffles, one atomic per CTA, last CTA advances the
//            device-resident time control).
//
// Out-of-domain cells are mirror ghosts in every dimension (ghost[-1-g] =
// cell[g], solver/boundary_loader.hpp:175-199) with the normal momentum
// negated as (-(m/rho))*rho at reflective ends (boundary_loader.hpp:66-73).
#pragma once

#include <cfloat>

#include "fl_internal.cuh"
#include "fl_numerics.cuh"

namespace fl {

// Output tile per (dims, sweep dim, dtype).  Widths favour contiguous x rows.
template <int D, int S, typename T>
struct TileShape {
  static constexpr int TX = (D == 1) ? 256 : (D == 2 ? (S == 0 ? 64 : 32) : 8);
  static constexpr int TY = (D == 1) ? 1 : (D == 2 ? (S == 0 ? 8 : 16) : 4);
  static constexpr int TZ = (D == 3) ? 4 : 1;
  static constexpr int THREADS = (D == 3) ? 128 : 256;
};

template <typename T, int D, int S>
struct SweepGeom {
  using TS_ = TileShape<D, S, T>;
  static constexpr int NC = D + 2;
  static constexpr int T0 = TS_::TX, T1 = TS_::TY, T2 = TS_::TZ;
  static constexpr int H0 = (D >= 1) ? (S == 0 ? 4 : 3) : 0;
  static constexpr int H1 = (D >= 2) ? (S == 1 ? 4 : 3) : 0;
  static constexpr int H2 = (D >= 3) ? (S == 2 ? 4 : 3) : 0;
  static constexpr int R0 = T0 + 2 * H0, R1 = T1 + 2 * H1, R2 = T2 + 2 * H2;
  static constexpr int R = R0 * R1 * R2;                      // region cells
  // evolve cells: tile extended by one cell on each side of the sweep dim
  static constexpr int E0 = T0 + (S == 0 ? 2 : 0);
  static constexpr int E1 = T1 + (S == 1 ? 2 : 0);
  static constexpr int E2 = T2 + (S == 2 ? 2 : 0);
  static constexpr int E = E0 * E1 * E2;
  // faces: tile plus one along the sweep dim
  static constexpr int F0 = T0 + (S == 0 ? 1 : 0);
  static constexpr int F1 = T1 + (S == 1 ? 1 : 0);
  static constexpr int F2 = T2 + (S == 2 ? 1 : 0);
  static constexpr int F = F0 * F1 * F2;
  static constexpr int OUT = T0 * T1 * T2;
  static constexpr int THREADS = TS_::THREADS;
  // shared memory: U (NC planes), P, velocities (D planes), chi bases (D
  // planes) over the region; evolved faces ER, EL; face fluxes FX alias the
  // velocity + chi planes (dead after stage C) when they fit.
  static constexpr bool FX_ALIAS = 2 * D * R >= NC * F;
  static constexpr size_t smem_elems =
      (size_t)NC * R + R + 2 * D * R + 2 * NC * E + (FX_ALIAS ? 0 : NC * F);
  static constexpr size_t smem_bytes = sizeof(T) * smem_elems + 64;
  __host__ __device__ static constexpr int rstride(int d) {
    return d == 0 ? 1 : (d == 1 ? R0 : R0 * R1);
  }
  __host__ __device__ static constexpr int estride(int d) {
    return d == 0 ? 1 : (d == 1 ? E0 : E0 * E1);
  }
  __host__ __device__ static constexpr int tile(int d) { return d == 0 ? T0 : (d == 1 ? T1 : T2); }
  __host__ __device__ static constexpr int halo(int d) { return d == 0 ? H0 : (d == 1 ? H1 : H2); }
};

__device__ __forceinline__ int64_t mirror_index(int64_t g, int64_t n, bool& flipped) {
  flipped = false;
  if (g < 0) { g = -1 - g; flipped = true; }
  else if (g >= n) { g = 2 * n - 1 - g; flipped = true; }
  // beyond one mirror (only cells whose results are discarded): clamp
  g = g < 0 ? 0 : (g >= n ? n - 1 : g);
  return g;
}

// acc = max(acc, v), except that a NaN, once seen, stays: a non-finite
// wavespeed anywhere must reach the step control (which stops the loop with
// FL_ENAN), whatever the order in which cells and lanes are folded.
__device__ __forceinline__ void ws_max(double& acc, double v) {
  if (acc == acc && !(v <= acc)) acc = v;
}

// Advance the time control after the last sweep of a step
// (Parameters::update_simulation_info / update_time_delta / continue_simulation,
// simulator/parameters.hpp:60-77).
__device__ __forceinline__ void finalize_control(StepControl* c, bool advance) {
  const double ws = __longlong_as_double((long long)atomicAdd(&c->ws_bits, 0ull));
  if (advance) {
    if (c->is_f32) c->run_time = (double)((float)c->run_time + (float)c->dt);
    else c->run_time = c->run_time + c->dt;
    c->iters += 1;
  }
  double dt, dtdh;
  if (c->is_f32) {
    dt = (double)(float)((double)(float)c->cfl * c->res / (double)(float)ws);
    dtdh = (double)(float)(dt / c->res);
  } else {
    dt = c->cfl * c->res / ws;
    dtdh = dt / c->res;
  }
  c->dt = dt;
  c->dtdh = dtdh;
  bool cont = (c->run_time < c->sim_time) && (c->iters < c->max_iters);
  if (!(ws > 0.0) || !(ws <= DBL_MAX)) {
    c->status = kENan;
    cont = false;
  }
  c->done = cont ? 0 : 1;
  c->ws_bits = 0ull;
  __threadfence();
  c->arrive = 0u;
}

// Block-wide max of per-thread wavespeeds, one atomic per CTA, and the
// last-CTA-done hand-off that advances the time control.
template <int THREADS>
__device__ __forceinline__ void cta_wavespeed_commit(double local, unsigned long long* accum,
                                                     StepControl* ctrl, int finalize,
                                                     bool advance, double* s_red) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) ws_max(local, __shfl_xor_sync(0xffffffffu, local, off));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) s_red[warp] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = s_red[0];
#pragma unroll
    for (int w = 1; w < THREADS / 32; ++w) ws_max(m, s_red[w]);
    atomicMax(accum, (unsigned long long)__double_as_longlong(m));
    if (finalize && ctrl) {
      __threadfence();
      const unsigned int total = gridDim.x * gridDim.y * gridDim.z;
      const unsigned int prev = atomicAdd(&ctrl->arrive, 1u);
      if (prev == total - 1) {
        __threadfence();
        finalize_control(ctrl, advance);
      }
    }
  }
}

template <typename T, int D, int S, int FLUX>
__global__ void __launch_bounds__(SweepGeom<T, D, S>::THREADS)
sweep_kernel(SweepParams p) {
  using G = SweepGeom<T, D, S>;
  constexpr int NC = G::NC;
  constexpr int NT = G::THREADS;

  if (p.ctrl != nullptr && *(volatile int*)&p.ctrl->done) return;
  const T dtdh = (p.ctrl != nullptr) ? (T)p.ctrl->dtdh : (T)p.dtdh;
  constexpr bool STIFF = (FLUX & kStiffEos) != 0;
  const T gamma = (T)p.gamma;
  const T pinf = (T)p.pinf;
  const T gm1 = gamma - T(1);
  const T adi = (gamma + T(1)) / (T(2) * gamma);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sU = reinterpret_cast<T*>(smem_raw);   // [NC][R]
  T* sP = sU + NC * G::R;                     // [R]
  T* sV = sP + G::R;                          // [D][R] velocities
  T* sChi = sV + D * G::R;                    // [D][R] chi bases
  T* sER = sChi + D * G::R;                   // [NC][E]
  T* sEL = sER + NC * G::E;                   // [NC][E]
  T* sFX = G::FX_ALIAS ? sV : sEL + NC * G::E;  // [NC][F]
  __shared__ double s_red[NT / 32];

  const T* __restrict__ in = static_cast<const T*>(p.in);
  T* __restrict__ out = static_cast<T*>(p.out);
  const int64_t pitch = p.pitch;
  const int64_t n0 = p.n[0], n1 = p.n[1], n2 = p.n[2];
  const int64_t o0 = (int64_t)blockIdx.x * G::T0;
  const int64_t o1 = (int64_t)blockIdx.y * G::T1;
  const int64_t o2 = (int64_t)blockIdx.z * G::T2;
  const bool muscl = !p.basic;
  const bool flatten = muscl && p.flatten;

  // ---- stage A: load tile + halo, mirror ghosts, derived quantities -----
  for (int r = threadIdx.x; r < G::R; r += NT) {
    const int l0 = r % G::R0;
    const int l1 = (r / G::R0) % G::R1;
    const int l2 = r / (G::R0 * G::R1);
    bool f0 = false, f1 = false, f2 = false;
    const int64_t g0 = mirror_index(o0 - G::H0 + l0, n0, f0);
    const int64_t g1 = (D >= 2) ? mirror_index(o1 - G::H1 + l1, n1, f1) : 0;
    const int64_t g2 = (D >= 3) ? mirror_index(o2 - G::H2 + l2, n2, f2) : 0;
    const int64_t gi = (g2 * n1 + g1) * n0 + g0;
    Cons<T, D> u;
#pragma unroll
    for (int c = 0; c < NC; ++c) u.v[c] = __ldg(in + c * pitch + gi);
    if (f0 && (p.reflect & 1u)) u.v[2] = (-(u.v[2] / u.v[0])) * u.v[0];
    if (D >= 2 && f1 && (p.reflect & 2u)) u.v[3] = (-(u.v[3] / u.v[0])) * u.v[0];
    if (D >= 3 && f2 && (p.reflect & 4u)) u.v[4] = (-(u.v[4] / u.v[0])) * u.v[0];
    const Derived<T, D> q = derive(u, gm1);
#pragma unroll
    for (int c = 0; c < NC; ++c) sU[c * G::R + r] = u.v[c];
    sP[r] = q.p;
#pragma unroll
    for (int d = 0; d < D; ++d) sV[d * G::R + r] = q.v[d];
  }
  __syncthreads();

  // ---- stage B: flattening bases chi(c, d) for every cell and dimension
  // that stage C reads (muscl_reconstructor.hpp:59-87) -------------------
  if (flatten) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      // box, in tile coordinates: along S the evolve range [-1, T_S] widened
      // by one more when d == S; along d != S the tile widened by one.
      int lo[3], ext[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        lo[k] = 0;
        ext[k] = (k < D) ? G::tile(k) : 1;
      }
      lo[S] = (d == S) ? -2 : -1;
      ext[S] = G::tile(S) + ((d == S) ? 4 : 2);
      if (d != S) { lo[d] = -1; ext[d] = G::tile(d) + 2; }
      const int count = ext[0] * ext[1] * ext[2];
      const int st = G::rstride(d);
      const T* vd = sV + d * G::R;
      for (int i = threadIdx.x; i < count; i += NT) {
        const int c0 = i % ext[0] + lo[0];
        const int c1 = (i / ext[0]) % ext[1] + lo[1];
        const int c2 = i / (ext[0] * ext[1]) + lo[2];
        const int q = ((c2 + G::H2) * G::R1 + (c1 + G::H1)) * G::R0 + (c0 + G::H0);
        sChi[d * G::R + q] = (T)chi_base<T>(sP[q + st], sP[q - st], sP[q + 2 * st],
                                            sP[q - 2 * st], vd[q - st], vd[q + st]);
      }
    }
    __syncthreads();
  }

  // ---- stage C: limited slope, evolved face states -----------------------
  constexpr int SS = G::rstride(S);
  for (int e = threadIdx.x; e < G::E; e += NT) {
    const int e0 = e % G::E0;
    const int e1 = (e / G::E0) % G::E1;
    const int e2 = e / (G::E0 * G::E1);
    const int q0 = e0 + G::H0 - (S == 0 ? 1 : 0);
    const int q1 = e1 + G::H1 - (S == 1 ? 1 : 0);
    const int q2 = e2 + G::H2 - (S == 2 ? 1 : 0);
    const int q = (q2 * G::R1 + q1) * G::R0 + q0;
    Cons<T, D> u;
#pragma unroll
    for (int c = 0; c < NC; ++c) u.v[c] = sU[c * G::R + q];
    Cons<T, D> er, el;
    if (!muscl) {
      er = u;
      el = u;
    } else {
      T chi_v = T(1);
      if (flatten) {
        chi_v = (sizeof(T) == 8) ? (T)DBL_MAX : (T)FLT_MAX;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const int st = G::rstride(d);
          const T diff = sP[q + st] - sP[q - st];
          const int sign = (T(0) < diff) - (diff < T(0));
          const T* cd = sChi + d * G::R;
          chi_v = std_min(chi_v, std_min(cd[q], cd[q + sign * st]));
        }
      }
      const T ch = chi_v * T(0.5);
      Cons<T, D> a, b;  // a = U - delta, b = U + delta
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const T um = sU[c * G::R + q - SS];
        const T up = sU[c * G::R + q + SS];
        const T delta = ch * limited_slope<T>(p.limiter, u.v[c] - um, up - u.v[c]);
        a.v[c] = u.v[c] - delta;
        b.v[c] = u.v[c] + delta;
      }
      Cons<T, D> fa, fb;
      flux_q(a, derive(a, gm1), S, fa);
      flux_q(b, derive(b, gm1), S, fb);
      const T hd = T(0.5) * dtdh;
      // right face: (U+d) + hd (F(U-d) - F(U+d)); left face: (U-d) + hd (F(U-d) - F(U+d))
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const T df = fa.v[c] - fb.v[c];
        er.v[c] = b.v[c] + hd * df;
        el.v[c] = a.v[c] + hd * df;
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      sER[c * G::E + e] = er.v[c];
      sEL[c * G::E + e] = el.v[c];
    }
  }
  __syncthreads();

  // ---- stage D: one Riemann solve per face ------------------------------
  constexpr int ES = G::estride(S);
  for (int f = threadIdx.x; f < G::F; f += NT) {
    const int f0 = f % G::F0;
    const int f1 = (f / G::F0) % G::F1;
    const int f2 = f / (G::F0 * G::F1);
    // face f sits between evolve cells f (left) and f + 1 (right) along S
    const int el_idx = (f2 * G::E1 + f1) * G::E0 + f0;
    Cons<T, D> ul, ur, fx;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      ul.v[c] = sER[c * G::E + el_idx];
      ur.v[c] = sEL[c * G::E + el_idx + ES];
    }
    riemann_q<FLUX>(ul, derive(ul, gm1), ur, derive(ur, gm1), S, gamma, gm1, adi, dtdh, fx,
                    pinf);
#pragma unroll
    for (int c = 0; c < NC; ++c) sFX[c * G::F + f] = fx.v[c];
  }
  __syncthreads();

  // ---- stage E: conservative update, store, fused wavespeed -------------
  constexpr int FS = (S == 0) ? 1 : (S == 1 ? G::F0 : G::F0 * G::F1);
  double ws_local = 0.0;
  const bool want_ws = (p.ws_accum != nullptr);
  for (int o = threadIdx.x; o < G::OUT; o += NT) {
    const int t0 = o % G::T0;
    const int t1 = (o / G::T0) % G::T1;
    const int t2 = o / (G::T0 * G::T1);
    const int64_t g0 = o0 + t0, g1 = o1 + t1, g2 = o2 + t2;
    if (g0 >= n0 || g1 >= n1 || g2 >= n2) continue;
    const int q = ((t2 + G::H2) * G::R1 + (t1 + G::H1)) * G::R0 + (t0 + G::H0);
    const int fi = (t2 * G::F1 + t1) * G::F0 + t0;   // left face of the cell
    const int64_t gi = (g2 * n1 + g1) * n0 + g0;
    Cons<T, D> r;
#pragma unroll
    for (int c = 0; c < NC; ++c)
      r.v[c] = sU[c * G::R + q] + dtdh * (sFX[c * G::F + fi] - sFX[c * G::F + fi + FS]);
#pragma unroll
    for (int c = 0; c < NC; ++c) out[c * pitch + gi] = r.v[c];
    if (want_ws && ws_row_counts(p, D == 1 ? g0 : (D == 2 ? g1 : g2)))
      ws_max(ws_local, (double)max_wavespeed_q<STIFF>(derive(r, gm1), gamma, pinf));
  }
  if (want_ws)
    cta_wavespeed_commit<NT>(ws_local, p.ws_accum, p.ctrl, p.finalize, true, s_red);
}

}  // namespace fl
