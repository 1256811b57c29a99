// fl_adjoint_sweep.cuh -- reverse of one dimensional sweep.
//
// Forward (sweep_kernel): U'_i = U_i + dtdh (F(i-1/2) - F(i+1/2)),
// F(f) = RS(er(f-1), el(f)), (er, el)(e) = evolve(U_{e-1}, U_e, U_{e+1}; chi_e).
// Reverse, for a given adjoint lam' of U':
//   g_f        = dtdh (lam'_f - lam'_{f-1})            for faces inside the domain
//   (er_b, el_b) from RS^T g_f                          (hllc_rev / force_rev)
//   (dUm, dU, dUp)_e from evolve^T (er_b_e, el_b_e)     (evolve_rev)
//   lam_i      = lam'_i + dUp_{i-1} + dU_i + dUm_{i+1}
// plus, at the two ends of the domain, the adjoints that reach ghost cells
// folded back onto the cells they mirror (the normal momentum negated at a
// reflective end).  chi and the wave/limiter branches are frozen (see
// fl_adjoint.cuh), so lines along the sweep are independent; chi's value
// still needs the cross-dimension neighbours.  Tile: T_S cells along the
// sweep, halo 5 along it (the forward faces of evolve cells [-2, T_S+1]),
// 3 across.
#pragma once

#include <cfloat>

#include "fl_adjoint.cuh"
#include "fl_internal.cuh"
#include "fl_numerics.cuh"
#include "fl_sweep.cuh"

namespace fl {

struct AdjointParams {
  const void* u;        // input state of the forward sweep
  const void* lam_out;  // adjoint of its output
  void* lam_in;         // adjoint of its input (written)
  int64_t pitch;
  int64_t n[3];
  double gamma;
  double pinf;          // stiffened fluid's p_inf (0: ideal gas)
  double dtdh;
  int flatten;
  int basic;
  uint32_t reflect;
};

template <int D, int S>
struct AdjTile {
  static constexpr int T0 = (D == 1) ? 128 : 32;
  static constexpr int T1 = (D == 1) ? 1 : 8;
  static constexpr int THREADS = 256;
};

template <typename T, int D, int S>
struct AdjGeom {
  using TS_ = AdjTile<D, S>;
  static constexpr int NC = D + 2;
  static constexpr int T0 = TS_::T0, T1 = TS_::T1;
  static constexpr int H0 = (S == 0) ? 5 : 3;
  static constexpr int H1 = (D >= 2) ? ((S == 1) ? 5 : 3) : 0;
  static constexpr int R0 = T0 + 2 * H0, R1 = T1 + 2 * H1;
  static constexpr int R = R0 * R1;
  // evolve cells [-2, T_S + 1] along S
  static constexpr int E0 = T0 + (S == 0 ? 4 : 0), E1 = T1 + (S == 1 ? 4 : 0);
  static constexpr int E = E0 * E1;
  static constexpr int OUT = T0 * T1;
  static constexpr int THREADS = TS_::THREADS;
  // CTAs per SM the registers are held to (shared memory allows 2 in FP64,
  // 4 or 5 in FP32)
#ifndef FL_ADJ_CTAS_F64
#define FL_ADJ_CTAS_F64 2
#endif
#ifndef FL_ADJ_CTAS_F32
#define FL_ADJ_CTAS_F32 3
#endif
  static constexpr int MIN_CTAS = sizeof(T) == 8 ? FL_ADJ_CTAS_F64 : FL_ADJ_CTAS_F32;
  // dUm, dU, dUp (stages E-F) reuse buffers dead by then: er and el (last
  // read in stage D) and the P, V, chi-base planes (last read in stage C)
  static_assert(NC * E <= R + 2 * D * R, "dUp must fit in the P, V and chi planes");
  static constexpr size_t smem_elems =
      (size_t)NC * R + R + 2 * D * R       // U, P, V, chi bases
      + E                                   // chi_v of evolve cells
      + 4 * NC * E                          // er, el, er_b, el_b
      + NC * E;                             // lam_out on evolve cells
  static constexpr size_t smem_bytes = sizeof(T) * smem_elems + 64;
  __host__ __device__ static constexpr int rstride(int d) { return d == 0 ? 1 : R0; }
  __host__ __device__ static constexpr int estride(int d) { return d == 0 ? 1 : E0; }
  __host__ __device__ static constexpr int tile(int d) { return d == 0 ? T0 : T1; }
};

template <typename T, int D, int S, int FLUX>
__global__ void __launch_bounds__(AdjGeom<T, D, S>::THREADS, AdjGeom<T, D, S>::MIN_CTAS)
adjoint_sweep_kernel(AdjointParams p) {
  using G = AdjGeom<T, D, S>;
  constexpr int NC = G::NC;
  constexpr int NT = G::THREADS;
  const T gamma = (T)p.gamma, gm1 = gamma - T(1);
  const T adi = (gamma + T(1)) / (T(2) * gamma);
  const T pinf = (T)p.pinf;
  const T dtdh = (T)p.dtdh;
  const bool muscl = !p.basic;
  const bool flatten = muscl && p.flatten;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sU = reinterpret_cast<T*>(smem_raw);
  T* sP = sU + NC * G::R;
  T* sV = sP + G::R;
  T* sChi = sV + D * G::R;
  T* sCv = sChi + D * G::R;       // [E]
  T* sER = sCv + G::E;            // [NC][E]
  T* sEL = sER + NC * G::E;
  T* sERb = sEL + NC * G::E;
  T* sELb = sERb + NC * G::E;
  T* sLam = sELb + NC * G::E;     // lam_out at evolve cells
  T* sDm = sER;                   // stages E-F: er, el and P/V/chi are dead
  T* sD0 = sEL;
  T* sDp = sP;

  const T* __restrict__ u_in = static_cast<const T*>(p.u);
  const T* __restrict__ lo = static_cast<const T*>(p.lam_out);
  T* __restrict__ li = static_cast<T*>(p.lam_in);
  const int64_t pitch = p.pitch;
  const int64_t n0 = p.n[0], n1 = (D >= 2) ? p.n[1] : 1;
  const int64_t nS = (S == 0) ? n0 : n1;
  const int64_t o0 = (int64_t)blockIdx.x * G::T0;
  const int64_t o1 = (int64_t)blockIdx.y * G::T1;
  const int64_t oS = (S == 0) ? o0 : o1;

  // ---- A: state tile + halo, mirror ghosts, derived quantities ----------
  for (int r = threadIdx.x; r < G::R; r += NT) {
    const int l0 = r % G::R0, l1 = r / G::R0;
    bool f0 = false, f1 = false;
    const int64_t g0 = mirror_index(o0 - G::H0 + l0, n0, f0);
    const int64_t g1 = (D >= 2) ? mirror_index(o1 - G::H1 + l1, n1, f1) : 0;
    const int64_t gi = g1 * n0 + g0;
    Cons<T, D> u;
#pragma unroll
    for (int c = 0; c < NC; ++c) u.v[c] = u_in[c * pitch + gi];
    if (f0 && (p.reflect & 1u)) u.v[2] = (-(u.v[2] / u.v[0])) * u.v[0];
    if (D >= 2 && f1 && (p.reflect & 2u)) u.v[3] = (-(u.v[3] / u.v[0])) * u.v[0];
    const Derived<T, D> q = derive(u, gm1);
#pragma unroll
    for (int c = 0; c < NC; ++c) sU[c * G::R + r] = u.v[c];
    sP[r] = q.p;
#pragma unroll
    for (int d = 0; d < D; ++d) sV[d * G::R + r] = q.v[d];
  }
  // lam_out on evolve cells (zero outside the domain along the sweep)
  for (int e = threadIdx.x; e < G::E; e += NT) {
    const int e0 = e % G::E0, e1 = e / G::E0;
    const int64_t g0 = o0 + e0 - (S == 0 ? 2 : 0);
    const int64_t g1 = o1 + e1 - (S == 1 ? 2 : 0);
    const bool in = g0 >= 0 && g0 < n0 && g1 >= 0 && g1 < n1;
#pragma unroll
    for (int c = 0; c < NC; ++c)
      sLam[c * G::E + e] = in ? lo[c * pitch + g1 * n0 + g0] : T(0);
  }
  __syncthreads();

  // ---- B: flattening bases (frozen chi) ---------------------------------
  if (flatten) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      int lo_[2] = {0, 0}, ext[2] = {G::T0, (D >= 2) ? G::T1 : 1};
      lo_[S] = -3;
      ext[S] = G::tile(S) + 6;                 // evolve range [-2, T+1] widened by one
      if (d != S) {
        lo_[d] = -1;
        ext[d] = G::tile(d) + 2;
      }
      const int count = ext[0] * ext[1];
      const int st = G::rstride(d);
      const T* vd = sV + d * G::R;
      for (int i = threadIdx.x; i < count; i += NT) {
        const int c0 = i % ext[0] + lo_[0];
        const int c1 = i / ext[0] + lo_[1];
        const int q = (c1 + G::H1) * G::R0 + (c0 + G::H0);
        sChi[d * G::R + q] = (T)chi_base<T>(sP[q + st], sP[q - st], sP[q + 2 * st],
                                            sP[q - 2 * st], vd[q - st], vd[q + st]);
      }
    }
    __syncthreads();
  }

  // ---- C: forward evolved faces of evolve cells [-2, T+1] ----------------
  constexpr int SS = G::rstride(S);
  for (int e = threadIdx.x; e < G::E; e += NT) {
    const int e0 = e % G::E0, e1 = e / G::E0;
    const int q0 = e0 + G::H0 - (S == 0 ? 2 : 0);
    const int q1 = e1 + G::H1 - (S == 1 ? 2 : 0);
    const int q = q1 * G::R0 + q0;
    Cons<T, D> u, um, up, er, el;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      u.v[c] = sU[c * G::R + q];
      um.v[c] = sU[c * G::R + q - SS];
      up.v[c] = sU[c * G::R + q + SS];
    }
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
    sCv[e] = chi_v;
    if (muscl) {
      evolve_fwd(um, u, up, chi_v, S, gm1, dtdh, er, el);
    } else {
      er = u;
      el = u;
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      sER[c * G::E + e] = er.v[c];
      sEL[c * G::E + e] = el.v[c];
      sERb[c * G::E + e] = T(0);
      sELb[c * G::E + e] = T(0);
    }
  }
  __syncthreads();

  // ---- D: reverse Riemann solve of faces [-1, T+1] -----------------------
  // face index fi (0-based) is tile face f = fi - 1, between cells f-1 and f;
  // in evolve indexing (offset 2) its left cell is fi, its right cell fi + 1.
  constexpr int ES = G::estride(S);
  {
    const int F0 = (S == 0) ? G::T0 + 3 : G::T0;
    const int F1 = (S == 1) ? G::T1 + 3 : G::T1;
    for (int i = threadIdx.x; i < F0 * F1; i += NT) {
      const int f0 = i % F0, f1 = i / F0;
      // evolve index of the face's left cell
      const int el_idx = f1 * G::E0 + f0;
      const int er_idx = el_idx + ES;
      const int64_t gf = oS + ((S == 0) ? f0 : f1) - 1;     // global face index
      if (gf < 0 || gf > nS) continue;                      // ghost faces carry no adjoint
      Cons<T, D> ul, ur, g, bl, br;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        ul.v[c] = sER[c * G::E + el_idx];
        ur.v[c] = sEL[c * G::E + er_idx];
        g.v[c] = dtdh * (sLam[c * G::E + er_idx] - sLam[c * G::E + el_idx]);
        bl.v[c] = T(0);
        br.v[c] = T(0);
      }
      if constexpr (FLUX == kForce)
        riemann_rev<kForce>(ul, ur, S, gamma, gm1, adi, dtdh, g, bl, br);
      else
        riemann_rev<kHllc>(ul, ur, S, gamma, gm1, adi, dtdh, g, bl, br, pinf);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        sERb[c * G::E + el_idx] = bl.v[c];
        sELb[c * G::E + er_idx] = br.v[c];
      }
    }
  }
  __syncthreads();

  // ---- E: reverse evolution of every evolve cell ---------------------------
  // Cells [-1, T] feed the tile's cells; -2 and T+1 matter only next to the
  // domain's ends, where their missing outer face lies outside the domain.
  for (int e = threadIdx.x; e < G::E; e += NT) {
    const int e0 = e % G::E0, e1 = e / G::E0;
    Cons<T, D> dm, d0, dp;
    zero(dm);
    zero(d0);
    zero(dp);
    {
      const int q0 = e0 + G::H0 - (S == 0 ? 2 : 0);
      const int q1 = e1 + G::H1 - (S == 1 ? 2 : 0);
      const int q = q1 * G::R0 + q0;
      Cons<T, D> u, um, up, erb, elb;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        u.v[c] = sU[c * G::R + q];
        um.v[c] = sU[c * G::R + q - SS];
        up.v[c] = sU[c * G::R + q + SS];
        erb.v[c] = sERb[c * G::E + e];
        elb.v[c] = sELb[c * G::E + e];
      }
      if (muscl) {
        evolve_rev(um, u, up, sCv[e], S, gm1, dtdh, erb, elb, dm, d0, dp);
      } else {
#pragma unroll
        for (int c = 0; c < NC; ++c) d0.v[c] = erb.v[c] + elb.v[c];
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      sDm[c * G::E + e] = dm.v[c];
      sD0[c * G::E + e] = d0.v[c];
      sDp[c * G::E + e] = dp.v[c];
    }
  }
  __syncthreads();

  // ---- F: gather lam_in --------------------------------------------------
  const bool refl = (p.reflect >> S) & 1u;
  for (int o = threadIdx.x; o < G::OUT; o += NT) {
    const int t0 = o % G::T0, t1 = o / G::T0;
    const int64_t g0 = o0 + t0, g1 = o1 + t1;
    if (g0 >= n0 || g1 >= n1) continue;
    const int e = (t1 + (S == 1 ? 2 : 0)) * G::E0 + t0 + (S == 0 ? 2 : 0);
    const int64_t gs = (S == 0) ? g0 : g1;
    T r[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c)
      r[c] = sLam[c * G::E + e] + sDp[c * G::E + e - ES] + sD0[c * G::E + e] +
             sDm[c * G::E + e + ES];
    // adjoints of the ghost positions fold back onto the cells they mirror:
    //   ghost -1 (= cell 0):       own part of evolve cell -1 and the left
    //                              neighbour part of evolve cell 0
    //   ghost -2 (= cell 1):       left neighbour part of evolve cell -1
    //   ghost n (= cell n-1):      own part of evolve cell n and the right
    //                              neighbour part of evolve cell n-1
    //   ghost n+1 (= cell n-2):    right neighbour part of evolve cell n
    // (evolve cells -2 and n+1 feed only ghost faces, which carry none).
    // The neighbour parts are non-zero where the limited slope of cell 0 or
    // n-1 takes the difference across the wall: at a reflective end, the
    // normal momentum's 2 m when it is the smaller one-sided difference.
    T m[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) m[c] = T(0);
    if (gs == 0) {
#pragma unroll
      for (int c = 0; c < NC; ++c) m[c] += sD0[c * G::E + e - ES] + sDm[c * G::E + e];
    }
    if (gs == 1) {
#pragma unroll
      for (int c = 0; c < NC; ++c) m[c] += sDm[c * G::E + e - 2 * ES];
    }
    if (gs == nS - 1) {
#pragma unroll
      for (int c = 0; c < NC; ++c) m[c] += sD0[c * G::E + e + ES] + sDp[c * G::E + e];
    }
    if (gs == nS - 2) {
#pragma unroll
      for (int c = 0; c < NC; ++c) m[c] += sDp[c * G::E + e + 2 * ES];
    }
    if (refl) m[2 + S] = -m[2 + S];
    const int64_t gi = g1 * n0 + g0;
#pragma unroll
    for (int c = 0; c < NC; ++c) li[c * pitch + gi] = r[c] + m[c];
  }
}

}  // namespace fl
