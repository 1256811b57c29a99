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
// reflective end).  The wave/limiter branches are frozen (see
// fl_adjoint.cuh), so lines along the sweep are independent, except for
// the flattening coefficient chi.  chi_v(e) = min over dimensions of
// min(chi_d(e), chi_d(e + sign e_d)) is differentiated through the one
// chi_d(c*) the minimum selects, where that one lies on its ramp
// eta = 1 - (z - 0.75) / 0.1, z = |p(c*+1) - p(c*-1)| / |p(c*+2) - p(c*-2)|
// along d (muscl_reconstructor.hpp:59-111); its clamps, the flattening test
// and the selection are frozen.  Those four pressures can lie on other
// lines, so each evolve cell leaves a record (which chi_d it selected, and
// dL/dchi dchi/dz), and a second kernel gathers per cell, in a fixed order,
// the records whose stencils read its pressure, and adds them to lam_in
// through dp/dU: no atomics, the same result on every run.  Tile: T_S cells
// along the sweep, halo 5 along it (the forward faces of evolve cells
// [-2, T_S+1]), 3 across.
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
  // nullable: the chi records, one per evolve cell of every line
  // ((n_S + 2) * lines, evolve cells -1 .. n_S along the sweep): chi_gz the
  // sweep's dtype, chi_epoch the sweep that wrote the record, chi_sel the
  // selection byte; a record counts only in the sweep chi_epoch names.
  // chi_flag[chi_epoch & 1] is set when the sweep wrote any record, and the
  // gather clears the other word for the next sweep.  Without records chi
  // is frozen.
  void* chi_gz;
  unsigned int* chi_epoch_of;
  unsigned char* chi_sel;
  unsigned int* chi_flag;
  unsigned int chi_epoch;
};

// Index of evolve cell (along the sweep eS in [-1, nS], across eA) in the
// chi records.
__host__ __device__ __forceinline__ int64_t chi_rec(int64_t eS, int64_t eA, int64_t nS) {
  return eA * (nS + 2) + (eS + 1);
}

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
  // plus one byte per evolve cell: which chi_d the minimum selected
  static constexpr size_t smem_bytes = sizeof(T) * smem_elems + E + 64;
  __host__ __device__ static constexpr int rstride(int d) { return d == 0 ? 1 : R0; }
  __host__ __device__ static constexpr int estride(int d) { return d == 0 ? 1 : E0; }
  __host__ __device__ static constexpr int tile(int d) { return d == 0 ? T0 : T1; }
};

// dchi/dz on the ramp eta = 1 - (z - 0.75) / (0.85 - 0.75)
template <typename T>
__host__ __device__ constexpr T chi_dz() { return T(-1.0 / (0.85 - 0.75)); }

// Pressure of the state at global position (x0, x1), mirrored into the
// domain (a reflective flip changes no pressure).
template <typename T, int D>
__device__ __forceinline__ T adj_pressure_at(const T* u_in, int64_t pitch, int64_t n0, int64_t n1,
                                             int64_t x0, int64_t x1, T gm1) {
  bool f;
  const int64_t g0 = mirror_index(x0, n0, f);
  const int64_t g1 = (D >= 2) ? mirror_index(x1, n1, f) : 0;
  const int64_t gi = g1 * n0 + g0;
  Cons<T, D> u;
#pragma unroll
  for (int c = 0; c < D + 2; ++c) u.v[c] = u_in[c * pitch + gi];
  return derive(u, gm1).p;
}

// Positions that mirror onto cell c of an extent-n dimension within 4
// cells of the domain: c, and its images -1 - c and 2n - 1 - c.
__device__ __forceinline__ int chi_images(int64_t c, int64_t n, int64_t* x) {
  int k = 0;
  x[k++] = c;
  if (-1 - c >= -4) x[k++] = -1 - c;
  if (2 * n - 1 - c <= n + 3) x[k++] = 2 * n - 1 - c;
  return k;
}

// The chi terms: per cell c, the pressure adjoint gathered from every evolve
// cell whose selected chi_d(c*) reads a position x that mirrors onto c
// (x = c* + o e_d, o = +-1, +-2), then lam_in(c) += lam_p dp/dU(c).
template <typename T, int D, int S>
__global__ void adj_chi_gather_kernel(const T* __restrict__ u_in, const T* __restrict__ gz,
                                      const unsigned int* __restrict__ epoch_of,
                                      const unsigned char* __restrict__ sel,
                                      unsigned int* __restrict__ flag, unsigned int epoch,
                                      T* __restrict__ lam_in, int64_t pitch, int64_t n0,
                                      int64_t n1, T gm1) {
  // the next sweep's flag word is free: this sweep's main kernel is done
  // with it and the next one has not started
  if (blockIdx.x == 0 && threadIdx.x == 0) flag[(epoch + 1u) & 1u] = 0u;
  if (*(volatile unsigned int*)(flag + (epoch & 1u)) == 0u) return;  // no chi terms
  const int64_t nS = (S == 0) ? n0 : n1;
  const int64_t nA = (D >= 2) ? ((S == 0) ? n1 : n0) : 1;
  const int64_t cells = n0 * ((D >= 2) ? n1 : 1);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c0 = i % n0, c1 = (D >= 2) ? i / n0 : 0;
    int64_t xs0[3], xs1[3];
    const int k0 = chi_images(c0, n0, xs0);
    int k1 = 1;
    xs1[0] = 0;
    if (D >= 2) k1 = chi_images(c1, n1, xs1);
    T lp = T(0);
    for (int ia = 0; ia < k0; ++ia)
      for (int ib = 0; ib < k1; ++ib)
        for (int d = 0; d < D; ++d) {
          const int64_t s0 = (d == 0) ? 1 : 0, s1 = (d == 1) ? 1 : 0;
          for (int oi = 0; oi < 4; ++oi) {
            const int o = (oi == 0) ? 1 : (oi == 1) ? -1 : (oi == 2) ? 2 : -2;
            const int64_t q0 = xs0[ia] - o * s0, q1 = xs1[ib] - o * s1;   // c*
            for (int si = 0; si < 3; ++si) {
              const int side = si - 1;
              const int64_t e0 = q0 - side * s0, e1 = q1 - side * s1;
              const int64_t eS = (S == 0) ? e0 : e1, eA = (S == 0) ? e1 : e0;
              if (eS < -1 || eS > nS || eA < 0 || eA >= nA) continue;
              const int64_t r = chi_rec(eS, eA, nS);
              if (epoch_of[r] != epoch || sel[r] != d * 3 + si) continue;
              const T pp1 = adj_pressure_at<T, D>(u_in, pitch, n0, n1, q0 + s0, q1 + s1, gm1);
              const T pm1 = adj_pressure_at<T, D>(u_in, pitch, n0, n1, q0 - s0, q1 - s1, gm1);
              const T pp2 = adj_pressure_at<T, D>(u_in, pitch, n0, n1, q0 + 2 * s0,
                                                  q1 + 2 * s1, gm1);
              const T pm2 = adj_pressure_at<T, D>(u_in, pitch, n0, n1, q0 - 2 * s0,
                                                  q1 - 2 * s1, gm1);
              const T a = pp1 - pm1, b = pp2 - pm2;
              const T ab = fl_abs<T>(b);
              const T sa = (a < T(0)) ? T(-1) : T(1), sb = (b < T(0)) ? T(-1) : T(1);
              T dzdp;  // dz / dp(x), z = |a| / |b|
              if (o == 1) dzdp = sa / ab;
              else if (o == -1) dzdp = -sa / ab;
              else if (o == 2) dzdp = -(fl_abs<T>(a) / ab) * sb / ab;
              else dzdp = (fl_abs<T>(a) / ab) * sb / ab;
              lp += gz[r] * dzdp;
            }
          }
        }
    if (lp == T(0)) continue;
    Cons<T, D> u, ub;
#pragma unroll
    for (int c = 0; c < D + 2; ++c) {
      u.v[c] = u_in[c * pitch + i];
      ub.v[c] = T(0);
    }
    DerivedBar<T, D> qb = zero_bar<T, D>();
    qb.p = lp;
    derive_rev(u, derive(u, gm1), gm1, qb, ub);
#pragma unroll
    for (int c = 0; c < D + 2; ++c) lam_in[c * pitch + i] += ub.v[c];
  }
}

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
  // chi selection per evolve cell: 255 = no derivative, else
  // d * 3 + (side + 1) with chi_d taken at e + side e_d
  unsigned char* sSel = reinterpret_cast<unsigned char*>(sLam + NC * G::E);
  const bool chi_diff = flatten && p.chi_gz != nullptr;

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
    int sel = 255;
    if (flatten) {
      chi_v = (sizeof(T) == 8) ? (T)DBL_MAX : (T)FLT_MAX;
#pragma unroll
      for (int d = 0; d < D; ++d) {
        const int st = G::rstride(d);
        const T diff = sP[q + st] - sP[q - st];
        const int sign = (T(0) < diff) - (diff < T(0));
        const T* cd = sChi + d * G::R;
        // std_min(a, b) keeps a unless b < a: the same choice recorded
        const T c0 = cd[q], c1 = cd[q + sign * st];
        const bool nb = c1 < c0;
        const T m = nb ? c1 : c0;
        if (m < chi_v) {
          chi_v = m;
          sel = d * 3 + (nb ? sign : 0) + 1;
        }
      }
      // on the ramp only: the clamps and an unflattened 1 carry no derivative
      if (!(chi_v > T(0) && chi_v < T(1))) sel = 255;
    }
    sCv[e] = chi_v;
    sSel[e] = (unsigned char)sel;
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
        T dchi;
        evolve_rev(um, u, up, sCv[e], S, gm1, dtdh, erb, elb, dm, d0, dp, dchi);
        if (chi_diff) {
          // records of the evolve cells owned here: the tile's cells, and
          // the ghost evolve cells -1 and nS at the domain's ends (nS in the
          // tile of cell nS - 1 only); -2 and nS + 1 feed ghost faces only
          const int es = (S == 0) ? e0 : e1;
          const int64_t ge0 = o0 + e0 - (S == 0 ? 2 : 0);
          const int64_t ge1 = o1 + e1 - (S == 1 ? 2 : 0);
          const int64_t gs = (S == 0) ? ge0 : ge1;
          const int64_t ga = (S == 0) ? ge1 : ge0;
          const int64_t na = (D >= 2) ? ((S == 0) ? n1 : n0) : 1;
          const bool own = ((es >= 2 && es < 2 + G::tile(S) && gs < nS) || gs == -1 ||
                            (gs == nS && oS <= nS - 1 && nS - 1 < oS + G::tile(S))) &&
                           ga < na;
          if (own && sSel[e] != 255 && dchi != T(0)) {
            const int64_t r = chi_rec(gs, ga, nS);
            static_cast<T*>(p.chi_gz)[r] = dchi * chi_dz<T>();
            p.chi_sel[r] = sSel[e];
            p.chi_epoch_of[r] = p.chi_epoch;
            p.chi_flag[p.chi_epoch & 1u] = 1u;
          }
        }
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
