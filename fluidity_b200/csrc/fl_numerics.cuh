// fl_numerics.cuh -- per-cell arithmetic of the split-solver step.
//
// Each function restates one of the reference's numerics functors
// (robclu/fluidity include/fluidity/...).  The order of every floating-point
// operation follows the reference expression, so that a build without FMA
// contraction (-fmad=false) reproduces the reference bit for bit and the
// default build differs only by FMA rounding.
//
// States are conservative, component order [rho, E, m_x, (m_y), (m_z)]
// (state/state.hpp:88-98).  NC = D + 2.
#pragma once

#include <cmath>
#include <cstdint>

// Functions are host + device so that the host tests of the adjoint can run
// them on the CPU; kernels use them on the device.
#if defined(__CUDACC__)
#define FL_HD __host__ __device__ __forceinline__
#else
#define FL_HD inline
#endif

namespace fl {

enum FluxKind : int { kHllc = 0, kForce = 1, kLaxFriedrichs = 2, kRichtmyer = 3 };
// Added to a FLUX template argument: the material is the stiffened fluid
// (material/stiff_fluid.hpp:38-133) rather than the ideal gas.
constexpr int kStiffEos = 4;
enum LimiterKind : int { kVanLeer = 0, kSuperbee = 1 };

template <typename T> FL_HD T fl_sqrt(T x);
template <> FL_HD double fl_sqrt<double>(double x) { return std::sqrt(x); }
template <> FL_HD float fl_sqrt<float>(float x) { return std::sqrt(x); }
template <typename T> FL_HD T fl_abs(T x);
template <> FL_HD double fl_abs<double>(double x) { return std::fabs(x); }
template <> FL_HD float fl_abs<float>(float x) { return std::fabs(x); }

// std::min / std::max as the reference's <algorithm> defines them.
template <typename T> FL_HD T std_min(T a, T b) { return (b < a) ? b : a; }
template <typename T> FL_HD T std_max(T a, T b) { return (a < b) ? b : a; }

template <typename T, int D>
struct Cons {
  static constexpr int NC = D + 2;
  T v[NC];
};

// velocity m_d / rho (state_impl.hpp:88-96)
template <typename T, int D>
FL_HD T velocity(const Cons<T, D>& u, int d) {
  return u.v[2 + d] / u.v[0];
}

// (gamma - 1) (E - 0.5 rho sum_d (m_d / rho)^2) (state_impl.hpp:117-128, 49-61)
template <typename T, int D>
FL_HD T pressure(const Cons<T, D>& u, T gamma) {
  T sum = T(0);
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const T v = u.v[2 + d] / u.v[0];
    sum += v * v;
  }
  return (gamma - T(1)) * (u.v[1] - T(0.5) * u.v[0] * sum);
}

// Conservative physical flux in dimension d, given its velocity and pressure
// (state_impl.hpp:293-310, make_other_fluxes 228-244).
template <typename T, int D>
FL_HD void flux_vp(const Cons<T, D>& u, int d, T v, T p,
                                        Cons<T, D>& f) {
  f.v[0] = u.v[2 + d];
  f.v[2 + d] = u.v[2 + d] * v + p;
  f.v[1] = v * (u.v[1] + p);
#pragma unroll
  for (int t = 0; t < D; ++t)
    if (t != d) f.v[2 + t] = u.v[2 + t] * v;
}

template <typename T, int D>
FL_HD void flux(const Cons<T, D>& u, int d, T gamma,
                                     Cons<T, D>& f) {
  flux_vp(u, d, velocity(u, d), pressure(u, gamma), f);
}

// The pressure under the sound speed's root: p for the ideal gas
// (material/ideal_gas.hpp:75-78), p + p_inf for the stiffened fluid
// (material/stiff_fluid.hpp:92-96).  For both materials the state's pressure
// is (gamma - 1)(E - rho |v|^2 / 2) (state_impl.hpp:117-128): the reference
// subtracts no gamma p_inf there, so a stiffened fluid's energy, filled with
// e = (p + gamma p_inf) / ((gamma - 1) rho), reads back as p + gamma p_inf.
template <bool STIFF, typename T>
FL_HD T sound_p(T p, T pinf) {
  if constexpr (STIFF) {
    return p + pinf;
  } else {
    return p;
  }
}

// sqrt(gamma p / rho) (material/ideal_gas.hpp:75-78); the caller passes
// sound_p's pressure
template <typename T, int D>
FL_HD T sound_speed_p(const Cons<T, D>& u, T gamma, T p) {
  return fl_sqrt<T>(gamma * p / u.v[0]);
}

// max_d |u_d| + a (state_impl.hpp:167-178)
template <bool STIFF = false, typename T, int D>
FL_HD T max_wavespeed(const Cons<T, D>& u, T gamma, T pinf = T(0)) {
  T m = fl_abs<T>(velocity(u, 0));
#pragma unroll
  for (int d = 1; d < D; ++d) m = std_max(m, fl_abs<T>(velocity(u, d)));
  return m + sound_speed_p(u, gamma, sound_p<STIFF>(pressure(u, gamma), pinf));
}

// ---- HLLC (flux_method/flux_hllc.hpp:56-245) ---------------------------

template <typename T, int D>
FL_HD void hllc_star(const Cons<T, D>& u, int d, T s, T sstar,
                                          T vel, T p, Cons<T, D>& out) {
  const T sf = s - vel;
  const T scale = sf / (s - sstar);
#pragma unroll
  for (int c = 0; c < D + 2; ++c) out.v[c] = scale * u.v[c];
  out.v[2 + d] = sstar * u.v[0] * scale;
  out.v[1] = scale * (u.v[1] + u.v[0] * (sstar - vel) * (sstar + p / (u.v[0] * sf)));
}

template <bool STIFF = false, typename T, int D>
FL_HD void hllc(const Cons<T, D>& ul, const Cons<T, D>& ur, int d,
                                     T gamma, Cons<T, D>& f, T pinf = T(0)) {
  const T pl = pressure(ul, gamma), pr = pressure(ur, gamma);
  const T vl = velocity(ul, d), vr = velocity(ur, d);
  const T al = sound_speed_p(ul, gamma, sound_p<STIFF>(pl, pinf));
  const T ar = sound_speed_p(ur, gamma, sound_p<STIFF>(pr, pinf));
  const T adi = (gamma + T(1)) / (T(2) * gamma);
  const T p_pvrs = T(0.5) * ((pl + pr) - (T(0.25) * (vr - vl) * (ur.v[0] + ul.v[0]) * (al + ar)));
  const T p_star = std_max(T(0), p_pvrs);
  // wavespeed(): rarefaction if p* <= p_K, else shock (flux_hllc.hpp:81-99)
  const T wsl = (p_star <= pl) ? vl + (-al)
                               : vl + (-al) * fl_sqrt<T>(T(1) + adi * (p_star / pl - T(1)));
  if (T(0) <= wsl) { flux_vp(ul, d, vl, pl, f); return; }
  const T wsr = (p_star <= pr) ? vr + ar
                               : vr + ar * fl_sqrt<T>(T(1) + adi * (p_star / pr - T(1)));
  if (T(0) >= wsr) { flux_vp(ur, d, vr, pr, f); return; }
  // star_speed (flux_hllc.hpp:113-137)
  const T factl = ul.v[0] * (wsl - vl);
  const T factr = ur.v[0] * (wsr - vr);
  const T sstar = (pr - pl + vl * factl - vr * factr) / (factl - factr);
  Cons<T, D> st;
  if (T(0) <= sstar) {
    flux_vp(ul, d, vl, pl, f);
    hllc_star(ul, d, wsl, sstar, vl, pl, st);
#pragma unroll
    for (int c = 0; c < D + 2; ++c) f.v[c] = f.v[c] + wsl * (st.v[c] - ul.v[c]);
  } else {
    flux_vp(ur, d, vr, pr, f);
    hllc_star(ur, d, wsr, sstar, vr, pr, st);
#pragma unroll
    for (int c = 0; c < D + 2; ++c) f.v[c] = f.v[c] + wsr * (st.v[c] - ur.v[c]);
  }
}

// ---- FORCE = (LF + Richtmyer) / 2 (flux_force.hpp:73-84) ----------------

template <typename T, int D>
FL_HD void lax_friedrichs_ff(const Cons<T, D>& ul, const Cons<T, D>& ur,
                                                  const Cons<T, D>& fl, const Cons<T, D>& fr,
                                                  T dtdh, Cons<T, D>& f) {
  // flux_lax_friedrichs.hpp:63-78; dhdt = 1 / dtdh
  const T dhdt = T(1.0) / dtdh;
#pragma unroll
  for (int c = 0; c < D + 2; ++c)
    f.v[c] = T(0.5) * (fl.v[c] + fr.v[c] + dhdt * (ul.v[c] - ur.v[c]));
}

template <typename T, int D>
FL_HD void richtmyer_ff(const Cons<T, D>& ul, const Cons<T, D>& ur,
                                             const Cons<T, D>& fl, const Cons<T, D>& fr,
                                             int d, T gamma, T dtdh, Cons<T, D>& f) {
  // flux_richtmyer.hpp:78-88
  Cons<T, D> u;
#pragma unroll
  for (int c = 0; c < D + 2; ++c)
    u.v[c] = T(0.5) * (ul.v[c] + ur.v[c] + dtdh * (fl.v[c] - fr.v[c]));
  flux(u, d, gamma, f);
}

// FLUX: a FluxKind, plus kStiffEos for the stiffened fluid's sound speed
// (which only HLLC uses; p_inf is ignored otherwise).
template <int FLUX, typename T, int D>
FL_HD void riemann(const Cons<T, D>& ul, const Cons<T, D>& ur, int d,
                                        T gamma, T dtdh, Cons<T, D>& f, T pinf = T(0)) {
  constexpr int RS = FLUX & 3;
  if constexpr (RS == kHllc) {
    hllc<(FLUX & kStiffEos) != 0>(ul, ur, d, gamma, f, pinf);
  } else {
    Cons<T, D> fl, fr;
    flux(ul, d, gamma, fl);
    flux(ur, d, gamma, fr);
    if constexpr (RS == kLaxFriedrichs) {
      lax_friedrichs_ff(ul, ur, fl, fr, dtdh, f);
    } else if constexpr (RS == kRichtmyer) {
      richtmyer_ff(ul, ur, fl, fr, d, gamma, dtdh, f);
    } else {
      Cons<T, D> a, b;
      lax_friedrichs_ff(ul, ur, fl, fr, dtdh, a);
      richtmyer_ff(ul, ur, fl, fr, d, gamma, dtdh, b);
#pragma unroll
      for (int c = 0; c < D + 2; ++c) f.v[c] = T(0.5) * (a.v[c] + b.v[c]);
    }
  }
}

// ---- limiters (limiting/van_leer_limiter.hpp:65-74, superbee 72-89) -----

template <typename T>
FL_HD T limit_single(int limiter, T left, T right) {
  const T r = left / right;
  if (limiter == kSuperbee) {
    if (r <= T(0) || right == T(0)) return T(0);
    if (r <= T(0.5)) return T(2) * r;
    if (r <= T(1)) return T(1);
    const T er = T(2) / (T(1) + r);
    return std_min(er, std_min(r, T(2)));
  }
  return (r <= T(0) || right == T(0)) ? T(0) : T(2) * std_min(r, T(1)) / (T(1) + r);
}

// FL_FAST_DIV 1 (the default): the HLLC star speed, star scale, energy
// term and shock pressure ratios multiply by one reciprocal instead of
// dividing, and the flattening threshold test compares a product; results
// differ from the divisions by rounding (measured 2.6% faster in the FP64
// sweep before the shock ratios joined).
#ifndef FL_FAST_DIV
#define FL_FAST_DIV 1
#endif
// FL_CHI_FAST 1 (the default): the flattening ratio z and its ramp multiply
// by reciprocals (the ramp's a compile-time constant) instead of dividing: a
// rounding-level change that takes the divisions' inlined code out of every
// sweep's loop body (+1.6% on the FP64 staged sweep, +3.3% on the FP32 one,
// +4.6% on the batched kernel).
#ifndef FL_CHI_FAST
#define FL_CHI_FAST 1
#endif

// ---- fast forms used by the sweep kernel ---------------------------------
// One reciprocal per state replaces the reference's one division per
// velocity (m_d / rho -> m_d * (1 / rho)); every other expression keeps the
// reference's order.  The results differ from the reference by rounding only
// (a few ulp), well inside the 1e-12 (FP64) / 1e-5 (FP32) per-step bars.

// FL_FAST_F32 1 (the default): in FP32 the kernels' reciprocal and square
// root use the hardware approximations (PTX rcp.approx.f32 / sqrt.approx.f32,
// about one ulp) and the flattening test runs in float; FP64 is unaffected.
// Measured +12% (HLLC) and +8% (FORCE) on the FP32 sweep, within the FP32
// parity bar.
#ifndef FL_FAST_F32
#define FL_FAST_F32 1
#endif

// FL_FAST_F64 1: the FP64 reciprocal and square root of the fast forms start
// from the hardware approximations (PTX rcp.approx.ftz.f64, rsqrt.approx.f64,
// good to about 2^-22) and refine them with one third-order Householder step
// each, which triples the correct bits (to beyond 2^-60 before rounding):
//   1/x:       e = 1 - x y,      y <- y + y (e + e^2);
//   1/sqrt(x): h = 1 - x r^2,    r <- r + r h (1/2 + 3h/8),
// then s = x r and one Heron correction s <- s + (r/2)(x - s^2); accurate
// to about an ulp.  Two Newton steps (y <- y + y (1 - x y), twice) reach the
// same accuracy with one more dependent multiply-add per reciprocal; the
// kernels evaluate about nine reciprocals and three roots per cell.
#ifndef FL_FAST_F64
#define FL_FAST_F64 1
#endif

template <typename T> FL_HD T fl_rcp(T x);
#if defined(__CUDA_ARCH__)
#if FL_FAST_F64
template <> FL_HD double fl_rcp<double>(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
}
#else
template <> FL_HD double fl_rcp<double>(double x) { return __drcp_rn(x); }
#endif
#if FL_FAST_F32
template <> FL_HD float fl_rcp<float>(float x) {
  float r;
  asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
#else
template <> FL_HD float fl_rcp<float>(float x) { return __frcp_rn(x); }
#endif
#else
template <> FL_HD double fl_rcp<double>(double x) { return 1.0 / x; }
template <> FL_HD float fl_rcp<float>(float x) { return 1.0f / x; }
#endif

// Square root of the fast forms (the reference-order forms keep fl_sqrt).
template <typename T> FL_HD T fl_ksqrt(T x) { return fl_sqrt<T>(x); }
#if defined(__CUDA_ARCH__) && FL_FAST_F64
template <> FL_HD double fl_ksqrt<double>(double x) {
  // refine for a positive stand-in and select: sqrt(+-0) = +-0, and a
  // negative or NaN argument gives NaN.  No branch to the library's root,
  // whose inlined code sat at each of the sweep loop's five call sites
  // (+1.2% on the FP64 staged sweep).
  const double xs = (x > 0.0) ? x : 1.0;
  double r;
  asm("rsqrt.approx.f64 %0, %1;" : "=d"(r) : "d"(xs));
  const double h = fma(-(xs * r), r, 1.0);
  r = fma(r * h, fma(h, 0.375, 0.5), r);
  const double sq = xs * r;
  const double s = fma(0.5 * r, fma(-sq, sq, xs), sq);
  return (x > 0.0) ? s : ((x == 0.0) ? x : __longlong_as_double(0x7ff8000000000000ll));
}
#endif
#if defined(__CUDA_ARCH__) && FL_FAST_F32
template <> FL_HD float fl_ksqrt<float>(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
#endif

// ---- flattening (reconstruction/muscl_reconstructor.hpp:59-87) ----------
// Inputs: pressures at c+1, c-1, c+2, c-2 and velocities (sweep of chi's own
// dimension) at c-1, c+1.  Ratio in T; sigma test and eta in double.

template <typename T>
FL_HD double chi_base(T p_next, T p_prev, T p_nnext, T p_pprev,
                                           T u_prev, T u_next) {
  const T u_factor = u_prev - u_next;
  const T dp = fl_abs<T>(p_next - p_prev);
#if FL_FAST_DIV
  // the ratio test as a product: differs from the division only where
  // dp / min(p) is within an ulp of 0.33
#if FL_FAST_F32
  const bool flatten = sizeof(T) == 4
                           ? (u_factor > T(0) && dp > T(0.33) * std_min(p_next, p_prev))
                           : ((double)u_factor > 0.0 &&
                              (double)dp > 0.33 * (double)std_min(p_next, p_prev));
#else
  const bool flatten = ((double)u_factor > 0.0) &&
                       ((double)dp > 0.33 * (double)std_min(p_next, p_prev));
#endif
#else
  const bool flatten = ((double)u_factor > 0.0) && ((double)(dp / std_min(p_next, p_prev)) > 0.33);
#endif
  if (!flatten) return 1.0;
#if FL_CHI_FAST
  constexpr double kInvRamp = 1.0 / (0.85 - 0.75);
  const T z = dp * fl_rcp<T>(fl_abs<T>(p_nnext - p_pprev));
  const double temp = 1.0 - (((double)z - 0.75) * kInvRamp);
#else
  const T z = dp / fl_abs<T>(p_nnext - p_pprev);
  const double temp = 1.0 - (((double)z - 0.75) / (0.85 - 0.75));
#endif
  return std_min(1.0, std_max(0.0, temp));
}


// Primitive quantities derived from a conservative state.
template <typename T, int D>
struct Derived {
  T rinv;   // 1 / rho
  T v[D];   // velocities
  T p;      // pressure
};

template <typename T, int D>
FL_HD Derived<T, D> derive(const Cons<T, D>& u, T gm1) {
  Derived<T, D> q;
  q.rinv = fl_rcp<T>(u.v[0]);
  T sum = T(0);
#pragma unroll
  for (int d = 0; d < D; ++d) {
    q.v[d] = u.v[2 + d] * q.rinv;
    sum += q.v[d] * q.v[d];
  }
  q.p = gm1 * (u.v[1] - T(0.5) * u.v[0] * sum);
  return q;
}

template <typename T, int D>
FL_HD void flux_q(const Cons<T, D>& u, const Derived<T, D>& q, int d,
                                       Cons<T, D>& f) {
  flux_vp(u, d, q.v[d], q.p, f);
}

// max_d |u_d| + sqrt(gamma p / rho); p + p_inf under the root when STIFF
template <bool STIFF = false, typename T, int D>
FL_HD T max_wavespeed_q(const Derived<T, D>& q, T gamma, T pinf = T(0)) {
  T m = fl_abs<T>(q.v[0]);
#pragma unroll
  for (int d = 1; d < D; ++d) m = std_max(m, fl_abs<T>(q.v[d]));
  return m + fl_ksqrt<T>(gamma * sound_p<STIFF>(q.p, pinf) * q.rinv);
}

// HLLC with precomputed side quantities; adi = (gamma + 1) / (2 gamma).
template <bool STIFF = false, typename T, int D>
FL_HD void hllc_q(const Cons<T, D>& ul, const Derived<T, D>& ql,
                                       const Cons<T, D>& ur, const Derived<T, D>& qr, int d,
                                       T gamma, T adi, Cons<T, D>& f, T pinf = T(0)) {
  const T pl = ql.p, pr = qr.p, vl = ql.v[d], vr = qr.v[d];
  const T al = fl_ksqrt<T>(gamma * sound_p<STIFF>(pl, pinf) * ql.rinv);
  const T ar = fl_ksqrt<T>(gamma * sound_p<STIFF>(pr, pinf) * qr.rinv);
  const T p_pvrs = T(0.5) * ((pl + pr) - (T(0.25) * (vr - vl) * (ur.v[0] + ul.v[0]) * (al + ar)));
  const T p_star = std_max(T(0), p_pvrs);
#if FL_FAST_DIV
  // the shock speeds' pressure ratios by reciprocal (rounding-level change)
  const T wsl = (p_star <= pl)
                    ? vl + (-al)
                    : vl + (-al) * fl_ksqrt<T>(T(1) + adi * (p_star * fl_rcp<T>(pl) - T(1)));
  if (T(0) <= wsl) { flux_vp(ul, d, vl, pl, f); return; }
  const T wsr = (p_star <= pr)
                    ? vr + ar
                    : vr + ar * fl_ksqrt<T>(T(1) + adi * (p_star * fl_rcp<T>(pr) - T(1)));
#else
  const T wsl = (p_star <= pl) ? vl + (-al)
                               : vl + (-al) * fl_ksqrt<T>(T(1) + adi * (p_star / pl - T(1)));
  if (T(0) <= wsl) { flux_vp(ul, d, vl, pl, f); return; }
  const T wsr = (p_star <= pr) ? vr + ar
                               : vr + ar * fl_ksqrt<T>(T(1) + adi * (p_star / pr - T(1)));
#endif
  if (T(0) >= wsr) { flux_vp(ur, d, vr, pr, f); return; }
  const T factl = ul.v[0] * (wsl - vl);
  const T factr = ur.v[0] * (wsr - vr);
#if FL_FAST_DIV
  const T sstar = (pr - pl + vl * factl - vr * factr) * fl_rcp<T>(factl - factr);
#else
  const T sstar = (pr - pl + vl * factl - vr * factr) / (factl - factr);
#endif
  // star state (flux_hllc.hpp:150-188) folded into F_K + S_K (U*_K - U_K)
  const bool left = T(0) <= sstar;
  const Cons<T, D>& u = left ? ul : ur;
  const T s = left ? wsl : wsr;
  const T vel = left ? vl : vr;
  const T p = left ? pl : pr;
  const T sf = s - vel;
#if FL_FAST_DIV
  const T scale = sf * fl_rcp<T>(s - sstar);
  const T p_rsf = p * fl_rcp<T>(u.v[0] * sf);
#else
  const T scale = sf / (s - sstar);
  const T p_rsf = p / (u.v[0] * sf);
#endif
  flux_vp(u, d, vel, p, f);
  Cons<T, D> st;
#pragma unroll
  for (int c = 0; c < D + 2; ++c) st.v[c] = scale * u.v[c];
  st.v[2 + d] = sstar * u.v[0] * scale;
  st.v[1] = scale * (u.v[1] + u.v[0] * (sstar - vel) * (sstar + p_rsf));
#pragma unroll
  for (int c = 0; c < D + 2; ++c) f.v[c] = f.v[c] + s * (st.v[c] - u.v[c]);
}

// FLUX as for riemann.  dhdt = 1 / dtdh, the Lax-Friedrichs coefficient
// (flux_lax_friedrichs.hpp:63-78), given by a caller that computes it once.
template <int FLUX, typename T, int D>
FL_HD void riemann_qh(const Cons<T, D>& ul, const Derived<T, D>& ql,
                                           const Cons<T, D>& ur, const Derived<T, D>& qr, int d,
                                           T gamma, T gm1, T adi, T dtdh, T dhdt, Cons<T, D>& f,
                                           T pinf = T(0)) {
  constexpr int RS = FLUX & 3;
  if constexpr (RS == kHllc) {
    hllc_q<(FLUX & kStiffEos) != 0>(ul, ql, ur, qr, d, gamma, adi, f, pinf);
  } else {
    Cons<T, D> fl, fr;
    flux_q(ul, ql, d, fl);
    flux_q(ur, qr, d, fr);
    Cons<T, D> lf, ri;
    if constexpr (RS != kRichtmyer) {
#pragma unroll
      for (int c = 0; c < D + 2; ++c)
        lf.v[c] = T(0.5) * (fl.v[c] + fr.v[c] + dhdt * (ul.v[c] - ur.v[c]));
    }
    if constexpr (RS != kLaxFriedrichs) {
      Cons<T, D> m;
#pragma unroll
      for (int c = 0; c < D + 2; ++c)
        m.v[c] = T(0.5) * (ul.v[c] + ur.v[c] + dtdh * (fl.v[c] - fr.v[c]));
      flux_q(m, derive(m, gm1), d, ri);
    }
    if constexpr (RS == kLaxFriedrichs) {
      f = lf;
    } else if constexpr (RS == kRichtmyer) {
      f = ri;
    } else {
#pragma unroll
      for (int c = 0; c < D + 2; ++c) f.v[c] = T(0.5) * (lf.v[c] + ri.v[c]);
    }
  }
}

template <int FLUX, typename T, int D>
FL_HD void riemann_q(const Cons<T, D>& ul, const Derived<T, D>& ql,
                                          const Cons<T, D>& ur, const Derived<T, D>& qr, int d,
                                          T gamma, T gm1, T adi, T dtdh, Cons<T, D>& f,
                                          T pinf = T(0)) {
  riemann_qh<FLUX>(ul, ql, ur, qr, d, gamma, gm1, adi, dtdh, T(1.0) / dtdh, f, pinf);
}

// The reference's van Leer slope 0.5 (bd + fd) * 2 min(r, 1) / (1 + r) with
// r = bd / fd equals, in exact arithmetic, minmod(bd, fd): bd when
// 0 < r <= 1, fd when r > 1, 0 when r <= 0 or fd == 0.  Superbee keeps the
// reference's formula.
template <typename T>
FL_HD T limited_slope(int limiter, T bd, T fd) {
  if (limiter == kSuperbee) {
    T lim = T(0.5) * (bd + fd);
    return lim * limit_single<T>(kSuperbee, bd, fd);
  }
  const bool same = (bd > T(0) && fd > T(0)) || (bd < T(0) && fd < T(0));
  if (!same) return T(0);
  return (fl_abs<T>(bd) <= fl_abs<T>(fd)) ? bd : fd;
}

}  // namespace fl
