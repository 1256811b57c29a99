// fl_adjoint.cuh -- hand-written reverse mode of the split-solver arithmetic.
//
// No reference counterpart: the reference has no differentiation.  Each
// function below is the exact reverse (vector-Jacobian product) of the
// forward function of the same name in fl_numerics.cuh, with every branch
// taken as the forward pass takes it: the HLLC wave region and shock /
// rarefaction choice, the max(0, p_pvrs) clamp and the minmod (van Leer)
// selection are frozen at the forward values.  evolve_rev returns the
// adjoint of the flattening coefficient chi; the sweep kernel carries it on
// through chi's ramp (fl_adjoint_sweep.cuh).  Functions are host + device so
// that tests/cpp/adjoint_fd.cpp can check them against finite differences on
// the CPU.
#pragma once

#include "fl_numerics.cuh"

namespace fl {

// Adjoints of the derived quantities of one state.
template <typename T, int D>
struct DerivedBar {
  T r;      // d/d(1/rho)
  T v[D];   // d/d(velocity)
  T p;      // d/d(pressure)
};

template <typename T, int D>
FL_HD DerivedBar<T, D> zero_bar() {
  DerivedBar<T, D> b;
  b.r = T(0);
  b.p = T(0);
#pragma unroll
  for (int d = 0; d < D; ++d) b.v[d] = T(0);
  return b;
}

template <typename T, int D>
FL_HD void zero(Cons<T, D>& u) {
#pragma unroll
  for (int c = 0; c < D + 2; ++c) u.v[c] = T(0);
}

// derive(): r = 1/rho, v_d = m_d r, p = gm1 (E - 0.5 rho sum v^2).
template <typename T, int D>
FL_HD void derive_rev(const Cons<T, D>& u, const Derived<T, D>& q, T gm1,
                      const DerivedBar<T, D>& qb, Cons<T, D>& ub) {
  T sum = T(0);
#pragma unroll
  for (int d = 0; d < D; ++d) sum += q.v[d] * q.v[d];
  ub.v[1] += gm1 * qb.p;
  ub.v[0] += T(-0.5) * gm1 * qb.p * sum;
  const T sbar = T(-0.5) * gm1 * qb.p * u.v[0];
  T rbar = qb.r;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const T vb = qb.v[d] + T(2) * q.v[d] * sbar;
    ub.v[2 + d] += vb * q.rinv;
    rbar += vb * u.v[2 + d];
  }
  ub.v[0] += -rbar * q.rinv * q.rinv;
}

// flux_vp() in dimension d with v = q.v[d], p = q.p: accumulates into the
// state adjoint ub directly and into qb for v, p.
template <typename T, int D>
FL_HD void flux_rev_partial(const Cons<T, D>& u, const Derived<T, D>& q, int d,
                            const Cons<T, D>& fb, Cons<T, D>& ub, DerivedBar<T, D>& qb) {
  const T v = q.v[d], p = q.p;
  T vb = fb.v[2 + d] * u.v[2 + d] + fb.v[1] * (u.v[1] + p);
  ub.v[2 + d] += fb.v[0] + fb.v[2 + d] * v;
  qb.p += fb.v[2 + d] + fb.v[1] * v;
  ub.v[1] += fb.v[1] * v;
#pragma unroll
  for (int t = 0; t < D; ++t) {
    if (t == d) continue;
    vb += fb.v[2 + t] * u.v[2 + t];
    ub.v[2 + t] += fb.v[2 + t] * v;
  }
  qb.v[d] += vb;
}

// Full reverse of flux_q(u, derive(u), d): ub += J^T fb.
template <typename T, int D>
FL_HD void flux_rev(const Cons<T, D>& u, const Derived<T, D>& q, int d, T gm1,
                    const Cons<T, D>& fb, Cons<T, D>& ub) {
  DerivedBar<T, D> qb = zero_bar<T, D>();
  flux_rev_partial(u, q, d, fb, ub, qb);
  derive_rev(u, q, gm1, qb, ub);
}

// Reverse of hllc_q (fl_numerics.cuh): given the flux adjoint g, accumulate
// the adjoints of the left and right states.
template <typename T, int D>
FL_HD void hllc_rev(const Cons<T, D>& ul, const Derived<T, D>& ql, const Cons<T, D>& ur,
                    const Derived<T, D>& qr, int d, T gamma, T gm1, T adi, const Cons<T, D>& g,
                    Cons<T, D>& ubl, Cons<T, D>& ubr, T pinf = T(0)) {
  const T pl = ql.p, pr = qr.p, vl = ql.v[d], vr = qr.v[d];
  // sound speeds from p + p_inf (p_inf = 0: the ideal gas)
  const T al = fl_sqrt<T>(gamma * (pl + pinf) * ql.rinv);
  const T ar = fl_sqrt<T>(gamma * (pr + pinf) * qr.rinv);
  const T A1 = vr - vl, A2 = ur.v[0] + ul.v[0], A3 = al + ar;
  const T p_pvrs = T(0.5) * ((pl + pr) - (T(0.25) * A1 * A2 * A3));
  const T p_star = std_max(T(0), p_pvrs);
  const bool shock_l = !(p_star <= pl);
  const bool shock_r = !(p_star <= pr);
  const T Rl = p_star / pl, Rr = p_star / pr;
  const T qlv = shock_l ? fl_sqrt<T>(T(1) + adi * (Rl - T(1))) : T(1);
  const T qrv = shock_r ? fl_sqrt<T>(T(1) + adi * (Rr - T(1))) : T(1);
  const T wsl = vl + (-al) * qlv;
  DerivedBar<T, D> bl = zero_bar<T, D>(), br = zero_bar<T, D>();
  if (T(0) <= wsl) {
    flux_rev_partial(ul, ql, d, g, ubl, bl);
    derive_rev(ul, ql, gm1, bl, ubl);
    return;
  }
  const T wsr = vr + ar * qrv;
  if (T(0) >= wsr) {
    flux_rev_partial(ur, qr, d, g, ubr, br);
    derive_rev(ur, qr, gm1, br, ubr);
    return;
  }
  const T factl = ul.v[0] * (wsl - vl);
  const T factr = ur.v[0] * (wsr - vr);
  const T N = pr - pl + vl * factl - vr * factr;
  const T Dn = factl - factr;
  const T sstar = N / Dn;
  const bool left = T(0) <= sstar;
  const Cons<T, D>& u = left ? ul : ur;
  const Derived<T, D>& q = left ? ql : qr;
  Cons<T, D>& ub = left ? ubl : ubr;
  DerivedBar<T, D>& bk = left ? bl : br;
  const T S = left ? wsl : wsr;
  const T v = q.v[d], p = q.p, rho = u.v[0];
  const T sf = S - v;
  const T Z = S - sstar;
  const T sc = sf / Z;
  const T Y = rho * sf;
  const T X = sstar + p / Y;
  const T B1 = rho * (sstar - v);
  const T Q = u.v[1] + B1 * X;
  // star state st and F = F(U) + S (st - U)
  Cons<T, D> st;
#pragma unroll
  for (int c = 0; c < D + 2; ++c) st.v[c] = sc * u.v[c];
  st.v[2 + d] = sstar * rho * sc;
  st.v[1] = sc * Q;
  flux_rev_partial(u, q, d, g, ub, bk);
  T Sb = T(0), scb = T(0), sb = T(0), vb = T(0);
#pragma unroll
  for (int c = 0; c < D + 2; ++c) {
    Sb += g.v[c] * (st.v[c] - u.v[c]);
    ub.v[c] += -S * g.v[c];
  }
#pragma unroll
  for (int c = 0; c < D + 2; ++c) {
    const T stb = S * g.v[c];
    if (c == 2 + d) {
      sb += stb * rho * sc;
      ub.v[0] += stb * sstar * sc;
      scb += stb * sstar * rho;
    } else if (c == 1) {
      scb += stb * Q;
      const T Qb = stb * sc;
      ub.v[1] += Qb;
      const T B1b = Qb * X;
      const T Xb = Qb * B1;
      ub.v[0] += B1b * (sstar - v);
      sb += B1b * rho;
      vb -= B1b * rho;
      sb += Xb;
      bk.p += Xb / Y;
      const T Yb = -Xb * p / (Y * Y);
      ub.v[0] += Yb * sf;
      const T sfb0 = Yb * rho;
      // sf adjoint from Y, accumulated below
      scb += T(0);
      // stash into sc's chain: sf gets sfb0 directly
      vb -= sfb0;
      Sb += sfb0;
    } else {
      scb += stb * u.v[c];
      ub.v[c] += stb * sc;
    }
  }
  // sc = sf / Z
  const T sfb = scb / Z;
  const T Zb = -scb * sc / Z;
  Sb += Zb;
  sb -= Zb;
  Sb += sfb;
  vb -= sfb;
  bk.v[d] += vb;
  // sstar = N / Dn
  const T Nb = sb / Dn;
  const T Dnb = -sb * sstar / Dn;
  T plb = -Nb, prb = Nb;
  T vlb = Nb * factl, vrb = -Nb * factr;
  T flb = Nb * vl + Dnb, frb = -Nb * vr - Dnb;
  T wslb = left ? Sb : T(0), wsrb = left ? T(0) : Sb;
  ubl.v[0] += flb * (wsl - vl);
  wslb += flb * ul.v[0];
  vlb -= flb * ul.v[0];
  ubr.v[0] += frb * (wsr - vr);
  wsrb += frb * ur.v[0];
  vrb -= frb * ur.v[0];
  // wsl = vl - al qlv ; wsr = vr + ar qrv
  vlb += wslb;
  T alb = -wslb * qlv;
  const T qlb = -wslb * al;
  vrb += wsrb;
  T arb = wsrb * qrv;
  const T qrb = wsrb * ar;
  T psb = T(0);
  if (shock_l) {
    const T Rb = qlb * adi / (T(2) * qlv);
    psb += Rb / pl;
    plb -= Rb * Rl / pl;
  }
  if (shock_r) {
    const T Rb = qrb * adi / (T(2) * qrv);
    psb += Rb / pr;
    prb -= Rb * Rr / pr;
  }
  const T pvb = (T(0) < p_pvrs) ? psb : T(0);
  plb += T(0.5) * pvb;
  prb += T(0.5) * pvb;
  const T Wb = T(-0.5) * pvb;
  const T A1b = Wb * T(0.25) * A2 * A3;
  const T A2b = Wb * T(0.25) * A1 * A3;
  const T A3b = Wb * T(0.25) * A1 * A2;
  vrb += A1b;
  vlb -= A1b;
  ubr.v[0] += A2b;
  ubl.v[0] += A2b;
  alb += A3b;
  arb += A3b;
  // a = sqrt(gamma (p + p_inf) r)
  if (al > T(0)) {
    const T Ab = alb / (T(2) * al);
    plb += Ab * gamma * ql.rinv;
    bl.r += Ab * gamma * (pl + pinf);
  }
  if (ar > T(0)) {
    const T Ab = arb / (T(2) * ar);
    prb += Ab * gamma * qr.rinv;
    br.r += Ab * gamma * (pr + pinf);
  }
  bl.p += plb;
  br.p += prb;
  bl.v[d] += vlb;
  br.v[d] += vrb;
  derive_rev(ul, ql, gm1, bl, ubl);
  derive_rev(ur, qr, gm1, br, ubr);
}

// Reverse of the FORCE flux (riemann_q<kForce>).
template <typename T, int D>
FL_HD void force_rev(const Cons<T, D>& ul, const Derived<T, D>& ql, const Cons<T, D>& ur,
                     const Derived<T, D>& qr, int d, T gm1, T dtdh, const Cons<T, D>& g,
                     Cons<T, D>& ubl, Cons<T, D>& ubr) {
  Cons<T, D> fl, fr, m, flb, frb, mb;
  flux_q(ul, ql, d, fl);
  flux_q(ur, qr, d, fr);
#pragma unroll
  for (int c = 0; c < D + 2; ++c)
    m.v[c] = T(0.5) * (ul.v[c] + ur.v[c] + dtdh * (fl.v[c] - fr.v[c]));
  const T dhdt = T(1.0) / dtdh;
  zero(flb);
  zero(frb);
  zero(mb);
  Cons<T, D> rib;
#pragma unroll
  for (int c = 0; c < D + 2; ++c) {
    const T lfb = T(0.5) * g.v[c];
    rib.v[c] = T(0.5) * g.v[c];
    flb.v[c] += T(0.5) * lfb;
    frb.v[c] += T(0.5) * lfb;
    ubl.v[c] += T(0.5) * dhdt * lfb;
    ubr.v[c] -= T(0.5) * dhdt * lfb;
  }
  flux_rev(m, derive(m, gm1), d, gm1, rib, mb);
#pragma unroll
  for (int c = 0; c < D + 2; ++c) {
    ubl.v[c] += T(0.5) * mb.v[c];
    ubr.v[c] += T(0.5) * mb.v[c];
    flb.v[c] += T(0.5) * dtdh * mb.v[c];
    frb.v[c] -= T(0.5) * dtdh * mb.v[c];
  }
  flux_rev(ul, ql, d, gm1, flb, ubl);
  flux_rev(ur, qr, d, gm1, frb, ubr);
}

template <int FLUX, typename T, int D>
FL_HD void riemann_rev(const Cons<T, D>& ul, const Cons<T, D>& ur, int d, T gamma, T gm1,
                       T adi, T dtdh, const Cons<T, D>& g, Cons<T, D>& ubl, Cons<T, D>& ubr,
                       T pinf = T(0)) {
  const Derived<T, D> ql = derive(ul, gm1), qr = derive(ur, gm1);
  if constexpr (FLUX == kForce) {
    force_rev(ul, ql, ur, qr, d, gm1, dtdh, g, ubl, ubr);
  } else {
    hllc_rev(ul, ql, ur, qr, d, gamma, gm1, adi, g, ubl, ubr, pinf);
  }
}

// Forward MUSCL-Hancock evolution of one cell (van Leer minmod slope times
// the frozen chi), as in stage C of sweep_kernel.
template <typename T, int D>
FL_HD void evolve_fwd(const Cons<T, D>& um, const Cons<T, D>& u, const Cons<T, D>& up, T chi,
                      int d, T gm1, T dtdh, Cons<T, D>& er, Cons<T, D>& el) {
  const T ch = chi * T(0.5);
  const T hd = T(0.5) * dtdh;
  Cons<T, D> a, b, fa, fb;
#pragma unroll
  for (int c = 0; c < D + 2; ++c) {
    const T delta = ch * limited_slope<T>(kVanLeer, u.v[c] - um.v[c], up.v[c] - u.v[c]);
    a.v[c] = u.v[c] - delta;
    b.v[c] = u.v[c] + delta;
  }
  flux_q(a, derive(a, gm1), d, fa);
  flux_q(b, derive(b, gm1), d, fb);
#pragma unroll
  for (int c = 0; c < D + 2; ++c) {
    const T df = fa.v[c] - fb.v[c];
    er.v[c] = b.v[c] + hd * df;
    el.v[c] = a.v[c] + hd * df;
  }
}

// Reverse of evolve_fwd: given the adjoints of both evolved faces, the
// adjoints of the cell and its two neighbours along the sweep, and in dchi
// the adjoint of the flattening coefficient: sum_c 0.5 lim_c (bb_c - ab_c),
// lim_c the limited slope that chi scales.
template <typename T, int D>
FL_HD void evolve_rev(const Cons<T, D>& um, const Cons<T, D>& u, const Cons<T, D>& up, T chi,
                      int d, T gm1, T dtdh, const Cons<T, D>& erb, const Cons<T, D>& elb,
                      Cons<T, D>& dum, Cons<T, D>& du, Cons<T, D>& dup, T& dchi) {
  const T ch = chi * T(0.5);
  const T hd = T(0.5) * dtdh;
  Cons<T, D> a, b, ab, bb, fab, fbb;
  int choice[D + 2];
#pragma unroll
  for (int c = 0; c < D + 2; ++c) {
    const T bd = u.v[c] - um.v[c], fd = up.v[c] - u.v[c];
    const bool same = (bd > T(0) && fd > T(0)) || (bd < T(0) && fd < T(0));
    choice[c] = !same ? 0 : (fl_abs<T>(bd) <= fl_abs<T>(fd) ? 1 : 2);
    const T lim = choice[c] == 0 ? T(0) : (choice[c] == 1 ? bd : fd);
    a.v[c] = u.v[c] - ch * lim;
    b.v[c] = u.v[c] + ch * lim;
    bb.v[c] = erb.v[c];
    ab.v[c] = elb.v[c];
    const T dfb = hd * (erb.v[c] + elb.v[c]);
    fab.v[c] = dfb;
    fbb.v[c] = -dfb;
  }
  flux_rev(a, derive(a, gm1), d, gm1, fab, ab);
  flux_rev(b, derive(b, gm1), d, gm1, fbb, bb);
  T gchi = T(0);
#pragma unroll
  for (int c = 0; c < D + 2; ++c) {
    du.v[c] += ab.v[c] + bb.v[c];
    const T lim = choice[c] == 0 ? T(0) : (choice[c] == 1 ? u.v[c] - um.v[c] : up.v[c] - u.v[c]);
    gchi += T(0.5) * lim * (bb.v[c] - ab.v[c]);
    const T limb = ch * (bb.v[c] - ab.v[c]);
    if (choice[c] == 1) {
      du.v[c] += limb;
      dum.v[c] -= limb;
    } else if (choice[c] == 2) {
      dup.v[c] += limb;
      du.v[c] -= limb;
    }
  }
  dchi = gchi;
}

// evolve_rev with the flattening coefficient's adjoint discarded.
template <typename T, int D>
FL_HD void evolve_rev(const Cons<T, D>& um, const Cons<T, D>& u, const Cons<T, D>& up, T chi,
                      int d, T gm1, T dtdh, const Cons<T, D>& erb, const Cons<T, D>& elb,
                      Cons<T, D>& dum, Cons<T, D>& du, Cons<T, D>& dup) {
  T dchi;
  evolve_rev(um, u, up, chi, d, gm1, dtdh, erb, elb, dum, du, dup, dchi);
}

}  // namespace fl
