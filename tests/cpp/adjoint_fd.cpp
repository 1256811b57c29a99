// Finite-difference check of the hand-written reverse mode
// (fluidity_b200/csrc/fl_adjoint.cuh) on the CPU: for random states and
// random output adjoints g, <g, J dx> from central differences must equal
// <J^T g, dx> from the reverse functions.  Prints the worst relative
// mismatch per function and exits non-zero above the tolerance.
#include <cmath>
#include <cstdio>
#include <random>

#include "fluidity_b200/csrc/fl_adjoint.cuh"

using namespace fl;
using C2 = Cons<double, 2>;

static std::mt19937_64 rng(12345);
static double U(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }

static C2 rand_state() {
  const double rho = std::exp(U(std::log(0.3), std::log(3.0)));
  const double p = std::exp(U(std::log(0.3), std::log(30.0)));
  const double vx = U(-1.5, 1.5), vy = U(-1.5, 1.5);
  C2 u;
  u.v[0] = rho;
  u.v[1] = p / 0.4 + 0.5 * rho * (vx * vx + vy * vy);
  u.v[2] = rho * vx;
  u.v[3] = rho * vy;
  return u;
}

static double dot(const C2& a, const C2& b) {
  double s = 0;
  for (int c = 0; c < 4; ++c) s += a.v[c] * b.v[c];
  return s;
}

static C2 axpy(const C2& x, double e, const C2& d) {
  C2 r;
  for (int c = 0; c < 4; ++c) r.v[c] = x.v[c] + e * d.v[c];
  return r;
}

static const double gam = 1.4, gm1 = 0.4, adi = 2.4 / 2.8;
static const double pinf_stiff = 6.0;  // stiffened fluid: p + p_inf under the sound speed

template <int FLUX>
static C2 rs(const C2& l, const C2& r, int d, double dtdh) {
  C2 f;
  const double pinf = (FLUX & kStiffEos) ? pinf_stiff : 0.0;
  riemann_q<FLUX>(l, derive(l, gm1), r, derive(r, gm1), d, gam, gm1, adi, dtdh, f, pinf);
  return f;
}

// which: 0 HLLC, 1 FORCE, 2 HLLC of the stiffened fluid
static C2 rs_which(int which, const C2& l, const C2& r, int d, double dtdh) {
  return which == 1 ? rs<kForce>(l, r, d, dtdh)
                    : which == 2 ? rs<kHllc | kStiffEos>(l, r, d, dtdh) : rs<kHllc>(l, r, d, dtdh);
}

int main() {
  double worst_flux = 0, worst_hllc = 0, worst_force = 0, worst_evolve = 0, worst_stiff = 0;
  double worst_chi = 0;
  int regions[4] = {0, 0, 0, 0};
  for (int trial = 0; trial < 4000; ++trial) {
    const C2 a = rand_state(), b = rand_state(), c3 = rand_state();
    C2 g, dl, dr, dm;
    for (int c = 0; c < 4; ++c) {
      g.v[c] = U(-1, 1);
      dl.v[c] = U(-1, 1) * std::fabs(a.v[c]) * 1e-2 + 1e-3 * U(-1, 1);
      dr.v[c] = U(-1, 1) * std::fabs(b.v[c]) * 1e-2 + 1e-3 * U(-1, 1);
      dm.v[c] = U(-1, 1) * std::fabs(c3.v[c]) * 1e-2 + 1e-3 * U(-1, 1);
    }
    const int d = trial & 1;
    const double dtdh = U(0.01, 0.2);
    const double eps = 1e-6;
    // physical flux
    {
      C2 fp, fm, ub;
      flux_q(axpy(a, eps, dl), derive(axpy(a, eps, dl), gm1), d, fp);
      flux_q(axpy(a, -eps, dl), derive(axpy(a, -eps, dl), gm1), d, fm);
      double fd = 0, sc = 0;
      for (int c = 0; c < 4; ++c) {
        fd += g.v[c] * (fp.v[c] - fm.v[c]) / (2 * eps);
        sc += std::fabs(g.v[c] * (fp.v[c] - fm.v[c]) / (2 * eps));
      }
      zero(ub);
      flux_rev(a, derive(a, gm1), d, gm1, g, ub);
      const double ad = dot(ub, dl);
      worst_flux = std::fmax(worst_flux, std::fabs(fd - ad) / std::fmax(std::fabs(ad), sc));
    }
    // Riemann fluxes; skip the rare draws where a branch flips within +-eps
    for (int which = 0; which < 3; ++which) {
      C2 fp = rs_which(which, axpy(a, eps, dl), axpy(b, eps, dr), d, dtdh);
      C2 fm = rs_which(which, axpy(a, -eps, dl), axpy(b, -eps, dr), d, dtdh);
      double fd = 0, sc = 0;
      for (int c = 0; c < 4; ++c) {
        fd += g.v[c] * (fp.v[c] - fm.v[c]) / (2 * eps);
        sc += std::fabs(g.v[c] * (fp.v[c] - fm.v[c]) / (2 * eps));
      }
      C2 ubl, ubr;
      zero(ubl);
      zero(ubr);
      if (which == 1)
        riemann_rev<kForce>(a, b, d, gam, gm1, adi, dtdh, g, ubl, ubr);
      else
        riemann_rev<kHllc>(a, b, d, gam, gm1, adi, dtdh, g, ubl, ubr,
                           which == 2 ? pinf_stiff : 0.0);
      const double ad = dot(ubl, dl) + dot(ubr, dr);
      const double err = std::fabs(fd - ad) / std::fmax(std::fabs(ad), sc);
      if (which != 1) {
        // classify the region for coverage
        const Derived<double, 2> ql = derive(a, gm1), qr = derive(b, gm1);
        (void)ql; (void)qr;
        if (err > 1e-4) {
          // check for a branch flip: the reverse of a piecewise function is
          // only defined inside a piece
          C2 f0 = rs_which(which, a, b, d, dtdh);
          double fd1 = 0, fd2 = 0;
          for (int c = 0; c < 4; ++c) {
            fd1 += g.v[c] * (fp.v[c] - f0.v[c]) / eps;
            fd2 += g.v[c] * (f0.v[c] - fm.v[c]) / eps;
          }
          if (std::fabs(fd1 - fd2) > 1e-3 * (std::fabs(fd1) + 1e-8)) continue;
        }
        if (which == 0) worst_hllc = std::fmax(worst_hllc, err);
        else worst_stiff = std::fmax(worst_stiff, err);
      } else {
        worst_force = std::fmax(worst_force, err);
      }
    }
    // evolve (chi held), and the adjoint of chi itself
    {
      const double chi = (trial % 3 == 0) ? 1.0 : U(0, 1);
      C2 erp, elp, erm, elm, eb, lb;
      evolve_fwd(axpy(a, eps, dl), axpy(b, eps, dm), axpy(c3, eps, dr), chi, d, gm1, dtdh, erp, elp);
      evolve_fwd(axpy(a, -eps, dl), axpy(b, -eps, dm), axpy(c3, -eps, dr), chi, d, gm1, dtdh, erm, elm);
      for (int c = 0; c < 4; ++c) {
        eb.v[c] = U(-1, 1);
        lb.v[c] = U(-1, 1);
      }
      double fd = 0, sc = 0;
      for (int c = 0; c < 4; ++c) {
        fd += eb.v[c] * (erp.v[c] - erm.v[c]) / (2 * eps) + lb.v[c] * (elp.v[c] - elm.v[c]) / (2 * eps);
        sc += std::fabs(eb.v[c] * (erp.v[c] - erm.v[c]) / (2 * eps)) +
              std::fabs(lb.v[c] * (elp.v[c] - elm.v[c]) / (2 * eps));
      }
      C2 dum, du, dup;
      zero(dum);
      zero(du);
      zero(dup);
      double dchi = 0.0;
      evolve_rev(a, b, c3, chi, d, gm1, dtdh, eb, lb, dum, du, dup, dchi);
      const double ad = dot(dum, dl) + dot(du, dm) + dot(dup, dr);
      // the adjoint of chi against a central difference in chi alone
      {
        const double he = 1e-6;
        C2 er2p, el2p, er2m, el2m;
        evolve_fwd(a, b, c3, chi + he, d, gm1, dtdh, er2p, el2p);
        evolve_fwd(a, b, c3, chi - he, d, gm1, dtdh, er2m, el2m);
        double fdc = 0, scc = 0;
        for (int c = 0; c < 4; ++c) {
          const double t = eb.v[c] * (er2p.v[c] - er2m.v[c]) / (2 * he) +
                           lb.v[c] * (el2p.v[c] - el2m.v[c]) / (2 * he);
          fdc += t;
          scc += std::fabs(t);
        }
        worst_chi = std::fmax(worst_chi, std::fabs(fdc - dchi) / std::fmax(std::fabs(dchi),
                                                                          std::fmax(scc, 1e-30)));
      }
      const double err = std::fabs(fd - ad) / std::fmax(std::fabs(ad), sc);
      // minmod selection flips are piecewise: skip draws whose selection differs across +-eps
      bool flip = false;
      for (int c = 0; c < 4 && !flip; ++c) {
        auto sel = [&](double e) {
          const double um = a.v[c] + e * dl.v[c], u = b.v[c] + e * dm.v[c], up = c3.v[c] + e * dr.v[c];
          const double bd = u - um, fdd = up - u;
          const bool same = (bd > 0 && fdd > 0) || (bd < 0 && fdd < 0);
          return !same ? 0 : (std::fabs(bd) <= std::fabs(fdd) ? 1 : 2);
        };
        flip = sel(eps) != sel(-eps);
      }
      if (!flip) worst_evolve = std::fmax(worst_evolve, err);
    }
    (void)regions;
  }
  std::printf("flux %.3e hllc %.3e stiff hllc %.3e force %.3e evolve %.3e chi %.3e\n",
              worst_flux, worst_hllc, worst_stiff, worst_force, worst_evolve, worst_chi);
  const double tol = 1e-5;
  return (worst_flux < tol && worst_hllc < tol && worst_stiff < tol && worst_force < tol &&
          worst_chi < tol &&
          worst_evolve < tol) ? 0 : 1;
}
