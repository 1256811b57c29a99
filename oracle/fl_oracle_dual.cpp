/*
 * fl_oracle_dual.cpp -- the oracle's split-solver sweep in forward-mode dual
 * numbers: the FP64 reference gradient of the discrete adjoint.
 *
 * TEST INFRASTRUCTURE ONLY (linked into liboracle.so beside fl_oracle.c).
 * The body of the sweep is the same source as the FP64 oracle
 * (fl_oracle_impl.inc), evaluated with T = Dual: each value carries its
 * derivative along one input direction, every arithmetic operation applies
 * the chain rule, and every comparison -- the limiter's branches, HLLC's wave
 * region and shock/rarefaction choice, the pressure clamp -- is taken on the
 * values, so the branches are the ones the primal run takes.  The
 * flattening coefficient is computed in double from the values
 * ((double) casts in the oracle's chi), so it enters as a constant; the time
 * step is given, not derived.  That is the map the hand-written adjoint
 * transposes (branches, chi and dt frozen at the forward pass), so the
 * directional derivative here equals <adjoint gradient, direction> up to
 * rounding.
 */
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>

#include "fl_oracle.h"

namespace {

struct Dual {
  double v;  // value
  double d;  // derivative along the seeded direction
  Dual() = default;
  Dual(double x) : v(x), d(0.0) {}  // constants carry no derivative
  Dual(double x, double y) : v(x), d(y) {}
  explicit operator double() const { return v; }
  explicit operator float() const { return (float)v; }
  Dual& operator+=(const Dual& o) { d += o.d; v += o.v; return *this; }
  Dual& operator*=(const Dual& o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
};

inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline bool operator!=(Dual a, Dual b) { return a.v != b.v; }
inline Dual dual_sqrt(Dual a) {
  const double s = std::sqrt(a.v);
  return Dual(s, a.d / (2.0 * s));
}
inline Dual dual_fabs(Dual a) { return (a.v < 0.0) ? -a : a; }

// the material constant of the C oracle (flo_set_p_inf)
inline double p_inf_now() { return flo_get_p_inf(); }

#define flo_p_inf_ p_inf_now()
#define T Dual
#define SQRT(x) dual_sqrt(x)
#define FABS(x) dual_fabs(x)
// chi frozen: computed in double from the values, a constant here
#define SFX _dual
#include "fl_oracle_impl.inc"
#undef SFX
// chi differentiated: its ramp eta in dual numbers too
#undef CHI_T
#define CHI_T Dual
#define SFX _dualchi
#include "fl_oracle_impl.inc"
#undef SFX
#undef CHI_T
#undef T
#undef SQRT
#undef FABS
#undef flo_p_inf_

// One sweep in dual numbers through SWEEP: out = sweep(in) and
// out_dot = d sweep(in) [in_dot], with dtdh held constant.
template <int (*SWEEP)(const flo_grid*, int, const Dual*, Dual*, Dual, Dual, const flo_policy*)>
int sweep_dual_with(const flo_grid* g, int dim, const double* in, const double* in_dot,
                    double* out, double* out_dot, double gamma, double dtdh,
                    const flo_policy* pol) {
  if (!g || g->dims < 1 || g->dims > 3) return -1;
  int64_t cells = 1;
  for (int d = 0; d < g->dims; ++d) {
    if (g->n[d] < 4) return -1;
    cells *= g->n[d];
  }
  if (g->pitch < cells) return -1;
  const size_t n = (size_t)(g->dims + 2) * (size_t)g->pitch;
  Dual* a = (Dual*)malloc(sizeof(Dual) * n);
  Dual* b = (Dual*)malloc(sizeof(Dual) * n);
  if (!a || !b) { free(a); free(b); return -2; }
  for (size_t i = 0; i < n; ++i) { a[i] = Dual(in[i], in_dot[i]); b[i] = Dual(0.0); }
  const int rc = SWEEP(g, dim, a, b, Dual(gamma), Dual(dtdh), pol);
  for (size_t i = 0; i < n; ++i) { out[i] = b[i].v; out_dot[i] = b[i].d; }
  free(a);
  free(b);
  return rc;
}

}  // namespace

extern "C" {

/* One sweep of the FP64 oracle in dual numbers, the flattening coefficient
 * frozen at its value (the map the adjoint transposes). */
int flo_sweep_dual(const flo_grid* g, int dim, const double* in, const double* in_dot,
                   double* out, double* out_dot, double gamma, double dtdh,
                   const flo_policy* pol) {
  return sweep_dual_with<sweep_impl_dual>(g, dim, in, in_dot, out, out_dot, gamma, dtdh, pol);
}

/* The same with the flattening coefficient differentiated through its ramp
 * eta = 1 - (z - 0.75) / 0.1 (its clamps and min selections taken on the
 * values): the derivative of the sweep as it is, where chi is active. */
int flo_sweep_dual_chi(const flo_grid* g, int dim, const double* in, const double* in_dot,
                       double* out, double* out_dot, double gamma, double dtdh,
                       const flo_policy* pol) {
  return sweep_dual_with<sweep_impl_dualchi>(g, dim, in, in_dot, out, out_dot, gamma, dtdh,
                                             pol);
}

}  /* extern "C" */
