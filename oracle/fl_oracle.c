/*
 * fl_oracle.c -- CPU oracle for the finite-volume Euler split-solver step.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's per-cell
 * arithmetic, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline as the checker.  The product never links it.  See fl_oracle.h for
 * the storage layout and the parity pin.
 */
#include "fl_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* The stiffened fluid's material constant (material/stiff_fluid.hpp:38-133);
 * 0 is the ideal gas.  One value for the whole library: the oracle runs one
 * material at a time (flo_set_p_inf). */
static double flo_p_inf_ = 0.0;

void flo_set_p_inf(double p_inf) { flo_p_inf_ = p_inf; }
double flo_get_p_inf(void) { return flo_p_inf_; }

/* Branch trace of the FP64 sweep (flo_sweep_trace_f64): while flo_trace_out
 * is set, every branch decision of an evolved cell or a face folds into a
 * per-thread running hash, stored per cell and face of each line.  Two runs
 * whose hashes differ at an entry took different branches there. */
static uint64_t* flo_trace_out = NULL;
static _Thread_local uint64_t flo_trace_h = 0;
static inline int flo_trace_bit(int c) {
  if (flo_trace_out) flo_trace_h = (flo_trace_h ^ (uint64_t)(c != 0)) * 0x100000001b3ull + 1u;
  return c;
}

/* |x| with its sign decision traced (its derivative switches sign there) */
static inline double flo_trace_fabs(double x) {
  (void)flo_trace_bit(x < 0.0);
  return fabs(x);
}

#define T double
#define SFX _f64
#define SQRT(x) sqrt(x)
#define FABS(x) flo_trace_fabs(x)
#define FLO_BR(c) flo_trace_bit(c)
#define FLO_TRACE_BEGIN() (flo_trace_h = 0)
#define FLO_TRACE_END(slot) \
  do {                      \
    if (flo_trace_out) flo_trace_out[(slot)] = flo_trace_h; \
  } while (0)
#include "fl_oracle_impl.inc"
#undef T
#undef SFX
#undef SQRT
#undef FABS
#undef FLO_BR
#undef FLO_TRACE_BEGIN
#undef FLO_TRACE_END

#define T float
#define SFX _f32
#define SQRT(x) sqrtf(x)
#define FABS(x) fabsf(x)
#include "fl_oracle_impl.inc"
#undef T
#undef SFX
#undef SQRT
#undef FABS

static int check_grid(const flo_grid* g) {
  if (!g || g->dims < 1 || g->dims > 3) return 0;
  int64_t cells = 1;
  for (int d = 0; d < g->dims; ++d) {
    if (g->n[d] < 4) return 0;   /* mirror ghosts reach 4 cells deep */
    cells *= g->n[d];
  }
  return g->pitch >= cells;
}

int flo_sweep_f64(const flo_grid* g, int dim, const double* in, double* out,
                  double gamma, double dtdh, const flo_policy* pol) {
  if (!check_grid(g)) return -1;
  return sweep_impl_f64(g, dim, in, out, gamma, dtdh, pol);
}

int flo_sweep_trace_f64(const flo_grid* g, int dim, const double* in, double* out,
                        double gamma, double dtdh, const flo_policy* pol, uint64_t* trace) {
  if (!check_grid(g) || !trace) return -1;
  flo_trace_out = trace;
  const int rc = sweep_impl_f64(g, dim, in, out, gamma, dtdh, pol);
  flo_trace_out = NULL;
  return rc;
}

int flo_sweep_f32(const flo_grid* g, int dim, const float* in, float* out,
                  float gamma, float dtdh, const flo_policy* pol) {
  if (!check_grid(g)) return -1;
  return sweep_impl_f32(g, dim, in, out, gamma, dtdh, pol);
}

double flo_max_wavespeed_f64(const flo_grid* g, const double* in, double gamma) {
  return max_wavespeed_impl_f64(g, in, gamma);
}

float flo_max_wavespeed_f32(const flo_grid* g, const float* in, float gamma) {
  return max_wavespeed_impl_f32(g, in, gamma);
}

void flo_wavespeeds_f64(const flo_grid* g, const double* in, double gamma,
                        double* ws) {
  const int D = g->dims;
  int64_t cells = 1;
  for (int d = 0; d < D; ++d) cells *= g->n[d];
  for (int64_t i = 0; i < cells; ++i) {
    double u[5];
    for (int k = 0; k < D + 2; ++k) u[k] = in[(int64_t)k * g->pitch + i];
    ws[i] = max_ws_f64(u, D, gamma);
  }
}

int64_t flo_simulate_f64(const flo_grid* g, double* a, double* b, double gamma,
                         double cfl, double res, double sim_time,
                         int64_t max_iters, const flo_policy* pol,
                         int* result_in_b, double* run_time, double* dts,
                         int64_t dts_cap) {
  if (!check_grid(g)) return -1;
  return simulate_impl_f64(g, a, b, gamma, cfl, res, sim_time, max_iters,
                               pol, result_in_b, run_time, dts, dts_cap);
}

int64_t flo_simulate_f32(const flo_grid* g, float* a, float* b, float gamma,
                         float cfl, double res, float sim_time,
                         int64_t max_iters, const flo_policy* pol,
                         int* result_in_b, double* run_time, double* dts,
                         int64_t dts_cap) {
  if (!check_grid(g)) return -1;
  return simulate_impl_f32(g, a, b, gamma, cfl, res, sim_time, max_iters,
                               pol, result_in_b, run_time, dts, dts_cap);
}

void flo_prim_to_cons_f64(int dims, const double* prim, double gamma, double* cons) {
  prim_to_cons_impl_f64(dims, prim, gamma, cons);
}

void flo_prim_to_cons_f32(int dims, const float* prim, float gamma, float* cons) {
  prim_to_cons_impl_f32(dims, prim, gamma, cons);
}

/* state_impl.hpp:346-359: rho, p, then v = m / rho. */
void flo_cons_to_prim_f64(int dims, const double* cons, double gamma, double* prim) {
  prim[0] = cons[0];
  prim[1] = pres_f64(cons, dims, gamma);
  for (int d = 0; d < dims; ++d) prim[2 + d] = cons[2 + d] / cons[0];
}

void flo_flux_f64(int dims, const double* cons, double gamma, int dim, double* f) {
  flux_f64(cons, dims, gamma, dim, f);
}

void flo_riemann_f64(int dims, const double* ul, const double* ur, double gamma,
                     double dtdh, int dim, int flux, double* out) {
  riemann_f64(flux, ul, ur, dims, gamma, dim, dtdh, out);
}

void flo_extend_f64(const flo_grid* g, const double* in, int pad,
                    uint32_t reflect, double* out) {
  const int D = g->dims;
  acc_t_f64 a;
  a.base = in; a.D = D; a.pitch = g->pitch; a.reflect = reflect;
  int64_t n[3], np[3];
  for (int d = 0; d < 3; ++d) {
    a.n[d] = n[d] = (d < D) ? g->n[d] : 1;
    np[d] = (d < D) ? n[d] + 2 * pad : 1;
  }
  const int64_t cells = np[0] * np[1] * np[2];
  for (int64_t z = 0; z < np[2]; ++z)
    for (int64_t y = 0; y < np[1]; ++y)
      for (int64_t x = 0; x < np[0]; ++x) {
        const int64_t c[3] = {x - pad, (D > 1) ? y - pad : 0, (D > 2) ? z - pad : 0};
        double u[5];
        load_f64(&a, c, u);
        const int64_t idx = (z * np[1] + y) * np[0] + x;
        for (int k = 0; k < D + 2; ++k) out[k * cells + idx] = u[k];
      }
}

void flo_fill_riemann_f64(const flo_grid* g, const double* states_prim,
                          double gamma, double* out) {
  fill_riemann_impl_f64(g, states_prim, gamma, out);
}

void flo_fill_riemann_f32(const flo_grid* g, const float* states_prim,
                          float gamma, float* out) {
  fill_riemann_impl_f32(g, states_prim, gamma, out);
}
