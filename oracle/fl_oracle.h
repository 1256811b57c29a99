/*
 * fl_oracle.h -- CPU oracle for the finite-volume Euler split-solver step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * per-cell arithmetic (robclu/fluidity, include/fluidity/...), used by the
 * test suite, the smoke check and the bench's CPU-baseline leg as the checker.
 * Nothing in the product (fluidity_b200/, include/) links or calls it.
 *
 * Parity pin: the restatement is checked bit-for-bit (FP64) against a host
 * build of the reference's own functors (oracle/ref_driver.cpp, built by
 * oracle/build_ref.sh into oracle/_ref/) through committed golden fixtures in
 * tests/golden/, and against the reference's host unit tests
 * (tests/state_tests_host.cpp, tests/solver_tests_host.cpp) as known answers.
 *
 * Storage: structure-of-arrays.  Component c of cell (x,y,z) lives at
 *   base[c * pitch + (z * ny + y) * nx + x]
 * with the conservative component order of the reference's State
 * (state/state.hpp:88-98): [rho, E, m_x, (m_y), (m_z)].
 */
#ifndef FL_ORACLE_H
#define FL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flux methods (flux_method/flux_hllc.hpp, flux_force.hpp,
 * flux_lax_friedrichs.hpp, flux_richtmyer.hpp). */
enum { FLO_FLUX_HLLC = 0, FLO_FLUX_FORCE = 1, FLO_FLUX_LF = 2, FLO_FLUX_RICHTMYER = 3 };
/* Limiters (limiting/van_leer_limiter.hpp, superbee_limiter.hpp). */
enum { FLO_LIMITER_VANLEER = 0, FLO_LIMITER_SUPERBEE = 1 };
/* Reconstructors (reconstruction/muscl_reconstructor.hpp,
 * basic_reconstructor.hpp). */
enum { FLO_RECON_MUSCL = 0, FLO_RECON_BASIC = 1 };

typedef struct flo_grid {
  int32_t dims;     /* 1, 2 or 3 */
  int64_t n[3];     /* cells per dimension, x fastest; unused dims = 1 */
  int64_t pitch;    /* elements between component planes, >= cell count */
} flo_grid;

typedef struct flo_policy {
  int32_t flux;       /* FLO_FLUX_* */
  int32_t limiter;    /* FLO_LIMITER_* */
  int32_t recon;      /* FLO_RECON_* */
  int32_t flatten;    /* 1: pressure-based slope flattening (chi) on */
  uint32_t reflect;   /* bit d set: dimension d has reflective ends */
} flo_policy;

/* Material: p_inf = 0 (the default) is the ideal gas; p_inf > 0 the
 * stiffened fluid (material/stiff_fluid.hpp:38-133), which changes the sound
 * speed and the energy of prim_to_cons / fill_riemann.  Applies to every
 * call that follows. */
void flo_set_p_inf(double p_inf);
double flo_get_p_inf(void);

/* One dimensional sweep: out = in + dtdh * (F(i-1/2) - F(i+1/2)) along dim. */
int flo_sweep_f64(const flo_grid* g, int dim, const double* in, double* out,
                  double gamma, double dtdh, const flo_policy* pol);
int flo_sweep_f32(const flo_grid* g, int dim, const float* in, float* out,
                  float gamma, float dtdh, const flo_policy* pol);

/* flo_sweep_f64 that also records the branch decisions (limiter cases, the
 * flattening test and clamps, HLLC's pressure clamp, wave and region tests)
 * as one hash per evolved cell and per face: trace[l * (2n + 3) + i + 1] for
 * the evolved cell i = -1..n of line l, trace[l * (2n + 3) + n + 2 + f] for
 * face f = 0..n (n = cells along dim; lines in the sweep's order).  Two
 * sweeps took the same branches at an entry iff the hashes agree there
 * (up to hash collisions). */
/* One FP64 sweep in forward-mode dual numbers (fl_oracle_dual.cpp):
 * out = sweep(in), out_dot = d sweep(in) [in_dot] with dtdh constant and the
 * branches of the values.  flo_sweep_dual takes the flattening coefficient
 * as a constant; flo_sweep_dual_chi differentiates it through its ramp. */
int flo_sweep_dual(const flo_grid* g, int dim, const double* in, const double* in_dot,
                   double* out, double* out_dot, double gamma, double dtdh,
                   const flo_policy* pol);
int flo_sweep_dual_chi(const flo_grid* g, int dim, const double* in, const double* in_dot,
                       double* out, double* out_dot, double gamma, double dtdh,
                       const flo_policy* pol);

int flo_sweep_trace_f64(const flo_grid* g, int dim, const double* in, double* out,
                        double gamma, double dtdh, const flo_policy* pol, uint64_t* trace);

/* Max over cells of max_d |u_d| + a (state/state_impl.hpp:167-178). */
double flo_max_wavespeed_f64(const flo_grid* g, const double* in, double gamma);
float  flo_max_wavespeed_f32(const flo_grid* g, const float* in, float gamma);

/* Per-cell wavespeed, written to ws[cells]. */
void flo_wavespeeds_f64(const flo_grid* g, const double* in, double gamma, double* ws);

/* Time loop of SimulatorImpl::simulate (simulator/simulator_impl.hpp:223-258).
 * a and b are the two state buffers; a holds the initial state.  Returns the
 * number of steps taken; *result_in_b tells which buffer holds the result and
 * *run_time the accumulated time.  dts (nullable) receives the dt of the
 * first dts_cap steps. */
int64_t flo_simulate_f64(const flo_grid* g, double* a, double* b, double gamma,
                         double cfl, double res, double sim_time,
                         int64_t max_iters, const flo_policy* pol,
                         int* result_in_b, double* run_time, double* dts,
                         int64_t dts_cap);
int64_t flo_simulate_f32(const flo_grid* g, float* a, float* b, float gamma,
                         float cfl, double res, float sim_time,
                         int64_t max_iters, const flo_policy* pol,
                         int* result_in_b, double* run_time, double* dts,
                         int64_t dts_cap);

/* Primitive (rho, p, v...) to conservative conversion of one state
 * (state/state_impl.hpp:390-406 with material/ideal_gas.hpp:59-63). */
void flo_prim_to_cons_f64(int dims, const double* prim, double gamma, double* cons);
void flo_prim_to_cons_f32(int dims, const float* prim, float gamma, float* cons);
void flo_cons_to_prim_f64(int dims, const double* cons, double gamma, double* prim);

/* Conservative flux of one state in dimension dim (state_impl.hpp:293-310). */
void flo_flux_f64(int dims, const double* cons, double gamma, int dim, double* flux);
/* Riemann flux between two states (policy flux only). */
void flo_riemann_f64(int dims, const double* ul, const double* ur, double gamma,
                     double dtdh, int dim, int flux, double* out);

/* Ghost extension used by every sweep (solver/boundary_loader.hpp:42-124,
 * 175-199): out is the grid padded by pad cells on both ends of every
 * dimension; a ghost at index -1-g takes cell g (and n+g takes n-1-g), and a
 * dimension with reflective ends negates its normal momentum as
 * m = (-(m/rho)) * rho (state/state.hpp:437-441).  out uses SoA planes of
 * the padded cell count. */
void flo_extend_f64(const flo_grid* g, const double* in, int pad,
                    uint32_t reflect, double* out);

/* Seeded quadrant / octant / two-state Riemann initial condition in
 * conservative SoA form.  states_prim holds 2^dims primitive states
 * (rho, p, v_x.. per state) indexed by (x >= 0.5) + 2 (y >= 0.5) + 4 (z >= 0.5),
 * cell positions being float(i)/float(N) (simulator_impl.hpp:318-335). */
void flo_fill_riemann_f64(const flo_grid* g, const double* states_prim,
                          double gamma, double* out);
void flo_fill_riemann_f32(const flo_grid* g, const float* states_prim,
                          float gamma, float* out);

#ifdef __cplusplus
}
#endif
#endif /* FL_ORACLE_H */
