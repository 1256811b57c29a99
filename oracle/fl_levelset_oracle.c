/*
 * fl_levelset_oracle.c -- CPU oracle for the level-set kernels of the
 * multimaterial (ghost-fluid) path.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's level-set
 * arithmetic, used by tests/ as the checker.  The product never links it.
 * FP64 (the level set is FP64 in the multimaterial workload).  Grids are 2-D,
 * x fastest; out-of-domain reads mirror the domain (ghost[-1-g] = cell[g]),
 * as boundary::load_padding_with_boundaries does with transmissive bounds
 * (boundary/boundary_loading.hpp:123-175).
 *
 * Parity pin: the reference's multimaterial driver does not run as shipped
 * (MultimaterialSimulator::simulate is commented out,
 * simulator/multimaterial_simulator.hpp:656-694, and several of its launches
 * swap grid and block), but its per-cell level-set functors are
 * __host__ __device__ and run on the host (oracle/ref_driver_ls.cpp).  The
 * flo_ls_* pieces below -- WENO-HJ5 derivatives, Godunov upwind gradients,
 * the Hamiltonian, the first two RK3 stages, the local eikonal solve and the
 * interface-normal velocity -- are pinned bit for bit to them through
 * tests/golden/levelset.npz (tests/test_levelset_pinned.py).  The CUDA
 * kernels are checked against this file.
 *
 * The row loops carry OpenMP pragmas: liboracle_omp.so (-fopenmp) shares rows
 * among threads for the timed CPU baseline; every cell is computed exactly
 * as in the single-threaded liboracle.so the tests use.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline int64_t mir(int64_t i, int64_t n) {
  if (i < 0) i = -1 - i;
  else if (i >= n) i = 2 * n - 1 - i;
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

static inline double at(const double* f, int64_t nx, int64_t ny, int64_t x, int64_t y) {
  return f[mir(y, ny) * nx + mir(x, nx)];
}

static inline double dmax(double a, double b) { return (a < b) ? b : a; }   /* std::max */
static inline double dmin(double a, double b) { return (b < a) ? b : a; }   /* std::min */

/* WENO-HJ5 combination of the five one-sided differences
 * (scheme/stencils/weno_hj_5.hpp:85-144). */
static double weno_diff(double d1, double d2, double d3, double d4, double d5) {
  const double phi_1 = 2.0 * d1 - 7.0 * d2 + 11.0 * d3;
  const double phi_2 = -d2 + 5.0 * d3 + 2.0 * d4;
  const double phi_3 = 2.0 * d3 + 5.0 * d4 - d5;
  const double f1 = 13.0 / 12.0, f2 = 1.0 / 4.0;
  const double t1 = d1 - 2.0 * d2 + d3, t2 = d1 - 4.0 * d2 + 3.0 * d3;
  const double t3 = d2 - 2 * d3 + d4, t4 = d2 - d4;
  const double t5 = d3 - 2.0 * d4 + d5, t6 = 3.0 * d3 - 4.0 * d4 + d5;
  double a1 = f1 * (t1 * t1) + f2 * (t2 * t2);
  double a2 = f1 * (t3 * t3) + f2 * (t4 * t4);
  double a3 = f1 * (t5 * t5) + f2 * (t6 * t6);
  const double e =
      10.0e-6 * dmax(dmax(dmax(dmax(d1 * d1, d2 * d2), d3 * d3), d4 * d4), d5 * d5) + 10.0e-99;
  const double s1 = a1 + e, s2 = a2 + e, s3 = a3 + e;
  a1 = 0.1 / (s1 * s1);
  a2 = 0.6 / (s2 * s2);
  a3 = 0.3 / (s3 * s3);
  const double w_denom = (a1 + a2 + a3) * 6.0;
  return (a1 * phi_1 + a2 * phi_2 + a3 * phi_3) / w_denom;
}

/* backward / forward WENO derivative in dimension d at (x, y)
 * (weno_hj_5.hpp:51-77). */
static double weno_back(const double* f, int64_t nx, int64_t ny, int64_t x, int64_t y, int d,
                        double h) {
  const int64_t sx = d == 0, sy = d == 1;
  double v[6];
  for (int k = -3; k <= 2; ++k) v[k + 3] = at(f, nx, ny, x + k * sx, y + k * sy);
  const double h1 = 1.0 / h;
  return weno_diff(h1 * (v[1] - v[0]), h1 * (v[2] - v[1]), h1 * (v[3] - v[2]),
                   h1 * (v[4] - v[3]), h1 * (v[5] - v[4]));
}

static double weno_fwrd(const double* f, int64_t nx, int64_t ny, int64_t x, int64_t y, int d,
                        double h) {
  const int64_t sx = d == 0, sy = d == 1;
  double v[6];
  for (int k = -2; k <= 3; ++k) v[k + 2] = at(f, nx, ny, x + k * sx, y + k * sy);
  const double h1 = 1.0 / h;
  /* d1 = phi[3]-phi[2], d2 = phi[2]-phi[1], d3 = phi[1]-phi[0],
   * d4 = phi[0]-phi[-1], d5 = phi[-1]-phi[-2] */
  return weno_diff(h1 * (v[5] - v[4]), h1 * (v[4] - v[3]), h1 * (v[3] - v[2]),
                   h1 * (v[2] - v[1]), h1 * (v[1] - v[0]));
}

/* Godunov upwind |grad phi| (scheme/schemes/godunov_upwind.hpp:94-166) and
 * the level-set Hamiltonian v * |grad phi| with the branch on sign(v)
 * (scheme/evaluators/levelset_hamiltonian.hpp:63-98). */
static double hamiltonian(const double* f, int64_t nx, int64_t ny, int64_t x, int64_t y,
                          double h, double v) {
  double r = 0.0;
  for (int d = 0; d < 2; ++d) {
    const double bk = weno_back(f, nx, ny, x, y, d, h);
    const double fw = weno_fwrd(f, nx, ny, x, y, d, h);
    double b, w;
    if (v <= 0.0) {   /* GodunovUpwind::forward */
      b = dmax(bk, 0.0);
      w = dmin(fw, 0.0);
    } else {          /* GodunovUpwind::backward */
      b = dmin(bk, 0.0);
      w = dmax(fw, 0.0);
    }
    r += dmax(b * b, w * w);
  }
  return v * sqrt(r);
}

/* The first two TVD-RK3 stages of phi_t + v |grad phi| = 0
 * (scheme/updaters/runge_kutta_3.hpp:110-148), each over the whole grid with
 * freshly mirrored ghosts. */
void flo_ls_rk3_stages_f64(int64_t nx, int64_t ny, const double* phi, const double* vel,
                           double dt, double h, double* s1, double* s2) {
#pragma omp parallel for schedule(static)
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      const int64_t i = y * nx + x;
      s1[i] = phi[i] - dt * hamiltonian(phi, nx, ny, x, y, h, vel[i]);
    }
#pragma omp parallel for schedule(static)
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      const int64_t i = y * nx + x;
      s2[i] = 0.75 * phi[i] + 0.25 * (s1[i] - dt * hamiltonian(s1, nx, ny, x, y, h, vel[i]));
    }
}

/* One TVD-RK3 step: the two stages above, then the third stage and the
 * final combination (1/3) phi^n + (2/3)(stage 3). */
void flo_ls_advect_f64(int64_t nx, int64_t ny, const double* phi, const double* vel, double dt,
                       double h, double* out) {
  const int64_t n = nx * ny;
  double* s1 = (double*)malloc(sizeof(double) * n);
  double* s2 = (double*)malloc(sizeof(double) * n);
  flo_ls_rk3_stages_f64(nx, ny, phi, vel, dt, h, s1, s2);
  const double f13 = 1.0 / 3.0, f23 = 2.0 * f13;
#pragma omp parallel for schedule(static)
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      const int64_t i = y * nx + x;
      const double s3 = s2[i] - dt * hamiltonian(s2, nx, ny, x, y, h, vel[i]);
      out[i] = (f13 * phi[i]) + (f23 * s3);
    }
  free(s1);
  free(s2);
}

/* Interface-normal velocity v_n = u . grad(phi)/|grad(phi)| of the first
 * material whose level set is <= 0 at the cell
 * (levelset/cuda/velocity_initialization.cuh:108-143, the normal by central
 * differences, iterator/multidim_iterator.hpp:291-306); 0 where no material
 * contains the cell.  states: per material (rho, E, m_x, m_y) planes. */
void flo_ls_velocity_f64(int64_t nx, int64_t ny, int nmat, const double* const* phis,
                         const double* const* states, int64_t pitch, double h, double* vel) {
#pragma omp parallel for schedule(static)
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      const int64_t i = y * nx + x;
      double v = 0.0;
      for (int m = 0; m < nmat; ++m) {
        const double* f = phis[m];
        if (!(f[i] <= 0.0 || f[i] <= -0.0)) continue;
        const double fact = 0.5 / h;
        const double g0 = fact * (at(f, nx, ny, x + 1, y) - at(f, nx, ny, x - 1, y));
        const double g1 = fact * (at(f, nx, ny, x, y + 1) - at(f, nx, ny, x, y - 1));
        const double mag = g0 * g0 + g1 * g1;
        const double s = sqrt(mag);
        const double* u = states[m];
        const double rho = u[i];
        v = (u[2 * pitch + i] / rho) * (g0 / s) + (u[3 * pitch + i] / rho) * (g1 / s);
        break;
      }
      vel[i] = v;
    }
}

/* Two level sets: remove overlaps and voids
 * (levelset/cuda/levelset_projection.cuh:54-67). */
void flo_ls_project_f64(int64_t n, double* a, double* b) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double avg = 0.5 * (a[i] + b[i]);
    a[i] -= avg;
    b[i] = -a[i];
  }
}

/* Godunov upwind local eikonal solve, f = 1, 2-D
 * (scheme/schemes/godunov_upwind_scheme.hpp:44-53); neighbours outside the
 * domain are +max (scheme/cuda/fast_iterative_method.cuh:256-266). */
static double eik_local(const double* d, int64_t nx, int64_t ny, int64_t x, int64_t y, double h) {
  const double xm = x > 0 ? d[y * nx + x - 1] : DBL_MAX;
  const double xp = x < nx - 1 ? d[y * nx + x + 1] : DBL_MAX;
  const double ym = y > 0 ? d[(y - 1) * nx + x] : DBL_MAX;
  const double yp = y < ny - 1 ? d[(y + 1) * nx + x] : DBL_MAX;
  const double a = dmin(xm, xp), b = dmin(ym, yp);
  const double fh = 1.0 * h;
  const double amb = a - b;
  if (fabs(amb) >= fh) return dmin(a, b) + fh;
  return 0.5 * (a + b + sqrt(2.0 * fh * fh - (amb * amb)));
}

static int sgn(double v) { return (0.0 < v) - (v < 0.0); }

/* ---- per-cell pieces, exported for the pin against the reference ------- */

/* WENO-HJ5 one-sided derivatives: back[d * n + i], fwrd[d * n + i]. */
void flo_ls_weno_f64(int64_t nx, int64_t ny, const double* phi, double h, double* back,
                     double* fwrd) {
  const int64_t n = nx * ny;
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x)
      for (int d = 0; d < 2; ++d) {
        back[d * n + y * nx + x] = weno_back(phi, nx, ny, x, y, d, h);
        fwrd[d * n + y * nx + x] = weno_fwrd(phi, nx, ny, x, y, d, h);
      }
}

/* Godunov upwind |grad phi|: the branch for v <= 0 (fwd) and v > 0 (bwd). */
void flo_ls_godunov_f64(int64_t nx, int64_t ny, const double* phi, double h, double* fwd,
                        double* bwd) {
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      fwd[y * nx + x] = hamiltonian(phi, nx, ny, x, y, h, -1.0) / -1.0;
      bwd[y * nx + x] = hamiltonian(phi, nx, ny, x, y, h, 1.0);
    }
}

/* v |grad phi| per cell. */
void flo_ls_hamiltonian_f64(int64_t nx, int64_t ny, const double* phi, const double* vel,
                            double h, double* out) {
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x)
      out[y * nx + x] = hamiltonian(phi, nx, ny, x, y, h, vel[y * nx + x]);
}

/* The local eikonal solve per cell (neighbours outside the domain +max). */
void flo_ls_local_solve_f64(int64_t nx, int64_t ny, const double* d, double h, double* out) {
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) out[y * nx + x] = eik_local(d, nx, ny, x, y, h);
}

/* Reinitialisation to a signed distance.  Sources are the cells next to a
 * sign change that are nearer the interface than that neighbour
 * (scheme/cuda/fast_iterative_method.cuh:48-89, which seeds the signed value
 * and patches the inside afterwards, :113-213); they keep |phi|, every other cell
 * starts at +max and takes the fixed point of the Godunov local solve
 * (iterated to convergence), and the result carries the sign of the input
 * (set_signs, :96-112).  Returns the number of sweeps. */
int flo_ls_reinit_f64(int64_t nx, int64_t ny, const double* phi, double h, double* out,
                      int max_sweeps) {
  const int64_t n = nx * ny;
  unsigned char* src = (unsigned char*)calloc((size_t)n, 1);
#pragma omp parallel for schedule(static)
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      const int64_t i = y * nx + x;
      const double c = phi[i];
      int s = 0;
      for (int d = 0; d < 2 && !s; ++d) {
        for (int k = -1; k <= 1 && !s; k += 2) {
          const int64_t xx = x + (d == 0 ? k : 0), yy = y + (d == 1 ? k : 0);
          const double o = at(phi, nx, ny, xx, yy);
          if (sgn(c) != sgn(o) && fabs(c) < fabs(o)) s = 1;
        }
      }
      src[i] = (unsigned char)s;
      out[i] = s ? fabs(c) : DBL_MAX;
    }
  double* nxt = (double*)malloc(sizeof(double) * n);
  int sweeps = 0;
  for (; sweeps < max_sweeps; ++sweeps) {
    int changed = 0;
#pragma omp parallel for schedule(static) reduction(| : changed)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t x = 0; x < nx; ++x) {
        const int64_t i = y * nx + x;
        if (src[i]) { nxt[i] = out[i]; continue; }
        const double q = eik_local(out, nx, ny, x, y, h);
        nxt[i] = dmin(out[i], q);
        if (nxt[i] != out[i]) changed = 1;
      }
    memcpy(out, nxt, sizeof(double) * n);
    if (!changed) break;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) out[i] = (double)sgn(phi[i]) * fabs(out[i]);
  free(nxt);
  free(src);
  return sweeps;
}
