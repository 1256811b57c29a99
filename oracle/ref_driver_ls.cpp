// ref_driver_ls.cpp -- host driver around the reference's level-set functors.
//
// TEST INFRASTRUCTURE ONLY (included by ref_driver.cpp, built into
// oracle/_ref/libfluidity_ref.so by oracle/build_ref.sh).  The reference's
// multimaterial driver does not run as shipped, but the per-cell level-set
// arithmetic is written as __host__ __device__ functors.  This file evaluates
// them cell by cell on host grids, so that the C restatement
// (oracle/fl_levelset_oracle.c) can be pinned to them:
//   HJWeno5::backward_deriv / forward_deriv   scheme/stencils/weno_hj_5.hpp:51-144
//   GodunovUpwind::forward / backward         scheme/schemes/godunov_upwind.hpp:94-166
//   LevelsetHamiltonian::evaluate             scheme/evaluators/levelset_hamiltonian.hpp:63-98
//   RungeKutta3::update_impl                  scheme/updaters/runge_kutta_3.hpp:110-148
//   GodunovUpwindScheme::solve                scheme/schemes/godunov_upwind_scheme.hpp:37-79
//   State::velocity_vec, MultidimIterator::norm, math::dot, levelset::inside
//       (the per-cell body of set_velocities, levelset/cuda/velocity_initialization.cuh:108-143)
//   MultidimIterator::norm, math::interp, State::velocity_vec / set_velocity,
//   math::dot, Hllc::solve_star_conservative_left
//       (the per-source body of RiemannGFM::invoke, ghost_fluid/riemann_ghost_fluid.hpp:70-190)
// The loops over cells are ours; every number comes from the reference's code.
//
// Host grids: 2-D, x fastest, padded by kLsPad cells on every side.  Ghost
// values are the mirror rule of the split path (ghost[-1-g] = cell[g]) for
// the derivative stencils and the interface normal, and +max for the local
// eikonal solve (out-of-domain neighbours never win its minimum), the
// boundary semantics the CUDA kernels and the C restatement define.

// levelset.hpp prints with std::cout / std::setw without including their
// headers; they come first here.
#include <iomanip>
#include <iostream>

#include <fluidity/iterator/multidim_iterator.hpp>
#include <fluidity/levelset/levelset.hpp>
#include <fluidity/math/interp.hpp>
#include <fluidity/math/math.hpp>
#include <fluidity/scheme/evaluators/levelset_hamiltonian.hpp>
#include <fluidity/scheme/schemes/godunov_upwind.hpp>
#include <fluidity/scheme/schemes/godunov_upwind_scheme.hpp>
#include <fluidity/scheme/stencils/weno_hj_5.hpp>
#include <fluidity/scheme/updaters/runge_kutta_3.hpp>
#include <fluidity/state/state.hpp>

#include <cfloat>
#include <cstdint>
#include <vector>

namespace {

constexpr int64_t kLsPad = 3;
using ls_it_t = fluid::MultidimIterator<double, fluid::DimInfo<2>, fluid::exec::cpu_t>;
using weno_t = fluid::scheme::stencil::HJWeno5;

int64_t ls_mirror(int64_t i, int64_t n) {
  if (i < 0) i = -1 - i;
  else if (i >= n) i = 2 * n - 1 - i;
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// A padded copy of a 2-D field; ghosts mirror the domain, or hold `fill`
// when fill_ghosts is set.
struct LsField {
  int64_t nx, ny, px, py;
  std::vector<double> v;
  LsField(int64_t nx_, int64_t ny_, const double* f, bool use_fill = false, double fill = 0.0)
      : nx(nx_), ny(ny_), px(nx_ + 2 * kLsPad), py(ny_ + 2 * kLsPad), v((size_t)(px * py)) {
    for (int64_t y = -kLsPad; y < ny + kLsPad; ++y)
      for (int64_t x = -kLsPad; x < nx + kLsPad; ++x) {
        const bool in = x >= 0 && x < nx && y >= 0 && y < ny;
        v[(size_t)((y + kLsPad) * px + x + kLsPad)] =
            (!in && use_fill) ? fill : f[ls_mirror(y, ny) * nx + ls_mirror(x, nx)];
      }
  }
  double* at(int64_t x, int64_t y) { return v.data() + (y + kLsPad) * px + x + kLsPad; }
  fluid::DimInfo<2> info() const { return fluid::DimInfo<2>(px, py); }
};

// A padded copy of a 2-D SoA state (rho, E, m_x, m_y), mirror ghosts.
struct LsStates {
  int64_t nx, ny, px, py;
  std::vector<fluid::state::conservative_t<double, 2>> v;
  LsStates(int64_t nx_, int64_t ny_, int64_t pitch, const double* u)
      : nx(nx_), ny(ny_), px(nx_ + 2 * kLsPad), py(ny_ + 2 * kLsPad), v((size_t)(px * py)) {
    for (int64_t y = -kLsPad; y < ny + kLsPad; ++y)
      for (int64_t x = -kLsPad; x < nx + kLsPad; ++x) {
        const int64_t i = ls_mirror(y, ny) * nx + ls_mirror(x, nx);
        auto& s = v[(size_t)((y + kLsPad) * px + x + kLsPad)];
        for (int k = 0; k < 4; ++k) s[k] = u[k * pitch + i];
      }
  }
  fluid::state::conservative_t<double, 2>* at(int64_t x, int64_t y) {
    return v.data() + (y + kLsPad) * px + x + kLsPad;
  }
  fluid::DimInfo<2> info() const { return fluid::DimInfo<2>(px, py); }
};

// Steps 1-4 of RiemannGFM::invoke for one source cell of material A
// (ghost_fluid/riemann_ghost_fluid.hpp:70-190): the star state it writes and
// the offset of the cell it writes it to.
template <typename EosA, typename EosB>
void gfm_star_cell(LsField& pa, LsStates& sa, LsStates& sb, int64_t x, int64_t y, double dh,
                   const EosA& eos_a, const EosB& eos_b, double* star_out, int* tx, int* ty) {
  using st_it_t =
      fluid::MultidimIterator<fluid::state::conservative_t<double, 2>, fluid::DimInfo<2>,
                              fluid::exec::cpu_t>;
  ls_it_t ls_it(pa.at(x, y), pa.info());
  st_it_t a_it(sa.at(x, y), sa.info());
  st_it_t b_it(sb.at(x, y), sb.info());
  // STEP 1: weights and Riemann inputs
  const auto norm = ls_it.norm();
  const auto abs_phi = std::abs(*ls_it);
  const auto dh_three_two = 1.5 * dh;
  auto weights = norm * (abs_phi - dh_three_two) / dh;
  auto w_l = fluid::math::interp(a_it, weights);
  weights = norm * (abs_phi + dh_three_two) / dh;
  auto w_r = fluid::math::interp(b_it, weights);
  // STEP 2: normal and tangential velocities
  const auto vl = w_l.velocity_vec();
  const auto vl_dot_n = fluid::math::dot(w_l.velocity_vec(), norm);
  const auto vr_dot_n = fluid::math::dot(w_r.velocity_vec(), norm);
  w_l.set_velocity(vl_dot_n, fluid::dim_x);
  w_r.set_velocity(vr_dot_n, fluid::dim_x);
  w_l.set_velocity(0, fluid::dim_y);
  w_r.set_velocity(0, fluid::dim_y);
  // STEP 3: the left star state
  auto star = fluid::flux::Hllc::solve_star_conservative_left(w_l, w_r, eos_a, eos_b,
                                                             fluid::dim_x);
  // STEP 4: rotate back
  fluid::unrolled_for<2>([&](auto dim) {
    star.set_velocity(vl[dim] + (star.velocity(dim) - vl_dot_n) * norm[dim], dim);
  });
  for (int k = 0; k < 4; ++k) star_out[k] = star[k];
  *tx = fluid::math::signum(norm[0]);
  *ty = fluid::math::signum(norm[1]);
}

}  // namespace

extern "C" {

// The star states the reference's GFM computes for the listed source cells
// of material A (states ua, level set pa) against material B (ub); a
// material is the ideal gas when its p_inf is 0, else StiffFluid(gamma,
// p_inf).  stars: 4 values per cell; (tx, ty): the target cell's offset.
void ref_gfm_star_2d(int64_t nx, int64_t ny, int64_t pitch, double h, const double* ua,
                     const double* ub, const double* pa, double ga, double ia, double gb,
                     double ib, int64_t ncells, const int64_t* xs, const int64_t* ys,
                     double* stars, int* tx, int* ty) {
  LsField fa(nx, ny, pa);
  LsStates sa(nx, ny, pitch, ua), sb(nx, ny, pitch, ub);
  for (int64_t k = 0; k < ncells; ++k) {
    auto run = [&](const auto& ea, const auto& eb) {
      gfm_star_cell(fa, sa, sb, xs[k], ys[k], h, ea, eb, stars + 4 * k, tx + k, ty + k);
    };
    if (ia == 0.0 && ib == 0.0) run(ideal_t(ga), ideal_t(gb));
    else if (ia == 0.0) run(ideal_t(ga), stiff_t(gb, ib));
    else if (ib == 0.0) run(stiff_t(ga, ia), ideal_t(gb));
    else run(stiff_t(ga, ia), stiff_t(gb, ib));
  }
}

// One-sided WENO-HJ5 derivatives: back[d * n + i], fwrd[d * n + i] for
// dimension d of cell i.
void ref_ls_weno_2d(int64_t nx, int64_t ny, const double* phi, double h, double* back,
                    double* fwrd) {
  LsField f(nx, ny, phi);
  const auto info = f.info();
  const int64_t n = nx * ny;
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      ls_it_t it(f.at(x, y), info);
      const int64_t i = y * nx + x;
      back[i] = weno_t{}.backward_deriv(it, h, fluid::dim_x);
      fwrd[i] = weno_t{}.forward_deriv(it, h, fluid::dim_x);
      back[n + i] = weno_t{}.backward_deriv(it, h, fluid::dim_y);
      fwrd[n + i] = weno_t{}.forward_deriv(it, h, fluid::dim_y);
    }
}

// GodunovUpwind<HJWeno5>::forward and ::backward (|grad phi| by upwinding).
void ref_ls_godunov_2d(int64_t nx, int64_t ny, const double* phi, double h, double* fwd,
                       double* bwd) {
  LsField f(nx, ny, phi);
  const auto info = f.info();
  const fluid::scheme::GodunovUpwind<weno_t> scheme;
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      ls_it_t it(f.at(x, y), info);
      fwd[y * nx + x] = scheme.forward(it, h);
      bwd[y * nx + x] = scheme.backward(it, h);
    }
}

// LevelsetHamiltonian<HJWeno5>::evaluate(phi, h, v): v |grad phi| with the
// upwind direction chosen by the sign of v.
void ref_ls_hamiltonian_2d(int64_t nx, int64_t ny, const double* phi, const double* vel,
                           double h, double* out) {
  LsField f(nx, ny, phi);
  LsField v(nx, ny, vel);
  const auto info = f.info();
  const fluid::scheme::evaluator::LevelsetHamiltonian<weno_t> ham;
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      ls_it_t it(f.at(x, y), info);
      ls_it_t vit(v.at(x, y), info);
      out[y * nx + x] = ham.evaluate(it, h, vit);
    }
}

// RungeKutta3<LevelsetHamiltonian<HJWeno5>>::update_impl(phi, out, dt, h, v)
// per cell, each call on fresh copies: `phi` holds phi^n and `out` the first
// stage over the whole grid (stage1), so that the second stage, which the
// call writes back into its input cell, reads the first stage of every
// neighbour -- the value of the stage-synchronised scheme.  Returns that
// second stage per cell.  (The call's later lines read the input grid again,
// which holds phi^n away from the cell, so its final output is not the
// synchronised third stage and is not used.)
void ref_ls_rk3_stage2_2d(int64_t nx, int64_t ny, const double* phi, const double* stage1,
                          const double* vel, double dt, double h, double* stage2) {
  LsField in(nx, ny, phi);
  LsField out(nx, ny, stage1);
  LsField v(nx, ny, vel);
  const auto info = in.info();
  const fluid::scheme::updater::RungeKutta3<
      fluid::scheme::evaluator::LevelsetHamiltonian<weno_t>> rk3;
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      double* pin = in.at(x, y);
      double* pout = out.at(x, y);
      const double keep_in = *pin, keep_out = *pout;
      ls_it_t iit(pin, info), oit(pout, info), vit(v.at(x, y), info);
      rk3.update_impl(iit, oit, dt, h, vit);
      stage2[y * nx + x] = *pin;
      *pin = keep_in;    // restore both grids for the next cell
      *pout = keep_out;
    }
}

// GodunovUpwindScheme::solve(it, h, f = 1): the local eikonal solve of the
// fast iterative method, neighbours outside the domain at +max.
void ref_ls_local_solve_2d(int64_t nx, int64_t ny, const double* d, double h, double* out) {
  LsField f(nx, ny, d, true, DBL_MAX);
  const auto info = f.info();
  const fluid::scheme::GodunovUpwindScheme scheme;
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      ls_it_t it(f.at(x, y), info);
      out[y * nx + x] = scheme.solve(it, h, 1.0);
    }
}

// The per-cell body of set_velocities: for the first material whose level
// set is inside (<= 0) at the cell, dot(state.velocity_vec(), phi.norm(h));
// 0 where no material holds the cell.  states: per material (rho, E, m_x,
// m_y) planes `pitch` apart.
void ref_ls_velocity_2d(int64_t nx, int64_t ny, int nmat, const double* const* phis,
                        const double* const* states, int64_t pitch, double h, double* vel) {
  std::vector<LsField> fs;
  for (int m = 0; m < nmat; ++m) fs.emplace_back(nx, ny, phis[m]);
  for (int64_t y = 0; y < ny; ++y)
    for (int64_t x = 0; x < nx; ++x) {
      const int64_t i = y * nx + x;
      double v = 0.0;
      for (int m = 0; m < nmat; ++m) {
        ls_it_t it(fs[m].at(x, y), fs[m].info());
        if (!fluid::levelset::inside(it)) continue;
        fluid::state::conservative_t<double, 2> s;
        for (int k = 0; k < 4; ++k) s[k] = states[m][k * pitch + i];
        v = fluid::math::dot(s.velocity_vec(), it.norm(h));
        break;
      }
      vel[i] = v;
    }
}

}  // extern "C"
