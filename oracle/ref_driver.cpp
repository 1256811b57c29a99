// ref_driver.cpp -- host driver around the reference's own numerics functors.
//
// TEST INFRASTRUCTURE ONLY.  The reference (robclu/fluidity) has no working
// CPU execution path: its CPU SimulationData, set_wavespeeds and
// load_boundaries are empty stubs (simulator/simulation_data.hpp:38-41,
// simulator/wavespeed_initialization.hpp:34-37, solver/load_boundaries.hpp:32-36).
// Its per-cell arithmetic, however, is written as __host__ __device__ functors.
// This file drives those functors -- FaceFlux (solver/flux_solver.hpp:27-202),
// MHReconstructor/BasicReconstructor, VanLeer/Superbee, Hllc/Force/
// LaxFriedrichs/Richtmyer, State, IdealGas, BoundarySetter and the simulator's
// Parameters time control (simulator/parameters.hpp:60-99) -- with a host loop
// that reproduces SplitSolver::solve (solver/split_solver.hpp:105-162,
// solver/cuda/split_solver.cuh:57-80) and SimulatorImpl::simulate
// (simulator/simulator_impl.hpp:223-258).  The loop is ours; every number is
// computed by the reference's code.  It is built by oracle/build_ref.sh into
// oracle/_ref/libfluidity_ref.so and serves as (a) the pin of the C oracle and
// (b) the reference CPU baseline.  OpenMP parallelises over cell rows.
//
// Ghost semantics: the grid is padded by 4 cells in every dimension; ghost
// cells are filled with the reference's BoundarySetter, dimension by
// dimension in x, y, z order (mirror: ghost[-1-g] = cell[g]).  Within one
// sweep this reproduces BoundaryLoader::load_boundary
// (solver/boundary_loader.hpp:175-199) in the sweep dimension and defines the
// cross-dimension reads of the flattening coefficient, which the reference's
// GPU tile leaves undefined at tile edges.

#include <fluidity/flux_method/flux_force.hpp>
#include <fluidity/flux_method/flux_hllc.hpp>
#include <fluidity/flux_method/flux_lax_friedrichs.hpp>
#include <fluidity/flux_method/flux_richtmyer.hpp>
#include <fluidity/iterator/multidim_iterator.hpp>
#include <fluidity/limiting/superbee_limiter.hpp>
#include <fluidity/limiting/van_leer_limiter.hpp>
#include <fluidity/material/ideal_gas.hpp>
#include <fluidity/material/stiff_fluid.hpp>
#include <fluidity/reconstruction/basic_reconstructor.hpp>
#include <fluidity/reconstruction/muscl_reconstructor.hpp>
#include <fluidity/simulator/parameters.hpp>
#include <fluidity/solver/boundary_loader.hpp>
#include <fluidity/solver/flux_solver.hpp>
#include <fluidity/state/state.hpp>

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

using ideal_t = fluid::material::IdealGas<double>;
using stiff_t = fluid::material::StiffFluid<double>;
using form_t = fluid::limit::cons_form_t;

// The material of the calls that follow: the ideal gas while p_inf is 0, else
// the reference's StiffFluid(gamma, p_inf).
double g_p_inf = 0.0;

template <typename Mat> Mat make_mat(double gamma);
template <> ideal_t make_mat<ideal_t>(double gamma) { return ideal_t(gamma); }
template <> stiff_t make_mat<stiff_t>(double gamma) { return stiff_t(gamma, g_p_inf); }
constexpr int kPad = 4;

template <int D>
using state_t = fluid::state::conservative_t<double, D>;

struct Grid {
  int dims;
  int64_t n[3];
  int64_t pitch;
};

template <int D>
struct Padded {
  int64_t n[3];
  int64_t np[3];
  std::vector<state_t<D>> cells;

  explicit Padded(const Grid& g) {
    for (int d = 0; d < 3; ++d) {
      n[d] = d < D ? g.n[d] : 1;
      np[d] = d < D ? n[d] + 2 * kPad : 1;
    }
    cells.resize(static_cast<size_t>(np[0] * np[1] * np[2]));
  }
  int64_t index(int64_t x, int64_t y, int64_t z) const {
    return (z * np[1] + y) * np[0] + x;
  }
  int64_t interior(int64_t x, int64_t y, int64_t z) const {
    return index(x + kPad, D > 1 ? y + kPad : 0, D > 2 ? z + kPad : 0);
  }
};

template <int D>
fluid::DimInfo<D> make_info(const int64_t* np) {
  if constexpr (D == 1) return fluid::DimInfo<1>(np[0]);
  else if constexpr (D == 2) return fluid::DimInfo<2>(np[0], np[1]);
  else return fluid::DimInfo<3>(np[0], np[1], np[2]);
}

// Fills ghosts of dimension Dd for every (already filled or ghost) position of
// the other dimensions, using the reference's BoundarySetter.
template <int D, int Dd>
void fill_ghosts(Padded<D>& p, const fluid::solver::BoundarySetter& setter) {
  using dim_t = fluid::Dimension<Dd>;
  const int64_t n = p.n[Dd];
  int64_t lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  for (int d = 0; d < D; ++d) {
    // dimensions filled earlier (d < Dd) span their ghosts as well
    lo[d] = d < Dd ? 0 : kPad;
    hi[d] = d < Dd ? p.np[d] : kPad + p.n[d];
  }
  lo[Dd] = 0; hi[Dd] = 1;
  for (int64_t a = lo[0]; a < hi[0]; ++a)
    for (int64_t b = lo[1]; b < hi[1]; ++b)
      for (int64_t c = lo[2]; c < hi[2]; ++c) {
        int64_t q[3] = {a, b, c};
        for (int g = 0; g < kPad; ++g) {
          int64_t src[3] = {q[0], q[1], q[2]}, dst[3] = {q[0], q[1], q[2]};
          src[Dd] = kPad + g;             dst[Dd] = kPad - 1 - g;
          setter(p.cells[p.index(src[0], src[1], src[2])],
                 p.cells[p.index(dst[0], dst[1], dst[2])], dim_t{},
                 fluid::solver::BoundaryIndex::first);
          src[Dd] = kPad + n - 1 - g;     dst[Dd] = kPad + n + g;
          setter(p.cells[p.index(src[0], src[1], src[2])],
                 p.cells[p.index(dst[0], dst[1], dst[2])], dim_t{},
                 fluid::solver::BoundaryIndex::second);
        }
      }
}

template <int D>
void load_padded(const Grid& g, const double* in, uint32_t reflect, Padded<D>& p) {
  fluid::solver::BoundarySetter setter;
  fluid::unrolled_for<D>([&](auto d) {
    setter.configure(fluid::Dimension<d>{}, fluid::solver::BoundaryIndex::first,
                     ((reflect >> d) & 1u) ? fluid::solver::BoundaryKind::reflective
                                           : fluid::solver::BoundaryKind::transmissive);
  });
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t z = 0; z < p.n[2]; ++z)
    for (int64_t y = 0; y < p.n[1]; ++y)
      for (int64_t x = 0; x < p.n[0]; ++x) {
        const int64_t idx = (z * p.n[1] + y) * p.n[0] + x;
        auto& s = p.cells[p.interior(x, y, z)];
        for (int k = 0; k < D + 2; ++k) s[k] = in[k * g.pitch + idx];
      }
  fill_ghosts<D, 0>(p, setter);
  if constexpr (D > 1) fill_ghosts<D, 1>(p, setter);
  if constexpr (D > 2) fill_ghosts<D, 2>(p, setter);
}

// One sweep: out = U + dtdh * FaceFlux::flux_delta(U, dim)
// (split_solver.hpp:160).
template <int D, typename Mat, typename Recon, typename Flux, int Dim>
void sweep_t(const Grid& g, const double* in, double* out, double gamma,
             double dtdh, uint32_t reflect) {
  using ff_t = fluid::solver::FaceFlux<Recon, Flux, Mat>;
  using it_t = fluid::MultidimIterator<state_t<D>, fluid::DimInfo<D>, fluid::exec::cpu_t>;
  Padded<D> p(g);
  load_padded<D>(g, in, reflect, p);
  const auto info = make_info<D>(p.np);
  const ff_t ff(make_mat<Mat>(gamma), dtdh);
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t z = 0; z < p.n[2]; ++z)
    for (int64_t y = 0; y < p.n[1]; ++y)
      for (int64_t x = 0; x < p.n[0]; ++x) {
        it_t it(p.cells.data() + p.interior(x, y, z), info);
        const auto res = *it + dtdh * ff.flux_delta(it, fluid::Dimension<Dim>{});
        const int64_t idx = (z * p.n[1] + y) * p.n[0] + x;
        for (int k = 0; k < D + 2; ++k) out[k * g.pitch + idx] = res[k];
      }
}

template <int D, typename Mat, typename Recon, typename Flux>
void sweep_dim(const Grid& g, int dim, const double* in, double* out, double gamma,
               double dtdh, uint32_t reflect) {
  if (dim == 0) sweep_t<D, Mat, Recon, Flux, 0>(g, in, out, gamma, dtdh, reflect);
  if constexpr (D > 1) if (dim == 1) sweep_t<D, Mat, Recon, Flux, 1>(g, in, out, gamma, dtdh, reflect);
  if constexpr (D > 2) if (dim == 2) sweep_t<D, Mat, Recon, Flux, 2>(g, in, out, gamma, dtdh, reflect);
}

template <int D, typename Mat, typename Recon>
int sweep_flux(const Grid& g, int dim, const double* in, double* out, double gamma,
               double dtdh, int flux, uint32_t reflect) {
  using namespace fluid::flux;
  switch (flux) {
    case 0: sweep_dim<D, Mat, Recon, Hllc>(g, dim, in, out, gamma, dtdh, reflect); return 0;
    case 1: sweep_dim<D, Mat, Recon, Force>(g, dim, in, out, gamma, dtdh, reflect); return 0;
    case 2: sweep_dim<D, Mat, Recon, LaxFriedrichs>(g, dim, in, out, gamma, dtdh, reflect); return 0;
    case 3: sweep_dim<D, Mat, Recon, Richtmyer>(g, dim, in, out, gamma, dtdh, reflect); return 0;
  }
  return -1;
}

template <int D, typename Mat>
int sweep_recon(const Grid& g, int dim, const double* in, double* out, double gamma,
                double dtdh, int flux, int limiter, int recon, uint32_t reflect) {
  if (recon == 1)
    return sweep_flux<D, Mat, fluid::recon::BasicReconstructor<fluid::limit::VanLeer<form_t>>>(
        g, dim, in, out, gamma, dtdh, flux, reflect);
  if (limiter == 1)
    return sweep_flux<D, Mat, fluid::recon::MHReconstructor<fluid::limit::Superbee<form_t>>>(
        g, dim, in, out, gamma, dtdh, flux, reflect);
  return sweep_flux<D, Mat, fluid::recon::MHReconstructor<fluid::limit::VanLeer<form_t>>>(
      g, dim, in, out, gamma, dtdh, flux, reflect);
}

template <int D>
int sweep_all(const Grid& g, int dim, const double* in, double* out, double gamma,
              double dtdh, int flux, int limiter, int recon, uint32_t reflect) {
  if (g_p_inf != 0.0)
    return sweep_recon<D, stiff_t>(g, dim, in, out, gamma, dtdh, flux, limiter, recon, reflect);
  return sweep_recon<D, ideal_t>(g, dim, in, out, gamma, dtdh, flux, limiter, recon, reflect);
}

bool valid(const Grid& g) {
  if (g.dims < 1 || g.dims > 3) return false;
  int64_t cells = 1;
  for (int d = 0; d < g.dims; ++d) {
    if (g.n[d] < kPad) return false;
    cells *= g.n[d];
  }
  return g.pitch >= cells;
}

template <int D, typename Mat>
double max_ws(const Grid& g, const double* in, double gamma) {
  const Mat mat = make_mat<Mat>(gamma);
  int64_t cells = 1;
  for (int d = 0; d < D; ++d) cells *= g.n[d];
  double m = 0.0;
  bool first = true;
  // serial: std::max reduction in cell order (algorithm/max_element.hpp:28-38)
  for (int64_t i = 0; i < cells; ++i) {
    state_t<D> s;
    for (int k = 0; k < D + 2; ++k) s[k] = in[k * g.pitch + i];
    const double w = s.max_wavespeed(mat);
    m = first ? w : std::max(m, w);
    first = false;
  }
  return m;
}

}  // namespace

extern "C" {

int ref_sweep_f64(int dims, const int64_t* n, int64_t pitch, int dim,
                  const double* in, double* out, double gamma, double dtdh,
                  int flux, int limiter, int recon, uint32_t reflect) {
  const Grid g{dims, {n[0], dims > 1 ? n[1] : 1, dims > 2 ? n[2] : 1}, pitch};
  if (!valid(g) || dim < 0 || dim >= dims) return -1;
  switch (dims) {
    case 1: return sweep_all<1>(g, dim, in, out, gamma, dtdh, flux, limiter, recon, reflect);
    case 2: return sweep_all<2>(g, dim, in, out, gamma, dtdh, flux, limiter, recon, reflect);
    case 3: return sweep_all<3>(g, dim, in, out, gamma, dtdh, flux, limiter, recon, reflect);
  }
  return -1;
}

double ref_max_wavespeed_f64(int dims, const int64_t* n, int64_t pitch,
                             const double* in, double gamma) {
  const Grid g{dims, {n[0], dims > 1 ? n[1] : 1, dims > 2 ? n[2] : 1}, pitch};
  const bool stiff = g_p_inf != 0.0;
  switch (dims) {
    case 1: return stiff ? max_ws<1, stiff_t>(g, in, gamma) : max_ws<1, ideal_t>(g, in, gamma);
    case 2: return stiff ? max_ws<2, stiff_t>(g, in, gamma) : max_ws<2, ideal_t>(g, in, gamma);
    case 3: return stiff ? max_ws<3, stiff_t>(g, in, gamma) : max_ws<3, ideal_t>(g, in, gamma);
  }
  return -1.0;
}

void ref_set_p_inf(double p_inf) { g_p_inf = p_inf; }

// Hllc::solve_star_conservative_left (flux_method/flux_hllc.hpp:330-361) for
// 2-D conservative states of two materials, normal direction x; a material
// is the ideal gas when its p_inf is 0, else StiffFluid(gamma, p_inf).
void ref_star_left_2d(const double* ul, const double* ur, double gl, double il, double gr,
                      double ir, double* out) {
  using st_t = state_t<2>;
  st_t l, r;
  for (int k = 0; k < 4; ++k) {
    l[k] = ul[k];
    r[k] = ur[k];
  }
  auto run = [&](const auto& eosl, const auto& eosr) {
    const st_t s = fluid::flux::Hllc::solve_star_conservative_left(l, r, eosl, eosr,
                                                                  fluid::dimx_t());
    for (int k = 0; k < 4; ++k) out[k] = s[k];
  };
  if (il == 0.0 && ir == 0.0) run(ideal_t(gl), ideal_t(gr));
  else if (il == 0.0) run(ideal_t(gl), stiff_t(gr, ir));
  else if (ir == 0.0) run(stiff_t(gl, il), ideal_t(gr));
  else run(stiff_t(gl, il), stiff_t(gr, ir));
}

// Primitive -> conservative with the reference's State::conservative
// (state/state_impl.hpp:390-406) and the current material's eos.
void ref_prim_to_cons_f64(int dims, const double* prim, double gamma, double* cons) {
  auto run = [&](auto dim_tag, auto mat) {
    constexpr int D = decltype(dim_tag)::value;
    fluid::state::primitive_t<double, D> s;
    for (int k = 0; k < D + 2; ++k) s[k] = prim[k];
    const auto c = s.conservative(mat);
    for (int k = 0; k < D + 2; ++k) cons[k] = c[k];
  };
  const bool stiff = g_p_inf != 0.0;
  switch (dims) {
    case 1: stiff ? run(std::integral_constant<int, 1>{}, make_mat<stiff_t>(gamma))
                  : run(std::integral_constant<int, 1>{}, make_mat<ideal_t>(gamma)); break;
    case 2: stiff ? run(std::integral_constant<int, 2>{}, make_mat<stiff_t>(gamma))
                  : run(std::integral_constant<int, 2>{}, make_mat<ideal_t>(gamma)); break;
    default: stiff ? run(std::integral_constant<int, 3>{}, make_mat<stiff_t>(gamma))
                   : run(std::integral_constant<int, 3>{}, make_mat<ideal_t>(gamma)); break;
  }
}

// SimulatorImpl::simulate's loop with the reference's own Parameters.
int64_t ref_simulate_f64(int dims, const int64_t* n, int64_t pitch, double* a,
                         double* b, double gamma, double cfl, double res,
                         double sim_time, int64_t max_iters, int flux,
                         int limiter, int recon, uint32_t reflect,
                         int* result_in_b, double* run_time, double* dts,
                         int64_t dts_cap) {
  const Grid g{dims, {n[0], dims > 1 ? n[1] : 1, dims > 2 ? n[2] : 1}, pitch};
  if (!valid(g)) return -1;
  fluid::sim::Parameters<double> params(static_cast<std::size_t>(dims));
  params.domain.set_resolution(res);
  params.cfl = cfl;
  params.sim_time = sim_time;
  params.max_iters = static_cast<std::size_t>(max_iters);
  double* in = a;
  double* out = b;
  while (params.continue_simulation()) {
    params.update_time_delta(ref_max_wavespeed_f64(dims, n, pitch, in, gamma));
    if (dts && static_cast<int64_t>(params.iters) < dts_cap) dts[params.iters] = params.dt();
    const double dtdh = params.dt_dh();
    double* si = in;
    double* so = out;
    for (int d = 0; d < dims; ++d) {
      ref_sweep_f64(dims, n, pitch, d, si, so, gamma, dtdh, flux, limiter, recon, reflect);
      if (dims != 1 && d < dims - 1) std::swap(si, so);
    }
    params.update_simulation_info();
    in = so;
    out = si;
  }
  if (result_in_b) *result_in_b = (in == b);
  if (run_time) *run_time = params.run_time;
  return static_cast<int64_t>(params.iters);
}

}  // extern "C"

// The level-set functors' driver.  The reference's headers define some
// functions outside classes without `inline` (state/state_components.hpp's
// literal operators), so the whole driver is one translation unit.
#include "ref_driver_ls.cpp"
