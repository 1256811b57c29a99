// fluidity.hpp -- C++ template-policy interface of the B200 split solver.
//
// Mirrors the reference's policy types and simulator interface
// (robclu/fluidity include/fluidity/...) so that code written against
//   fluid::sim::SimulatorImpl<T, Num<D>, IdealGas<T>, cons_form_t,
//                             VanLeer<cons_form_t>, MHReconstructor<...>, Hllc>
// reads the same here.  The policy types carry no arithmetic: they resolve,
// at compile time, to the policy bits of the C ABI (include/fluidity_b200.h),
// and every numerical operation runs in libfluidity_b200.so on the GPU.
// Header-only; link with -lfluidity_b200 -lcudart.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <functional>
#include <stdexcept>
#include <string>
#include <utility>
#include <memory>
#include <vector>

#include "../fluidity_b200.h"

namespace fluid {

// ---- errors -----------------------------------------------------------------

// A C-ABI call failed; carries the FL_* status.  (The reference prints and
// calls std::terminate, utility/debug.hpp:42-50.)
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

inline void check(int rc) {
  if (rc != FL_OK) throw Error(rc, std::string("fluidity_b200: ") + fl_last_error_string());
}

inline void check_cuda(cudaError_t e) {
  if (e != cudaSuccess) throw Error(FL_ECUDA, cudaGetErrorString(e));
}

// ---- dimensions (dimension/dimension.hpp:48-93) ------------------------------

template <std::size_t V>
struct Num {
  static constexpr std::size_t value = V;
  constexpr operator std::size_t() const { return V; }
};

template <std::size_t V>
struct Dimension {
  static constexpr std::size_t value = V;
  constexpr operator std::size_t() const { return V; }
};
using dimx_t = Dimension<0>;
using dimy_t = Dimension<1>;
using dimz_t = Dimension<2>;
static constexpr dimx_t dim_x{};
static constexpr dimy_t dim_y{};
static constexpr dimz_t dim_z{};

// ---- state (state/state.hpp:449-466) -----------------------------------------

namespace state {
enum class FormType { primitive = 0, conservative = 1 };
template <typename T, std::size_t D, FormType F>
struct StateTag {
  using value_t = T;
  static constexpr std::size_t dimensions = D;
  static constexpr std::size_t elements = D + 2;
  static constexpr FormType format = F;
};
template <typename T, std::size_t D>
using primitive_t = StateTag<T, D, FormType::primitive>;
template <typename T, std::size_t D>
using conservative_t = StateTag<T, D, FormType::conservative>;
}  // namespace state

// ---- materials (material/ideal_gas.hpp:27-119, material/stiff_fluid.hpp:38-133) ----

namespace material {
template <typename T>
struct IdealGas {
  using value_t = T;
  constexpr IdealGas() = default;
  constexpr explicit IdealGas(T adi) : adi_index(adi) {}
  constexpr T adiabatic() const { return adi_index; }
  constexpr T p_inf() const { return T(0); }
  T adi_index = T(1.4);
};

// Stiffened fluid: sound speed sqrt(gamma (p + p_inf) / rho), filled energy
// (p + gamma p_inf) / ((gamma - 1) rho).  Defaults and the one-argument
// constructor keep the reference's p_inf = 0.613 (and gamma = 5.5).
template <typename T>
struct StiffFluid {
  using value_t = T;
  constexpr StiffFluid() = default;
  constexpr explicit StiffFluid(T adi) : adi_index(adi) {}
  constexpr StiffFluid(T adi, T pinf) : adi_index(adi), p_inf_(pinf) {}
  constexpr T adiabatic() const { return adi_index; }
  constexpr T p_inf() const { return p_inf_; }
  T adi_index = T(5.5);
  T p_inf_ = T(0.613);
};

template <typename Mat>
fl_material to_fl(const Mat& m) {
  return fl_material{(double)m.adiabatic(), (double)m.p_inf()};
}
}  // namespace material

// ---- limiters (limiting/) -----------------------------------------------------

namespace limit {
template <state::FormType F>
struct LimitForm {
  static constexpr state::FormType form = F;
};
using cons_form_t = LimitForm<state::FormType::conservative>;

template <typename Form>
struct VanLeer {
  static_assert(Form::form == state::FormType::conservative,
                "the B200 solver limits conservative differences (cons_form_t)");
  static constexpr uint32_t bits = FL_LIMITER_VANLEER;
  static constexpr std::size_t width = 4;  // limiter_traits.hpp:96-110
};
template <typename Form>
struct Superbee {
  static_assert(Form::form == state::FormType::conservative,
                "the B200 solver limits conservative differences (cons_form_t)");
  static constexpr uint32_t bits = FL_LIMITER_SUPERBEE;
  static constexpr std::size_t width = 4;
};
}  // namespace limit

// ---- reconstruction (reconstruction/) --------------------------------------------

namespace recon {
template <typename Limiter>
struct MHReconstructor {
  using limiter_t = Limiter;
  static constexpr uint32_t bits = FL_RECON_MUSCL | Limiter::bits;
  static constexpr std::size_t width = Limiter::width;
};
template <typename Limiter>
struct BasicReconstructor {
  using limiter_t = Limiter;
  static constexpr uint32_t bits = FL_RECON_BASIC | Limiter::bits;
  static constexpr std::size_t width = 1;
};
}  // namespace recon

// ---- flux methods (flux_method/) ---------------------------------------------------

namespace flux {
struct Hllc { static constexpr uint32_t bits = FL_FLUX_HLLC; };
struct Force { static constexpr uint32_t bits = FL_FLUX_FORCE; };
struct LaxFriedrichs { static constexpr uint32_t bits = FL_FLUX_LF; };
struct Richtmyer { static constexpr uint32_t bits = FL_FLUX_RICHTMYER; };
}  // namespace flux

template <typename T>
constexpr uint32_t dtype_bits() {
  static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value,
                "data_t must be float or double");
  return std::is_same<T, double>::value ? FL_DTYPE_F64 : FL_DTYPE_F32;
}

// ---- device storage -----------------------------------------------------------------

// Owning SoA device buffer of conservative states (replaces the AoS
// DeviceTensor<State, D> of container/device_tensor.hpp:34-316).
template <typename T, std::size_t D>
class DeviceStates {
 public:
  DeviceStates() = default;
  explicit DeviceStates(const fl_grid& g) { resize(g); }
  DeviceStates(const DeviceStates&) = delete;
  DeviceStates& operator=(const DeviceStates&) = delete;
  DeviceStates(DeviceStates&& o) noexcept { swap(o); }
  DeviceStates& operator=(DeviceStates&& o) noexcept { swap(o); return *this; }
  ~DeviceStates() { if (ptr_) cudaFree(ptr_); }

  void resize(const fl_grid& g) {
    if (ptr_) cudaFree(ptr_);
    ptr_ = nullptr;
    grid_ = g;
    check_cuda(cudaMalloc(&ptr_, bytes()));
  }
  std::size_t bytes() const { return (D + 2) * (std::size_t)grid_.pitch * sizeof(T); }
  T* data() { return ptr_; }
  const T* data() const { return ptr_; }
  const fl_grid& grid() const { return grid_; }
  void swap(DeviceStates& o) noexcept { std::swap(ptr_, o.ptr_); std::swap(grid_, o.grid_); }

  // Host copy, SoA planes (D + 2) x pitch.
  std::vector<T> as_host() const {
    std::vector<T> h((D + 2) * (std::size_t)grid_.pitch);
    check_cuda(cudaMemcpy(h.data(), ptr_, bytes(), cudaMemcpyDeviceToHost));
    return h;
  }

 private:
  T* ptr_ = nullptr;
  fl_grid grid_{};
};

// ---- solver (solver/) ----------------------------------------------------------------

namespace solver {

enum class BoundaryKind { transmissive = 0, reflective = 1 };
enum class BoundaryIndex { first = 0, second = 1 };

// BoundarySetter (solver/boundary_loader.hpp:42-124): one setting per
// dimension, shared by both of its ends, as the reference's bit_index does.
struct BoundarySetter {
  template <typename Dim>
  void configure(Dim dim, BoundaryIndex, BoundaryKind kind) {
    const uint32_t bit = 1u << static_cast<std::size_t>(dim);
    mask = kind == BoundaryKind::reflective ? (mask | bit) : (mask & ~bit);
  }
  uint32_t mask = 0;
};

template <std::size_t Padding>
struct BoundaryLoader {
  static constexpr std::size_t padding = Padding;
};

template <typename Recon, typename Flux, typename Eos>
struct FaceFlux {
  using reconstructor_t = Recon;
  using flux_method_t = Flux;
  using eos_t = Eos;
  using value_t = typename Eos::value_t;
  static constexpr uint32_t bits = dtype_bits<value_t>() | Recon::bits | Flux::bits;
};

// SplitSolver<FaceFlux, Loader, Num<D>> (solver/split_solver.hpp:37-233).
template <typename FaceFluxT, typename Loader, typename Dims = Num<1>>
struct SplitSolver {
  using flux_solver_t = FaceFluxT;
  using value_t = typename FaceFluxT::value_t;
  static constexpr std::size_t num_dimensions = Dims::value;
  static constexpr std::size_t padding = Loader::padding;
  static constexpr uint32_t policy = FaceFluxT::bits;

  // solve(in, out, mat, dtdh, setter): all sweeps, x -> y -> z, swapping in
  // and out between sweeps like split_solver.cuh:67-79; afterwards `out`
  // refers to the new state.  stream defaults to the legacy stream.  The
  // step itself allocates nothing: the solver keeps one workspace
  // (fl_workspace_bytes; strip counters, and in 3-D the flattening plane),
  // allocated on the first solve for that grid and shared by copies of the
  // solver; solves sharing it must be ordered on one stream.
  template <typename Mat>
  void solve(DeviceStates<value_t, num_dimensions>& in,
             DeviceStates<value_t, num_dimensions>& out, const Mat& mat, value_t dtdh,
             const BoundarySetter& setter, cudaStream_t stream = nullptr,
             double* max_ws_out = nullptr) const {
    void* pin = in.data();
    void* pout = out.data();
    const fl_material m = material::to_fl(mat);
    check(fl_split_solve_ws(&in.grid(), &pin, &pout, &m, (double)dtdh, policy, setter.mask,
                            max_ws_out, workspace(in.grid()), stream));
    if (pout != out.data()) in.swap(out);
  }

 private:
  void* workspace(const fl_grid& g) const {
    const int64_t bytes = fl_workspace_bytes(&g, policy);
    if (bytes < 0) throw std::runtime_error(fl_last_error_string());
    if (!ws_ || ws_bytes_ < bytes) {
      void* p = nullptr;
      check_cuda(cudaMalloc(&p, (std::size_t)bytes));
      ws_ = std::shared_ptr<void>(p, [](void* q) { cudaFree(q); });
      check_cuda(cudaMemset(p, 0, (std::size_t)bytes));
      ws_bytes_ = bytes;
    }
    return ws_.get();
  }
  mutable std::shared_ptr<void> ws_;
  mutable int64_t ws_bytes_ = 0;
};

}  // namespace solver

// ---- simulator (simulator/) -------------------------------------------------------------

namespace sim {

// Filler: (name, f(pos) -> value); values are assigned by ORDER to
// (rho, p, v_x, v_y, v_z), as SimulatorImpl::fill_data does
// (simulator_impl.hpp:328-333); names are only checked.
struct FillInfo {
  const char* data_name;
  std::function<double(const float*)> filler;
};

// SimulatorImpl<data_t, Num<D>, Material, LimitForm, Limiter, Recon, Flux>
// (simulator/simulator_impl.hpp:43-512; positional policy list of
// simulator_traits.hpp:61-84).  Recon is a template template parameter
// taking the limiter, as the reference's MHReconstructor<Limiter>.
template <typename T, typename Dims, typename Material, typename LimitForm,
          template <typename> class Limiter, template <typename> class Recon, typename Flux>
class SimulatorImpl {
 public:
  static constexpr std::size_t dimensions = Dims::value;
  using value_t = T;
  using limiter_t = Limiter<LimitForm>;
  using recon_t = Recon<limiter_t>;
  using face_flux_t = solver::FaceFlux<recon_t, Flux, Material>;
  using solver_t = solver::SplitSolver<face_flux_t, solver::BoundaryLoader<limiter_t::width>, Dims>;
  static constexpr uint32_t policy = face_flux_t::bits;

  SimulatorImpl() : extent_(dimensions, {0.0, 1.0}) {}
  ~SimulatorImpl() { if (sim_) fl_sim_destroy(sim_); }

  void configure_cfl(double cfl) { cfl_ = cfl; }
  void configure_dimension(std::size_t dim, double start, double end) {
    extent_.at(dim) = {start, end};
  }
  void configure_resolution(double res) { res_ = res; }
  void configure_sim_time(double t) { sim_time_ = t; }
  void configure_max_iterations(std::size_t n) { max_iters_ = (int64_t)n; }
  void configure_boundary(const solver::BoundarySetter& s) { setter_ = s; }
  void configure_material(const Material& m) { mat_ = m; }

  // Domain::elements (simulator/domain.hpp:69-73).
  std::size_t elements(std::size_t dim) const {
    return static_cast<std::size_t>((extent_[dim].second - extent_[dim].first) / res_);
  }

  fl_grid grid() const {
    fl_grid g{};
    g.dims = (int32_t)dimensions;
    int64_t cells = 1;
    for (std::size_t d = 0; d < 3; ++d) {
      g.n[d] = d < dimensions ? (int64_t)elements(d) : 1;
      cells *= g.n[d];
    }
    g.pitch = cells;
    return g;
  }

  // fill_data (simulator_impl.hpp:294-340): host evaluation of the fillers
  // at pos[d] = float(i_d) / float(N_d), then one upload.
  void fill_data(std::vector<FillInfo>&& fillers) {
    if (fillers.size() != dimensions + 2)
      throw Error(FL_EINVAL, "fill_data needs one filler per primitive element");
    const fl_grid g = grid();
    const int64_t cells = g.n[0] * g.n[1] * g.n[2];
    std::vector<T> host((dimensions + 2) * (std::size_t)g.pitch);
    const T gm = mat_.adiabatic();
    const T pinf = mat_.p_inf();
    float pos[3] = {0.f, 0.f, 0.f};
    for (int64_t i = 0; i < cells; ++i) {
      const int64_t c[3] = {i % g.n[0], (i / g.n[0]) % g.n[1], i / (g.n[0] * g.n[1])};
      for (std::size_t d = 0; d < dimensions; ++d) pos[d] = float(c[d]) / float(g.n[d]);
      T prim[5];
      for (std::size_t k = 0; k < dimensions + 2; ++k) prim[k] = (T)fillers[k].filler(pos);
      // primitive -> conservative (state_impl.hpp:390-406), e from the eos
      // (ideal_gas.hpp:59-63; stiff_fluid.hpp:76-80)
      T v2 = T(0);
      for (std::size_t d = 0; d < dimensions; ++d) v2 += prim[2 + d] * prim[2 + d];
      const T e = (prim[1] + gm * pinf) / ((gm - T(1)) * prim[0]);
      host[0 * g.pitch + i] = prim[0];
      host[1 * g.pitch + i] = prim[0] * (T(0.5) * v2 + e);
      for (std::size_t d = 0; d < dimensions; ++d) host[(2 + d) * g.pitch + i] = prim[2 + d] * prim[0];
    }
    a_.resize(g);
    b_.resize(g);
    check_cuda(cudaMemcpy(a_.data(), host.data(), a_.bytes(), cudaMemcpyHostToDevice));
    result_ = &a_;
  }

  // simulate (simulator_impl.hpp:223-258) with the time control on the device.
  void simulate(cudaStream_t stream = nullptr) {
    if (result_ == nullptr) throw Error(FL_EINVAL, "fill_data must be called before simulate");
    if (sim_ == nullptr) {
      fl_grid g = grid();
      check(fl_sim_create(&sim_, &g, (double)mat_.adiabatic(), policy, setter_.mask));
    }
    const fl_material m = material::to_fl(mat_);
    check(fl_sim_set_material(sim_, &m));
    void* res = nullptr;
    check(fl_simulate(sim_, a_.data(), b_.data(), cfl_, res_, sim_time_, max_iters_, stream,
                      &iters_, &run_time_, &res));
    result_ = (res == a_.data()) ? &a_ : &b_;
  }

  const DeviceStates<T, dimensions>& states() const { return *result_; }
  int64_t iterations() const { return iters_; }
  double run_time() const { return run_time_; }

  // write_results (simulator_impl.hpp:350-358, 436-508): ASCII columns of
  // cell-centre position(s) and primitive variables.
  void write_results(const std::string& prefix) const {
    const fl_grid g = grid();
    const auto h = result_->as_host();
    std::ofstream f(prefix + ".dat");
    f.precision(17);
    const int64_t cells = g.n[0] * g.n[1] * g.n[2];
    const T gm = mat_.adiabatic();
    for (int64_t i = 0; i < cells; ++i) {
      const int64_t c[3] = {i % g.n[0], (i / g.n[0]) % g.n[1], i / (g.n[0] * g.n[1])};
      for (std::size_t d = 0; d < dimensions; ++d)
        f << (extent_[d].first + (c[d] + 0.5) * res_) << ' ';
      const T rho = h[i];
      T v2 = 0;
      T v[3] = {0, 0, 0};
      for (std::size_t d = 0; d < dimensions; ++d) {
        v[d] = h[(2 + d) * g.pitch + i] / rho;
        v2 += v[d] * v[d];
      }
      const T p = (gm - T(1)) * (h[g.pitch + i] - T(0.5) * rho * v2);
      f << rho << ' ' << p;
      for (std::size_t d = 0; d < dimensions; ++d) f << ' ' << v[d];
      f << '\n';
    }
  }

  // write_results_separate_raw (simulator_impl.hpp:360-420): one file per
  // primitive variable, <prefix>_<name>_<sim_time>.dat with the stream's
  // default formatting; 1-D: the values on one line then a blank line;
  // 2-D: one line per row of x values; 3-D: the 2-D files of each z plane
  // under <prefix>_<z>.
  void write_results_separate_raw(const std::string& prefix) const {
    const fl_grid g = grid();
    const auto h = result_->as_host();
    const T gm = mat_.adiabatic();
    const char* names[5] = {"rho", "p", "v_x", "v_y", "v_z"};
    const int nz = dimensions == 3 ? (int)g.n[2] : 1;
    for (int z = 0; z < nz; ++z) {
      const std::string pre = dimensions == 3 ? prefix + "_" + std::to_string(z) : prefix;
      std::vector<std::ofstream> streams;
      for (std::size_t k = 0; k < dimensions + 2; ++k)
        streams.emplace_back(pre + "_" + names[k] + "_" + std::to_string(sim_time_) + ".dat");
      const int64_t ny = dimensions >= 2 ? g.n[1] : 1;
      for (int64_t y = 0; y < ny; ++y) {
        for (int64_t x = 0; x < g.n[0]; ++x) {
          const int64_t i = ((int64_t)z * g.n[1] + y) * g.n[0] + x;
          const T rho = h[i];
          T v2 = 0;
          T v[3] = {0, 0, 0};
          for (std::size_t d = 0; d < dimensions; ++d) {
            v[d] = h[(2 + d) * g.pitch + i] / rho;
            v2 += v[d] * v[d];
          }
          const T p = (gm - T(1)) * (h[g.pitch + i] - T(0.5) * rho * v2);
          streams[0] << rho << " ";
          streams[1] << p << " ";
          for (std::size_t d = 0; d < dimensions; ++d) streams[2 + d] << v[d] << " ";
        }
        for (auto& st : streams) st << "\n";
      }
      if (dimensions == 1)
        for (auto& st : streams) st << "\n";
    }
  }

 private:
  Material mat_{};
  solver::BoundarySetter setter_{};
  std::vector<std::pair<double, double>> extent_;
  double res_ = 0.0, sim_time_ = 0.0, cfl_ = 0.9;
  int64_t max_iters_ = INT64_MAX;
  int64_t iters_ = 0;
  double run_time_ = 0.0;
  DeviceStates<T, dimensions> a_, b_;
  const DeviceStates<T, dimensions>* result_ = nullptr;
  fl_sim* sim_ = nullptr;
};

}  // namespace sim
}  // namespace fluid
