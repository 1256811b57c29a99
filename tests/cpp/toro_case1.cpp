// Toro's test 1 (Sod-like shock tube) through the C++ policy interface, set up
// the way the reference's validation/1d_toro_case_1_validation.cu does:
// resolution 0.0025 on [0, 1], membrane at 0.3, sim_time 0.2, CFL 0.9.
// Writes the final primitive state to argv[1].dat and, one file per
// variable, to argv[1]_raw_<name>_0.200000.dat.
#include <cstdio>
#include <string>

#include "fluidity_b200/fluidity.hpp"

using namespace fluid;
using real_t = double;
using simulator_t =
    sim::SimulatorImpl<real_t, Num<1>, material::IdealGas<real_t>, limit::cons_form_t,
                       limit::VanLeer, recon::MHReconstructor, flux::Hllc>;

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <output prefix>\n", argv[0]);
    return 2;
  }
  try {
    simulator_t simulator;
    simulator.configure_resolution(0.0025);
    simulator.configure_dimension(0, 0.0, 1.0);
    simulator.configure_sim_time(0.2);
    simulator.configure_cfl(0.9);
    constexpr real_t membrane = 0.3;
    simulator.fill_data({
        {"rho", [](const float* pos) { return pos[0] < membrane ? 1.0 : 0.125; }},
        {"p", [](const float* pos) { return pos[0] < membrane ? 1.0 : 0.1; }},
        {"v_x", [](const float* pos) { return pos[0] < membrane ? 0.75 : 0.0; }},
    });
    simulator.simulate();
    simulator.write_results(argv[1]);
    simulator.write_results_separate_raw(std::string(argv[1]) + "_raw");
    std::printf("iterations %lld run_time %.17g\n", (long long)simulator.iterations(),
                simulator.run_time());
  } catch (const fluid::Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}
