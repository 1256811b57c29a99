// A stiffened-fluid shock tube through the C++ policy interface: the water
// of the reference's gas-water validation (StiffFluid{4.4}, p_inf = 0.613)
// on [0, 1] with a membrane at 0.5, (rho, p, v_x) = (1, 10, 0) | (1, 1, 0),
// resolution 0.005, CFL 0.9, to t = 0.05.  Writes the final primitive state
// to argv[1].dat.
#include <cstdio>

#include "fluidity_b200/fluidity.hpp"

using namespace fluid;
using real_t = double;
using simulator_t =
    sim::SimulatorImpl<real_t, Num<1>, material::StiffFluid<real_t>, limit::cons_form_t,
                       limit::VanLeer, recon::MHReconstructor, flux::Hllc>;

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <output prefix>\n", argv[0]);
    return 2;
  }
  try {
    simulator_t simulator;
    simulator.configure_material(material::StiffFluid<real_t>{4.4});
    simulator.configure_resolution(0.005);
    simulator.configure_dimension(0, 0.0, 1.0);
    simulator.configure_sim_time(0.05);
    simulator.configure_cfl(0.9);
    simulator.fill_data({
        {"rho", [](const float*) { return 1.0; }},
        {"p", [](const float* pos) { return pos[0] < 0.5f ? 10.0 : 1.0; }},
        {"v_x", [](const float*) { return 0.0; }},
    });
    simulator.simulate();
    simulator.write_results(argv[1]);
    std::printf("iterations %lld run_time %.17g\n", (long long)simulator.iterations(),
                simulator.run_time());
  } catch (const fluid::Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}
