// fl_internal.cuh -- device-side structures shared by the kernels and the
// C-ABI layer.
#pragma once

#include <cstdint>

namespace fl {

// Device-resident time control of one simulation (the state of
// sim::Parameters, simulator/parameters.hpp:27-99, kept in HBM so that a whole
// run can be launched, or captured in a CUDA graph, without host round trips).
// Values are stored as double; an FP32 run rounds them through float exactly
// where the reference's Parameters<float> would.
struct StepControl {
  double dt;          // time step of the step in flight
  double dtdh;        // dt / dh of the step in flight
  double run_time;    // accumulated simulated time
  double sim_time;    // stop when run_time >= sim_time
  double cfl;
  double res;         // grid spacing dh
  long long iters;    // completed steps
  long long max_iters;
  unsigned long long ws_bits;  // max wavespeed (double bits) of the state being produced
  unsigned int arrive;         // blocks of the finishing sweep that have arrived
  int done;                    // 1 once the loop condition fails
  int is_f32;                  // round dt, dtdh and run_time through float
  int status;                  // 0, or FL_ENAN when a wavespeed was not finite
  // strip counters of the dynamically scheduled walks, one per sweep
  // parity: a sweep takes strips from walk_next[slot] and clears the other
  unsigned int walk_next[2];
};

// Parameters of one dimensional sweep.
struct SweepParams {
  const void* in;
  void* out;
  int64_t pitch;          // elements between component planes
  int64_t n[3];           // cells per dimension (x fastest); unused = 1
  double gamma;
  double pinf;            // stiffened fluid's p_inf; kernels read it when FLUX has kStiffEos
  double dtdh;            // used when ctrl == nullptr
  int limiter;            // LimiterKind
  int basic;              // 1: piecewise-constant reconstruction
  int flatten;            // 1: slope flattening (chi) on
  uint32_t reflect;       // bit d: reflective ends in dimension d
  StepControl* ctrl;      // nullable: take dtdh / done from the control block
  unsigned long long* ws_accum;  // nullable: max wavespeed of the output (double bits)
  int finalize;           // 1: last sweep of a step; the last block advances ctrl
  // rows (index along the slowest dimension) whose cells enter the fused
  // max wavespeed: [ws_lo, ws_hi); every row when ws_hi <= ws_lo.  A slab
  // of a decomposed grid counts its own rows, not its ghost rows.
  int64_t ws_lo, ws_hi;
  // nullable: a plane of cell-count values of the sweep's type, scratch for
  // the 3-D walk (without it 3-D sweeps take the tile kernel)
  void* scratch;
  // nullable: two strip counters (StepControl::walk_next or the like); with
  // them the walk schedules its strips dynamically, taking them from
  // walk_next[walk_slot] and clearing the other counter for the next sweep
  unsigned int* walk_next;
  int walk_slot;
  int walk_ry;  // rows per strip of a dynamically scheduled 2-D walk (0: the compiled length)
  // nullable: a kernel whose bounded wait on its own copies gave up writes
  // kETimeout here (and stops the loop through ctrl->done when ctrl is set)
  int* status;
  // 2-D only: compute the output rows [row_lo, row_hi) of the slowest
  // dimension only (reads reach beyond as usual); every row when
  // row_hi <= row_lo.  Taken by the register walk and, for the y sweep, the
  // staged walk.
  int64_t row_lo, row_hi;
  // 2-D only, 1: the sweep of the layout-alternating loop.  `in` holds the
  // state with the sweep dimension slowest (x sweep: y fastest; y sweep:
  // x fastest) and `out` receives it transposed (x sweep: x fastest; y
  // sweep: y fastest).  Both layouts keep the planes `pitch` apart.
  int transposed;
};

}  // namespace fl

typedef struct fl_sim fl_sim;

namespace fl {

// One part of sweep `dim` of the current step of a 2-D fl_sim loop in its
// external-reduction mode: output rows [row_lo, row_hi) of the slowest
// dimension (nothing is launched for an empty range), strips taken from the
// two counters `counters` (slot `slot`; nullptr: the static grid).  The
// part with last_part set ends the sweep (the loop's cursor moves on).
// Defined in fl_api.cu; the slab step splits each sweep into parts.
int sim_sweep_part(fl_sim* sim, int dim, int64_t row_lo, int64_t row_hi, unsigned int* counters,
                   int slot, int last_part, void* stream);

// Tensor map of one SoA state buffer for the TMA-staged sweeps: a 3-D
// tensor (x, y, component plane) of n0 x n1 x planes elements with rows n0
// and planes `pitch` elements apart, boxes of box0 x box1 x planes.
// Returns 0, or an error status with the message recorded.  Defined in
// fl_tmap.cu; maps are cached per (address, shape, box).
int encode_state_map(void* map, const void* base, int64_t n0, int64_t n1, int64_t pitch,
                     int planes, int elem, int box0, int box1);


__host__ __device__ __forceinline__ bool ws_row_counts(const SweepParams& p, int64_t row) {
  return p.ws_hi <= p.ws_lo || (row >= p.ws_lo && row < p.ws_hi);
}

// Status codes, mirrored by include/fluidity_b200.h.
enum : int {
  kOk = 0,
  kEInval = 1,
  kECuda = 2,
  kETimeout = 3,
  kENan = 4,
  kENoMem = 5,
};

// Records the message returned by fl_last_error_string() (thread-local) and
// returns code.  Defined in fl_api.cu.
int set_error(int code, const char* fmt, ...);

}  // namespace fl
