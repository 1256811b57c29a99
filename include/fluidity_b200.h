/*
 * fluidity_b200.h -- C ABI of the B200-native split-solver step.
 *
 * Drop-in boundary for robclu/fluidity's finite-volume Euler hot path.  Each
 * entry point names the reference interface it replaces (paths relative to
 * the reference's include/fluidity/).  All device buffers belong to the
 * caller; no entry point that launches work allocates memory, except
 * fl_sim_create, which allocates one small control block.
 *
 * Storage.  The reference stores AoS states in a DeviceTensor
 * (container/device_tensor.hpp:34-316).  This library works on
 * structure-of-arrays component planes: component c (order
 * [rho, E, m_x, m_y, m_z], state/state.hpp:88-98) of cell (x, y, z) lives at
 *     base[c * pitch + (z * n[1] + y) * n[0] + x]        (x fastest)
 * fl_aos_to_soa / fl_soa_to_aos convert from and to the reference layout.
 *
 * Errors.  Every call returns an FL_* status and never terminates the process
 * (the reference prints and calls std::terminate, utility/debug.hpp:42-50).
 * fl_last_error_string() describes the last failure on the calling thread.
 *
 * Streams.  Work is enqueued on the given cudaStream_t (passed as void*;
 * NULL = legacy default stream) with no implicit device synchronisation,
 * except in fl_sim_status / fl_simulate, which wait for the stream.
 */
#ifndef FLUIDITY_B200_H
#define FLUIDITY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace fluidity_check_cuda_result, utility/debug.hpp:42-67) */
#define FL_OK        0
#define FL_EINVAL    1   /* invalid argument (sizes, pointers, policy)        */
#define FL_ECUDA     2   /* a CUDA runtime call failed                        */
#define FL_ETIMEOUT  3   /* a bounded wait gave up                            */
#define FL_ENAN      4   /* a wavespeed was not finite (state blew up)        */
#define FL_ENOMEM    5   /* fl_sim_create could not allocate its control      */

/* ---- policy bits: the reference's compile-time policy list
 * SimulatorImpl<data_t, Num<D>, Material, LimitForm, Limiter, Recon, Flux, ...>
 * (simulator/simulator_traits.hpp:41-84), as run-time bits. */
#define FL_DTYPE_F64        0u          /* data_t = double                       */
#define FL_DTYPE_F32        1u          /* data_t = float                        */
#define FL_FLUX_HLLC        (0u << 1)   /* flux::Hllc (flux_method/flux_hllc.hpp)  */
#define FL_FLUX_FORCE       (1u << 1)   /* flux::Force (flux_force.hpp)            */
#define FL_FLUX_LF          (2u << 1)   /* flux::LaxFriedrichs                     */
#define FL_FLUX_RICHTMYER   (3u << 1)   /* flux::Richtmyer                         */
#define FL_LIMITER_VANLEER  (0u << 3)   /* limit::VanLeer<cons_form_t>             */
#define FL_LIMITER_SUPERBEE (1u << 3)   /* limit::Superbee<cons_form_t>            */
#define FL_RECON_MUSCL      (0u << 4)   /* recon::MHReconstructor<Limiter>         */
#define FL_RECON_BASIC      (1u << 4)   /* recon::BasicReconstructor               */
#define FL_NO_FLATTEN       (1u << 5)   /* drop MUSCL's pressure flattening (chi); */
                                        /* not a reference option                  */

/* Grid description.  dims in 1..3, n[d] >= 4 for d < dims (mirror ghosts
 * reach 4 cells deep), n[d] = 1 for d >= dims, pitch >= n[0]*n[1]*n[2]. */
typedef struct fl_grid {
  int32_t dims;
  int64_t n[3];
  int64_t pitch;
} fl_grid;

/* Settings-file dispatch: the "simulator : { data_type : ..., dimensions : ...,
 * limit_form : ..., limiter : ..., material : ..., reconstructor : ...,
 * flux_method : ..., solve_method : ..., execution : ... }" block of a
 * fluidity settings text (Settings::from_string, setting/settings.hpp:50-105;
 * SimulatorParameter, setting/simulator_parameter.hpp:29-105) turned into the
 * policy bits and dimension count that OptionManager::create
 * (setting/option_manager.hpp:241-246) would have turned into a SimulatorImpl
 * type.  Missing entries take SimTraits' defaults (double, one, ideal-gas,
 * conservative, superbee, muscl-hancock, force, split, gpu); choices this
 * library does not build (primitive limit form, void/linear limiters,
 * unsplit) return FL_EINVAL.  Host-only: no device is touched. */
int fl_policy_from_settings(const char* text, uint32_t* policy, int32_t* dims);
int fl_policy_from_settings_file(const char* path, uint32_t* policy, int32_t* dims);

/* Library version (major * 10000 + minor * 100 + patch). */
int fl_version(void);

/* Description of the last failure on the calling thread ("" if none). */
const char* fl_last_error_string(void);

/* Number of bytes of one state buffer: (dims + 2) * pitch * sizeof(T). */
int64_t fl_state_bytes(const fl_grid* grid, uint32_t policy);

/* One dimensional sweep: out = in + dtdh * (F(i-1/2) - F(i+1/2)) along dim,
 * ghosts per boundary_mask (bit d set = reflective ends in dimension d,
 * transmissive otherwise; both ends of a dimension share one setting as in
 * BoundarySetter::bit_index, solver/boundary_loader.hpp:105-111).
 * Replaces solve_dim<SplitSolver> (solver/cuda/split_solver.cuh:39-44) and
 * SplitSolver::invoke (solver/split_solver.hpp:138-162).
 * max_ws_out (nullable, device pointer) receives the maximum wavespeed
 * max_d |u_d| + a of the OUTPUT state -- the fused form of set_wavespeeds +
 * max_element (simulator/cuda/wavespeed_initialization.cuh:85-97,
 * algorithm/max_element.hpp:28-38) for the next step.
 * Allocates nothing.  Strips are scheduled one per warp; 3-D sweeps take the
 * shared-memory tile kernel.  fl_split_sweep_ws (below) takes a workspace
 * and with it schedules strips dynamically and sweeps 3-D grids with the
 * register walk. */
int fl_split_sweep(const fl_grid* grid, int dim, const void* in, void* out,
                   double gamma, double dtdh, uint32_t policy,
                   uint32_t boundary_mask, double* max_ws_out, void* stream);

/* All dims sweeps of one step, x then y then z, with the reference's buffer
 * swap: replaces SplitSolver::solve (solver/split_solver.hpp:105-115) and
 * solve_impl_split (solver/cuda/split_solver.cuh:57-80).  On return *out
 * points at the buffer holding the new state and *in at the other one, just
 * as the reference swaps its iterators.  max_ws_out as for fl_split_sweep. */
int fl_split_solve(const fl_grid* grid, void** in, void** out, double gamma,
                   double dtdh, uint32_t policy, uint32_t boundary_mask,
                   double* max_ws_out, void* stream);

/* Max over cells of max_d |u_d| + a, written to *max_ws_out (device
 * pointer).  Replaces set_wavespeeds + max_element
 * (simulator/cuda/wavespeed_initialization.cuh:41-97, algorithm/reduce.cuh
 * :44-131) without the per-cell wavespeed buffer or the host-side finish. */
int fl_max_wavespeed(const fl_grid* grid, const void* in, double gamma,
                     uint32_t policy, double* max_ws_out, void* stream);

/* Piecewise-constant initial state (SimulatorImpl::fill_data,
 * simulator/simulator_impl.hpp:294-340): 2^dims primitive states
 * (rho, p, v_x, .., host memory, doubles) assigned by orthant
 * (x_d >= 0.5) << d of the cell position float(i_d)/float(n_d), converted to
 * conservative form in the policy's precision. */
int fl_fill_riemann(const fl_grid* grid, const double* states_prim,
                    double gamma, uint32_t policy, void* out, void* stream);

/* ---- materials.  The entry points above take the ideal gas
 * (material/ideal_gas.hpp) by its gamma.  The _mat forms take either of the
 * reference's equations of state: the ideal gas (p_inf = 0) or the stiffened
 * fluid StiffFluid (material/stiff_fluid.hpp:38-133).  For the stiffened
 * fluid:
 *   - the sound speed is sqrt(gamma (p + p_inf) / rho) (stiff_fluid.hpp:92-96);
 *   - a state filled from primitives gets the internal energy
 *     (p + gamma p_inf) / ((gamma - 1) rho) (stiff_fluid.hpp:76-80);
 *   - the pressure of a conservative state is (gamma - 1)(E - rho |v|^2 / 2),
 *     as for the ideal gas (state/state_impl.hpp:117-128).  The reference
 *     subtracts no gamma p_inf there, so pressures read back from a filled
 *     state are p + gamma p_inf.  Fluxes and flattening see that pressure.
 * With p_inf = 0 every _mat form equals its gamma-only form bit for bit.
 * gamma must exceed 1 and p_inf must be finite and >= 0 (else FL_EINVAL). */
typedef struct fl_material {
  double gamma;   /* adiabatic index */
  double p_inf;   /* stiffened fluid's material constant; 0 for the ideal gas */
} fl_material;

int fl_split_sweep_mat(const fl_grid* grid, int dim, const void* in, void* out,
                       const fl_material* mat, double dtdh, uint32_t policy,
                       uint32_t boundary_mask, double* max_ws_out, void* stream);
int fl_split_solve_mat(const fl_grid* grid, void** in, void** out,
                       const fl_material* mat, double dtdh, uint32_t policy,
                       uint32_t boundary_mask, double* max_ws_out, void* stream);
int fl_max_wavespeed_mat(const fl_grid* grid, const void* in, const fl_material* mat,
                         uint32_t policy, double* max_ws_out, void* stream);
int fl_fill_riemann_mat(const fl_grid* grid, const double* states_prim,
                        const fl_material* mat, uint32_t policy, void* out,
                        void* stream);

/* ---- the drop-in step with a workspace --------------------------------
 * Replaces SplitSolver::solve / solve_impl_split (solver/split_solver.hpp
 * :105-115, solver/cuda/split_solver.cuh:57-80) and solve_dim /
 * SplitSolver::invoke (split_solver.cuh:39-44, split_solver.hpp:138-162) as
 * fl_split_sweep / fl_split_solve do, with a caller-owned workspace of
 * fl_workspace_bytes(grid, policy) bytes of device memory, 256-byte aligned:
 * two strip counters and a status word, and for 3-D grids one value per
 * cell of scratch for the register walk's flattening plane.  The calls
 * allocate nothing.  Zero the workspace once before its first use (the
 * status word starts at 0); each sweep clears the strip counter it uses on
 * `stream`, so nothing needs clearing between calls.  Strips are taken dynamically
 * by the CTAs resident on the GPU, as in the device-resident loop.  Sweeps
 * sharing one workspace must be ordered on one stream.  A sweep whose
 * bounded wait for its staged copies gave up leaves FL_ETIMEOUT in the
 * status word (fl_workspace_status); it is never set otherwise. */
int64_t fl_workspace_bytes(const fl_grid* grid, uint32_t policy);
int fl_split_sweep_ws(const fl_grid* grid, int dim, const void* in, void* out,
                      const fl_material* mat, double dtdh, uint32_t policy,
                      uint32_t boundary_mask, double* max_ws_out, void* workspace,
                      void* stream);
int fl_split_solve_ws(const fl_grid* grid, void** in, void** out, const fl_material* mat,
                      double dtdh, uint32_t policy, uint32_t boundary_mask,
                      double* max_ws_out, void* workspace, void* stream);
/* Reads the workspace's status word after `stream` has finished (it
 * synchronises the stream): 0, or FL_ETIMEOUT. */
int fl_workspace_status(const void* workspace, void* stream, int* status);

/* Layout adapters for the reference's AoS DeviceTensor<State, D>
 * (container/device_tensor.hpp): aos holds cells * (dims + 2) values. */
int fl_aos_to_soa(const fl_grid* grid, uint32_t policy, const void* aos,
                  void* soa, void* stream);
int fl_soa_to_aos(const fl_grid* grid, uint32_t policy, const void* soa,
                  void* aos, void* stream);

/* ---- device-resident time loop: SimulatorImpl::simulate
 * (simulator/simulator_impl.hpp:223-258) with sim::Parameters
 * (simulator/parameters.hpp:27-99) kept in HBM.  The CFL reduction is fused
 * into each step's last sweep; the host does not read anything back per step,
 * so a run can be enqueued (or captured into a CUDA graph) in one go. */
typedef struct fl_sim fl_sim;

/* Allocates the control block on the current device. */
int fl_sim_create(fl_sim** sim, const fl_grid* grid, double gamma,
                  uint32_t policy, uint32_t boundary_mask);
int fl_sim_destroy(fl_sim* sim);

/* Sets the loop's material (gamma and p_inf; fl_sim_create's gamma is the
 * ideal gas).  Call before fl_sim_begin. */
int fl_sim_set_material(fl_sim* sim, const fl_material* mat);

/* Resets the loop: buffers a (initial state) and b, cfl, resolution dh,
 * stop time and step limit; enqueues the initial wavespeed reduction. */
int fl_sim_begin(fl_sim* sim, void* a, void* b, double cfl, double res,
                 double sim_time, int64_t max_iters, void* stream);

/* Enqueues nsteps further steps.  Steps after the loop condition fails are
 * launched but do no work. */
int fl_sim_steps(fl_sim* sim, int64_t nsteps, void* stream);

/* ---- simulations from host memory to host memory (no reference
 * counterpart beyond its fill_data / simulate / write_results sequence,
 * simulator/simulator_impl.hpp:223-358).  fl_host_pipe_run runs njobs
 * whole simulations of one grid: host_in[k] (a state laid out as on the
 * device: (dims + 2) planes of `pitch` values) is uploaded, simulated as
 * fl_simulate would, and its result downloaded to host_out[k].  The upload
 * of job k + 1 and the download of job k - 1 overlap job k's compute (three
 * streams; `sets` = 2..4 pairs of device buffers rotate, 3 keeps every
 * overlap free of shared buffers).  Host buffers should be page-locked.
 * iters / run_times (nullable) get each job's step count and time.  Returns
 * after the last download has finished. */
typedef struct fl_host_pipe fl_host_pipe;
int fl_host_pipe_create(fl_host_pipe** pipe, const fl_grid* grid, double gamma,
                        uint32_t policy, uint32_t boundary_mask, int sets);
int fl_host_pipe_destroy(fl_host_pipe* pipe);
int fl_host_pipe_set_material(fl_host_pipe* pipe, const fl_material* mat);
int fl_host_pipe_run(fl_host_pipe* pipe, int32_t njobs, const void* const* host_in,
                     void* const* host_out, double cfl, double res, double sim_time,
                     int64_t max_iters, int64_t* iters, double* run_times);

/* ---- one slab of a grid decomposed across GPUs (no reference counterpart:
 * the reference runs one GPU).  A rank holds its own rows (along the slowest
 * dimension) plus ghost rows that the host refreshes from the neighbouring
 * ranks before every sweep; the CFL maximum is reduced across ranks by the
 * host between the last sweep of a step and fl_sim_finalize. */

/* Rows [row_lo, row_hi) of the slowest dimension are this rank's own; only
 * their cells enter the wavespeed maxima (both 0: every row).  Set before
 * fl_sim_begin. */
int fl_sim_set_rows(fl_sim* sim, int64_t row_lo, int64_t row_hi);

/* on != 0: fl_sim_begin (which zeroes it) and the last sweep of each step
 * only accumulate the max wavespeed, as the bits of a non-negative double,
 * into the caller's 8-byte device word given to fl_sim_set_ws_word; the host
 * reduces that word over ranks (64-bit integer MAX) and then calls
 * fl_sim_finalize, which consumes and clears it. */
int fl_sim_set_external_reduce(fl_sim* sim, int on);
int fl_sim_set_ws_word(fl_sim* sim, void* word);

/* Enqueues sweep `dim` of the current step (dims in order 0, 1, ...), so
 * that the host can exchange ghost rows between sweeps. */
int fl_sim_sweep(fl_sim* sim, int dim, void* stream);

/* From the (reduced) wavespeed word: the next dt and dtdh and, with
 * advance != 0, run_time += dt, iters += 1 and the stop test -- the
 * finalisation the fused reduction otherwise does in its last block. */
int fl_sim_finalize(fl_sim* sim, int advance, void* stream);

/* Waits for the stream and reports the loop state.  *result points at the
 * buffer (a or b) holding the latest state.  Returns FL_ENAN if a wavespeed
 * was not finite. */
int fl_sim_status(fl_sim* sim, void* stream, int64_t* iters, double* run_time,
                  int* done, void** result);

/* ---- the decomposed step below the host (no reference counterpart: the
 * reference runs one GPU).  A slab is a 2-D local grid whose rows
 * [own_lo, own_hi) are its own, with ghost rows facing its neighbours (at
 * least 4 on each side that has one).  fl_slab_steps enqueues whole steps on
 * one stream -- exchange 3 ghost rows, x sweep, exchange 4 ghost rows, y
 * sweep, MAX of the wavespeed over the slabs, finalize -- and reads nothing
 * back, so the steps can be captured in a CUDA graph.  The result equals the
 * undivided run bit for bit.
 *
 * NCCL transport, one rank (process, GPU) per slab: rank 0 makes a 128-byte
 * id with fl_slab_nccl_id and hands it to every rank, which calls
 * fl_slab_create_nccl (collective; world 1 needs no id, and with one makes
 * a communicator of one rank).  The exchange is
 * ncclSend / ncclRecv into local ghost rows, the maximum one 64-bit
 * ncclAllReduce.  libnccl.so.2 is loaded at run time; fl_slab_nccl_available
 * says whether it could be.
 *
 * In-process transport: slabs made with fl_slab_create_local and stepped
 * together, bottom to top, in one fl_slab_begin / fl_slab_steps call (one
 * stream; neighbours are the adjacent array entries; at most 16). */
typedef struct fl_slab fl_slab;
int fl_slab_nccl_available(void);
int fl_slab_nccl_id(void* id);
int fl_slab_create_nccl(fl_slab** slab, const fl_grid* grid, double gamma, uint32_t policy,
                        uint32_t boundary_mask, int64_t own_lo, int64_t own_hi,
                        const void* nccl_id, int world, int rank);
int fl_slab_create_local(fl_slab** slab, const fl_grid* grid, double gamma, uint32_t policy,
                         uint32_t boundary_mask, int64_t own_lo, int64_t own_hi);
int fl_slab_set_material(fl_slab* slab, const fl_material* mat);
/* The slab's time loop, for fl_sim_status. */
int fl_slab_sim(fl_slab* slab, fl_sim** sim);
/* a[i], b[i]: slab i's state buffers (a holds its initial state, ghost rows
 * included); then the initial wavespeed maximum and time step. */
int fl_slab_begin(fl_slab* const* slabs, int count, void* const* a, void* const* b,
                  double cfl, double res, double sim_time, int64_t max_iters, void* stream);
int fl_slab_steps(fl_slab* const* slabs, int count, int64_t nsteps, void* stream);
int fl_slab_destroy(fl_slab* slab);

/* Convenience: begin + steps in chunks until done, like simulate(). */
int fl_simulate(fl_sim* sim, void* a, void* b, double cfl, double res,
                double sim_time, int64_t max_iters, void* stream,
                int64_t* iters, double* run_time, void** result);

/* fl_simulate without any allocation.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc (code that must not touch the CUDA
 * allocator: inside another framework's memory pool, real-time threads,
 * deployments that fix their memory up front).  Instead of the control block
 * of fl_sim_create, the loop uses a fixed 96-byte block in a static device
 * array of the library: one per GPU that loads it, held until the process
 * exits; no grid size needs more.  Same arguments as fl_sim_create +
 * fl_simulate.  1-D and 2-D results are the same as fl_simulate's bit for
 * bit; 3-D sweeps take the shared-memory tile kernel (the register walk
 * needs a scratch plane this entry point cannot allocate), which matches
 * fl_simulate to rounding, not bit for bit.  Every call resolves the
 * array's device address with the caller's device current; the first call
 * on a device may load the library's module there, so make it before any
 * stream capture.  Calls on the same GPU share the block: calls that
 * overlap there (two streams or threads) race. */
int fl_simulate_noalloc(const fl_grid* grid, double gamma, uint32_t policy,
                        uint32_t boundary_mask, void* a, void* b, double cfl, double res,
                        double sim_time, int64_t max_iters, void* stream, int64_t* iters,
                        double* run_time, void** result);


/* ---- batched solver: thousands of independent 1-D / 2-D problems ---------
 * No reference counterpart (the reference solves one grid per simulator);
 * each problem follows the time loop of SimulatorImpl::simulate with its own
 * CFL time step.  Problem states live in caller-owned arenas: problem i's
 * component c (order as above) of cell (x, y) is at
 *     arena[offset_i + c * pitch_i + y * n_i[0] + x].
 * Every result ends in arena_a; arena_b is the 2-D ping-pong partner (same
 * size).  1-D problems run resident in shared memory (n <= 9000 in FP32,
 * 4500 in FP64); 2-D problems run one batched launch per sweep.  HLLC or
 * FORCE; policy and boundary mask apply to all problems. */
typedef struct fl_batch_desc {
  int32_t dims;       /* 1 or 2 */
  int64_t n[2];       /* cells in x, y (n[1] ignored in 1-D) */
  int64_t offset;     /* element offset of the problem's first plane */
  int64_t pitch;      /* elements between the problem's component planes */
  double res;         /* grid spacing dh */
} fl_batch_desc;

typedef struct fl_batch fl_batch;

/* Uploads the problem list; allocates descriptors, per-problem time
 * control and work lists on the current device. */
int fl_batch_create(fl_batch** batch, const fl_batch_desc* problems, int32_t count,
                    double gamma, uint32_t policy, uint32_t boundary_mask);
int fl_batch_destroy(fl_batch* batch);

/* Gives every problem of the batch the material (gamma and p_inf; p_inf > 0
 * the stiffened fluid).  Call before fl_batch_begin; drops a captured graph. */
int fl_batch_set_material(fl_batch* batch, const fl_material* mat);

/* Per-problem initial wavespeed and dt (cfl, stop time, step limit shared). */
int fl_batch_begin(fl_batch* batch, void* arena_a, void* arena_b, double cfl,
                   double sim_time, int64_t max_iters, void* stream);

/* Enqueues nsteps time steps of every problem (1-D resident launches on a
 * side stream, forked from and joined back into `stream`). */
int fl_batch_steps(fl_batch* batch, int64_t nsteps, void* stream);

/* Captures fl_batch_steps(nsteps) into a CUDA graph (after fl_batch_begin,
 * for the arenas given there); fl_batch_launch replays it on `stream`. */
int fl_batch_capture(fl_batch* batch, int64_t nsteps);
int fl_batch_launch(fl_batch* batch, void* stream);

/* Waits for `stream`; per-problem step counts and times (nullable arrays of
 * `count` entries) and the number of finished problems.  FL_ENAN if a
 * problem's wavespeed was not finite. */
int fl_batch_status(fl_batch* batch, void* stream, int64_t* iters, double* run_time,
                    int32_t* done_count);

/* Autotuner: times the 1-D CTA width per size class and the 2-D warp-strip
 * height per size class on copies of the arenas (trial_steps steps each)
 * and keeps the fastest.  Allocates and frees its scratch copies. */
int fl_batch_autotune(fl_batch* batch, void* arena_a, void* arena_b, int64_t trial_steps,
                      void* stream);

/* Current tuning: [1-D CTA widths of classes 0..2, 1-D class bounds (2),
 * 2-D strip rows for small / mid / large sides]; n >= 8. */
int fl_batch_tuning(const fl_batch* batch, int32_t* out, int32_t n);

/* ---- discrete adjoint of the split step ------------------------------------
 * No reference counterpart (the reference has no differentiation).  Reverse
 * mode of the sweep with the HLLC wave region, shock/rarefaction choice,
 * pressure clamp and limiter (minmod) selection frozen at the forward pass,
 * the flattening coefficient chi differentiated through its ramp
 * eta = 1 - (z - 0.75) / 0.1 (its clamps, test and min selection frozen),
 * and the CFL time step frozen.  1-D and 2-D grids, HLLC or FORCE, van Leer
 * limiter.  With flattening on, fl_adjoint_sweep takes its chi records
 * from the stream-ordered pool for the call; fl_adj_create allocates them. */

/* lambda_in = (d sweep / d u_in)^T lambda_out for one dimensional sweep with
 * the given dtdh (u_in: the sweep's input state). */
int fl_adjoint_sweep(const fl_grid* grid, int dim, const void* u_in, const void* lambda_out,
                     void* lambda_in, double gamma, double dtdh, uint32_t policy,
                     uint32_t boundary_mask, void* stream);
/* The same for either material: the stiffened fluid's sound speed
 * sqrt(gamma (p + p_inf) / rho) in the HLLC wave-speed estimates is
 * differentiated with p_inf as a constant (material/stiff_fluid.hpp:92-96). */
int fl_adjoint_sweep_mat(const fl_grid* grid, int dim, const void* u_in,
                         const void* lambda_out, void* lambda_in, const fl_material* mat,
                         double dtdh, uint32_t policy, uint32_t boundary_mask, void* stream);

typedef struct fl_adj fl_adj;

/* Allocates checkpoint storage for nsteps steps with a checkpoint every
 * `interval` steps (<= 0: ceil(sqrt(nsteps))). */
int fl_adj_create(fl_adj** adj, const fl_grid* grid, double gamma, uint32_t policy,
                  uint32_t boundary_mask, int64_t nsteps, int64_t interval);
int fl_adj_destroy(fl_adj* adj);

/* Replaces the material given at creation (gamma and p_inf); the next
 * backward pass needs a new forward pass. */
int fl_adj_set_material(fl_adj* adj, const fl_material* mat);

/* Forward: nsteps steps from u0 into u_final (device), storing checkpoints.
 * frozen_dtdh == NULL: CFL steps (cfl, res) computed on the device and
 * recorded; else a host array of nsteps dt/dh values replayed as given. */
int fl_adj_forward(fl_adj* adj, const void* u0, void* u_final, double cfl, double res,
                   const double* frozen_dtdh, void* stream);

/* The dt/dh of each step of the last forward pass (host array of nsteps). */
int fl_adj_dtdh(const fl_adj* adj, double* out);

/* Backward: lambda_0 = (d u_final / d u0)^T lambda_final, recomputing each
 * checkpoint segment once. */
int fl_adj_backward(fl_adj* adj, const void* lambda_final, void* lambda_0, void* stream);

/* ---- level sets of the multimaterial (ghost-fluid) path ---------------------
 * FP64 level sets on 2-D grids (grid->dims == 2), x fastest, one value per
 * cell; reads outside the domain mirror it.  Each call is asynchronous on
 * `stream` except fl_ls_reinit, which waits for its convergence flag. */

/* Device workspace fl_ls_advect and fl_ls_reinit need (bytes; -1 on a bad
 * grid).  The caller allocates it; the calls never allocate. */
int64_t fl_ls_workspace_bytes(const fl_grid* grid);

/* Interface-normal velocity v = u . grad(phi)/|grad(phi)| of the first of
 * nmat (1 or 2) materials whose level set is <= 0 at the cell, else 0.
 * states[m]: the material's SoA state (rho, E, m_x, m_y; FP32 or FP64 by
 * policy bit 0) with `pitch`.  Replaces the velocity initialisation of
 * levelset/cuda/velocity_initialization.cuh:108-143 (set_velocities). */
int fl_ls_velocity(const fl_grid* grid, int nmat, const double* const* phis,
                   const void* const* states, int64_t pitch, uint32_t policy, double h,
                   double* vel, void* stream);

/* One TVD-RK3 step of phi_t + vel |grad phi| = 0 (WENO-HJ5 derivatives,
 * Godunov upwind Hamiltonian), three launches over the whole grid.
 * Replaces scheme/cuda/evolve.cuh:51-157 with the RK3 updater
 * (scheme/updaters/runge_kutta_3.hpp:110-148).  out != phi. */
int fl_ls_advect(const fl_grid* grid, const double* phi, const double* vel, double dt, double h,
                 double* out, void* workspace, void* stream);

/* a, b <- the two level sets without overlap or void: a -= (a + b) / 2,
 * b = -a.  Replaces levelset/cuda/levelset_projection.cuh:54-67. */
int fl_ls_project(int64_t cells, double* a, double* b, void* stream);

/* Reinitialisation to a signed distance (fast iterative method): cells next
 * to a sign change keep |phi|, every other cell converges to the Godunov
 * eikonal fixed point, the result takes phi's sign.  Active 16x16 tiles,
 * at most max_passes passes (FL_ETIMEOUT beyond); *passes (nullable) gets
 * the count.  Replaces scheme/cuda/fast_iterative_method.cuh:48-112 and its
 * driver (fast_iterative, :366-); the reference seeds sources with the signed
 * phi, here with |phi|, so both sides of the interface relax to distances.
 * out != phi. */
int fl_ls_reinit(const fl_grid* grid, const double* phi, double h, double* out, void* workspace,
                 int max_passes, int* passes, void* stream);

/* ---- two-material ghost-fluid path ------------------------------------------
 * Two materials on one 2-D grid, each with its own SoA state (rho, E, m_x,
 * m_y; FP32 or FP64 by policy bit 0; both with grid->pitch), its own ideal-gas
 * gamma and an FP64 level set (negative inside).  Replaces the
 * MultimaterialSimulator step (simulator/multimaterial_simulator.hpp:254-286),
 * whose own simulate() is not runnable as shipped. */
typedef struct fl_mm fl_mm;

/* Allocates the workspace (interface lists of grid size, the level-set
 * workspace, velocities).  gammas: 2 values; res: the cell size dh. */
int fl_mm_create(fl_mm** mm, const fl_grid* grid, const double* gammas, uint32_t policy,
                 double res);
int fl_mm_destroy(fl_mm* mm);

/* Replaces the two materials (2 entries; fl_mm_create's gammas are ideal
 * gases): an ideal gas or a stiffened fluid per material, as the reference's
 * add_material takes either (validation/1d_mm_shock_tube_gas_water.cu:63-80).
 * The GFM star state uses each side's sound speed
 * (flux_method/flux_hllc.hpp:330-361), the step and the CFL maximum each
 * material's own. */
int fl_mm_set_materials(fl_mm* mm, const fl_material* mats);

/* Ghost cells of both materials (ghost::load_ghost_cells,
 * ghost_fluid/cuda/load_ghost_cells.cuh:74-95): RiemannGFM<3> star states
 * (ghost_fluid/riemann_ghost_fluid.hpp:50-195) written beside the interface,
 * read from the states as they were before the pass, the highest source
 * index winning a shared target; then GhostCellExtrapolator
 * (ghost_fluid/ghost_fluid_extrapolator.hpp:54-202) as Jacobi sweeps over the
 * band dh <= phi <= 6 dh / sqrt(2) until no cell moves by 1e-8, at most
 * max_iters sweeps.  scratch0/1: state-sized buffers whose contents are
 * overwritten in the band. */
int fl_mm_ghost(fl_mm* mm, void* u0, void* u1, void* scratch0, void* scratch1,
                const double* phi0, const double* phi1, int max_iters, void* stream);

/* Counters of the last ghost pass and step: [GFM targets of material 0, 1,
 * band cells 0, 1, extrapolation sweeps 0, 1, reinitialisation passes 0, 1];
 * n >= 8.  Waits for the device. */
int fl_mm_stats(const fl_mm* mm, int32_t* out, int32_t n);

/* Cells with phi <= 0 take the conservative form of prim = (rho, p, v_x, v_y)
 * (state::set_states, state/cuda/state_initialization.cuh:72-119). */
int fl_mm_set_states(const fl_grid* grid, uint32_t policy, void* state, const double* phi,
                     const double* prim, double gamma, void* stream);
int fl_mm_set_states_mat(const fl_grid* grid, uint32_t policy, void* state, const double* phi,
                         const double* prim, const fl_material* mat, void* stream);

/* Cells with phi1 <= 0 copy material 1's state into u0
 * (material::combine_into_first, material/cuda/combine_materials.cuh:39-81). */
int fl_mm_combine(const fl_grid* grid, uint32_t policy, void* u0, const void* u1,
                  const double* phi1, void* stream);

/* Step loop.  u0a/u1a hold the states (and hold them again after every
 * step), u0b/u1b are their second buffers; phi0a/phi1a hold the level sets,
 * phi0b/phi1b are their second buffers (fl_mm_status says which one is
 * current).  Level sets are reinitialised after every reinit_every-th step
 * (0: never; the reference reinitialises every step). */
int fl_mm_begin(fl_mm* mm, void* u0a, void* u0b, void* u1a, void* u1b, double* phi0a,
                double* phi0b, double* phi1a, double* phi1b, double cfl, double sim_time,
                int64_t max_iters, int reinit_every);

/* Runs up to nsteps steps: ghost cells, CFL step over both materials (one
 * 16-byte read-back per step), each material's split step with its own
 * gamma, level-set velocity, advection, projection and reinitialisation.
 * FL_ENAN if a wavespeed is not finite. */
int fl_mm_steps(fl_mm* mm, int64_t nsteps, void* stream);

/* Waits for the stream; steps, simulated time, done flag and the current
 * level-set buffers (nullable outputs). */
int fl_mm_status(fl_mm* mm, void* stream, int64_t* iters, double* run_time, int* done,
                 double** phi0, double** phi1);

#ifdef __cplusplus
}
#endif
#endif /* FLUIDITY_B200_H */
