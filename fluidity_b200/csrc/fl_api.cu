// fl_api.cu -- C ABI of the split-solver step (include/fluidity_b200.h):
// argument checking, status codes, the wavespeed / fill / layout kernels and
// the device-resident time loop.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"
#include "fl_launch.cuh"
#include "fl_numerics.cuh"
#include "fl_sweep.cuh"

namespace fl {
namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

}  // namespace

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

namespace {

int cuda_fail(cudaError_t e, const char* where) {
  snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
  return kECuda;
}

struct Policy {
  bool f32;
  int flux;
  int limiter;
  int basic;
  int flatten;
};

Policy decode(uint32_t policy) {
  Policy p;
  p.f32 = (policy & 1u) != 0;
  p.flux = (int)((policy >> 1) & 3u);
  p.limiter = (int)((policy >> 3) & 1u);
  p.basic = (int)((policy >> 4) & 1u);
  p.flatten = ((policy >> 5) & 1u) ? 0 : 1;
  return p;
}

int check_grid(const fl_grid* g) {
  if (g == nullptr) return fail(kEInval, "grid is NULL");
  if (g->dims < 1 || g->dims > 3) return fail(kEInval, "dims must be 1..3 (got %d)", (int)g->dims);
  int64_t cells = 1;
  for (int d = 0; d < 3; ++d) {
    if (d < g->dims) {
      if (g->n[d] < 4)
        return fail(kEInval, "n[%d] must be >= 4 (got %lld)", d, (long long)g->n[d]);
    } else if (g->n[d] != 1) {
      return fail(kEInval, "n[%d] must be 1 beyond dims (got %lld)", d, (long long)g->n[d]);
    }
    cells *= g->n[d];
  }
  if (g->pitch < cells) return fail(kEInval, "pitch %lld smaller than the cell count %lld", (long long)g->pitch, (long long)cells);
  if ((uint64_t)g->n[1] > 65535ull * 64 || (uint64_t)g->n[2] > 65535ull * 4)
    return fail(kEInval, "grid too large in y or z");
  return kOk;
}

int check_policy(uint32_t policy) {
  if (policy & ~0x3fu) return fail(kEInval, "unknown policy bits (0x%x)", (unsigned)policy);
  return kOk;
}

int check_material(const fl_material* m) {
  if (m == nullptr) return fail(kEInval, "material is NULL");
  if (!(m->gamma > 1.0)) return fail(kEInval, "gamma must exceed 1");
  if (!(m->p_inf >= 0.0) || m->p_inf > DBL_MAX) return fail(kEInval, "p_inf must be finite and >= 0");
  return kOk;
}

size_t elem_size(const Policy& p) { return p.f32 ? sizeof(float) : sizeof(double); }

SweepParams make_params(const fl_grid* g, const Policy& pol, double gamma, double pinf,
                        double dtdh, uint32_t boundary) {
  SweepParams p;
  memset(&p, 0, sizeof(p));
  p.pitch = g->pitch;
  for (int d = 0; d < 3; ++d) p.n[d] = g->n[d];
  p.gamma = gamma;
  p.pinf = pinf;
  p.dtdh = dtdh;
  p.limiter = pol.limiter;
  p.basic = pol.basic;
  p.flatten = pol.flatten;
  p.reflect = boundary;
  return p;
}

cudaError_t launch_sweep(const SweepParams& p, const Policy& pol, int dims, int dim,
                         cudaStream_t st) {
  return pol.f32 ? launch_sweep_f32(p, dims, dim, pol.flux, st)
                 : launch_sweep_f64(p, dims, dim, pol.flux, st);
}

// ---- wavespeed reduction (set_wavespeeds + max_element) -----------------

template <typename T, int D>
__global__ void __launch_bounds__(256) wavespeed_kernel(const T* __restrict__ in, int64_t pitch,
                                                        int64_t cells, T gamma, T pinf,
                                                        unsigned long long* accum,
                                                        StepControl* ctrl) {
  __shared__ double s_red[8];
  double local = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells;
       i += (int64_t)gridDim.x * blockDim.x) {
    Cons<T, D> u;
#pragma unroll
    for (int c = 0; c < D + 2; ++c) u.v[c] = __ldg(in + c * pitch + i);
    // p + p_inf under the root; p_inf = 0 leaves the ideal gas's value
    ws_max(local, (double)max_wavespeed<true>(u, gamma, pinf));
  }
  cta_wavespeed_commit<256>(local, accum, ctrl, ctrl != nullptr ? 1 : 0, false, s_red);
}

template <typename T>
cudaError_t launch_wavespeed(const fl_grid* g, const void* in, double gamma, double pinf,
                             unsigned long long* accum, StepControl* ctrl, cudaStream_t st) {
  const int64_t cells = g->n[0] * g->n[1] * g->n[2];
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t blocks = (cells + 255) / 256;
  if (blocks > (int64_t)sms * 8) blocks = (int64_t)sms * 8;
  if (blocks < 1) blocks = 1;
  const T* p = static_cast<const T*>(in);
  switch (g->dims) {
    case 1: wavespeed_kernel<T, 1><<<(unsigned)blocks, 256, 0, st>>>(p, g->pitch, cells, (T)gamma, (T)pinf, accum, ctrl); break;
    case 2: wavespeed_kernel<T, 2><<<(unsigned)blocks, 256, 0, st>>>(p, g->pitch, cells, (T)gamma, (T)pinf, accum, ctrl); break;
    default: wavespeed_kernel<T, 3><<<(unsigned)blocks, 256, 0, st>>>(p, g->pitch, cells, (T)gamma, (T)pinf, accum, ctrl); break;
  }
  return cudaGetLastError();
}

// ---- initial state -------------------------------------------------------

template <typename T>
struct RiemannStates {
  T s[8][5];
};

template <typename T>
__global__ void fill_riemann_kernel(T* __restrict__ out, int64_t pitch, int64_t n0, int64_t n1,
                                    int64_t n2, int dims, RiemannStates<T> st) {
  const int64_t cells = n0 * n1 * n2;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c[3] = {i % n0, (i / n0) % n1, i / (n0 * n1)};
    const int64_t n[3] = {n0, n1, n2};
    int s = 0;
    for (int d = 0; d < dims; ++d) {
      // pos[d] = float(i_d) / N_d in float (simulator_impl.hpp:324)
      const float pos = __fdiv_rn((float)c[d], (float)n[d]);
      if (!((double)pos < 0.5)) s |= 1 << d;
    }
    for (int k = 0; k < dims + 2; ++k) out[k * pitch + i] = st.s[s][k];
  }
}

template <typename T>
void prim_to_cons_host(int D, const double* prim_d, T gamma, T pinf, T* cons) {
  // state_impl.hpp:390-406 (energy 136-142, eos ideal_gas.hpp:59-63 and
  // stiff_fluid.hpp:76-80: e = (p + gamma p_inf) / ((gamma - 1) rho); p_inf = 0
  // gives the ideal gas's value exactly)
  T prim[5];
  for (int k = 0; k < D + 2; ++k) prim[k] = (T)prim_d[k];
  // host code is compiled with -ffp-contract=off: every product is rounded
  T v2 = T(0);
  for (int d = 0; d < D; ++d) v2 += prim[2 + d] * prim[2 + d];
  const T e = (prim[1] + gamma * pinf) / ((gamma - T(1)) * prim[0]);
  cons[0] = prim[0];
  cons[1] = prim[0] * (T(0.5) * v2 + e);
  for (int d = 0; d < D; ++d) cons[2 + d] = prim[2 + d] * prim[0];
}

template <typename T>
cudaError_t launch_fill(const fl_grid* g, const double* states, double gamma, double pinf,
                        void* out, cudaStream_t st) {
  RiemannStates<T> rs;
  memset(&rs, 0, sizeof(rs));
  const int D = g->dims;
  for (int s = 0; s < (1 << D); ++s)
    prim_to_cons_host<T>(D, states + s * (D + 2), (T)gamma, (T)pinf, rs.s[s]);
  const int64_t cells = g->n[0] * g->n[1] * g->n[2];
  int64_t blocks = (cells + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  fill_riemann_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(static_cast<T*>(out), g->pitch, g->n[0],
                                                           g->n[1], g->n[2], D, rs);
  return cudaGetLastError();
}

// ---- AoS <-> SoA -----------------------------------------------------------

template <typename T>
__global__ void aos_soa_kernel(const T* __restrict__ src, T* __restrict__ dst, int64_t cells,
                               int nc, int64_t pitch, int to_soa) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells * nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (to_soa) {
      const int64_t cell = i / nc, c = i % nc;
      dst[c * pitch + cell] = src[i];
    } else {
      const int64_t cell = i / nc, c = i % nc;
      dst[i] = src[c * pitch + cell];
    }
  }
}

template <typename T>
cudaError_t launch_layout(const fl_grid* g, const void* src, void* dst, int to_soa,
                          cudaStream_t st) {
  const int64_t cells = g->n[0] * g->n[1] * g->n[2];
  int64_t blocks = (cells * (g->dims + 2) + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  aos_soa_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(static_cast<const T*>(src),
                                                      static_cast<T*>(dst), cells, g->dims + 2,
                                                      g->pitch, to_soa);
  return cudaGetLastError();
}

// ---- time control ----------------------------------------------------------

// Takes the reduced max wavespeed from `word` (when given; it is then reset
// for the next accumulation) and finalises the step.
__global__ void finalize_kernel(StepControl* c, unsigned long long* word, int advance) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (word != nullptr) {
      c->ws_bits = *word;
      *word = 0ull;
    }
    if (!c->done) finalize_control(c, advance != 0);
  }
}

// Transposes every component plane of a 2-D state: plane c of `in` holds
// ns rows of nf cells (nf fastest), plane c of `out` receives nf rows of ns
// cells; planes are `pitch` elements apart in both.  32 x 32 tiles through
// shared memory, so that both the loads and the stores are coalesced.
template <typename T>
__global__ void __launch_bounds__(256) transpose_planes_kernel(const T* __restrict__ in,
                                                               T* __restrict__ out, int64_t pitch,
                                                               int64_t nf, int64_t ns) {
  __shared__ T tile[32][33];
  const T* src = in + (int64_t)blockIdx.z * pitch;
  T* dst = out + (int64_t)blockIdx.z * pitch;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t f0 = (int64_t)blockIdx.x * 32;
  for (int64_t s0 = (int64_t)blockIdx.y * 32; s0 < ns; s0 += (int64_t)gridDim.y * 32) {
    for (int i = ty; i < 32; i += 8) {
      const int64_t sr = s0 + i, f = f0 + tx;
      if (sr < ns && f < nf) tile[i][tx] = src[sr * nf + f];
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
      const int64_t f = f0 + i, sr = s0 + tx;
      if (f < nf && sr < ns) dst[f * ns + sr] = tile[tx][i];
    }
    __syncthreads();
  }
}

template <typename T>
cudaError_t launch_transpose(const void* in, void* out, int64_t pitch, int64_t nf, int64_t ns,
                             cudaStream_t st) {
  const int64_t gy = (ns + 31) / 32;
  const dim3 grid((unsigned)((nf + 31) / 32), (unsigned)(gy < 65535 ? gy : 65535), 4);
  transpose_planes_kernel<T><<<grid, dim3(32, 8), 0, st>>>(static_cast<const T*>(in),
                                                          static_cast<T*>(out), pitch, nf, ns);
  return cudaGetLastError();
}

__global__ void init_control_kernel(StepControl* c, double cfl, double res, double sim_time,
                                    long long max_iters, int is_f32) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    c->dt = 0.0;
    c->dtdh = 0.0;
    c->run_time = 0.0;
    c->sim_time = is_f32 ? (double)(float)sim_time : sim_time;
    c->cfl = is_f32 ? (double)(float)cfl : cfl;
    c->res = res;
    c->iters = 0;
    c->max_iters = max_iters;
    c->ws_bits = 0ull;
    c->arrive = 0u;
    c->done = 0;
    c->is_f32 = is_f32;
    c->status = 0;
    c->walk_next[0] = 0u;
    c->walk_next[1] = 0u;
  }
}

}  // namespace
}  // namespace fl

struct fl_sim {
  fl_grid grid;
  fl::Policy pol;
  uint32_t policy;
  double gamma;
  double pinf;             // stiffened fluid's p_inf (0: ideal gas)
  uint32_t boundary;
  int device;
  fl::StepControl* ctrl;   // device
  void* a;
  void* b;
  int64_t enqueued;        // steps enqueued since fl_sim_begin
  int64_t own_lo, own_hi;  // rows (slowest index) counted in wavespeeds; all if hi <= lo
  int external;            // 1: the host reduces the wavespeed word and calls fl_sim_finalize
  unsigned long long* ws_word;  // external: the caller's device word (else ctrl->ws_bits)
  int cursor;              // next sweep of the current step (fl_sim_sweep)
  void* scratch;           // 3-D: the walk's chi plane (else nullptr)
  // a counted sweep failed to launch: it neither took its strips nor
  // cleared the other counter, so both are re-zeroed before the next sweep
  int counters_dirty;
};

using namespace fl;

namespace {

// Re-zeroes both strip counters of sim's control block on the stream when a
// counted sweep failed before (the failed launch cleared neither).
int settle_counters(fl_sim* sim, cudaStream_t st, const char* where) {
  if (!sim->counters_dirty) return kOk;
  cudaError_t e = cudaMemsetAsync(sim->ctrl->walk_next, 0, sizeof(sim->ctrl->walk_next), st);
  if (e != cudaSuccess) return cuda_fail(e, where);
  sim->counters_dirty = 0;
  return kOk;
}

}  // namespace

extern "C" {

int fl_version(void) { return 100; }

const char* fl_last_error_string(void) { return g_err; }

int64_t fl_state_bytes(const fl_grid* grid, uint32_t policy) {
  if (check_grid(grid) != kOk) return -1;
  return (int64_t)(grid->dims + 2) * grid->pitch * (int64_t)elem_size(decode(policy));
}

}  // extern "C"

namespace fl {
int split_sweep_counted(const fl_grid* grid, int dim, const void* in, void* out,
                        const fl_material* mat, double dtdh, uint32_t policy,
                        uint32_t boundary_mask, double* max_ws_out, unsigned int* walk_next,
                        int walk_slot, void* stream, void* scratch = nullptr,
                        int* status = nullptr);

// Workspace of the drop-in sweep (fl_workspace_bytes): two strip counters and
// a status word in the first 256 bytes, then, for 3-D grids, the register
// walk's chi plane (one value per cell).
constexpr size_t kWsHead = 256;
struct WorkspaceHead {
  unsigned int walk_next[2];
  int status;
};
}  // namespace fl

extern "C" {

int fl_split_sweep_mat(const fl_grid* grid, int dim, const void* in, void* out,
                       const fl_material* mat, double dtdh, uint32_t policy,
                       uint32_t boundary_mask, double* max_ws_out, void* stream) {
  return fl::split_sweep_counted(grid, dim, in, out, mat, dtdh, policy, boundary_mask,
                                 max_ws_out, nullptr, 0, stream);
}

}  // extern "C"

namespace fl {

// fl_split_sweep_mat with strip counters (nullable) and their parity slot
// (the two-material loop owns a pair), the 3-D walk's chi plane (nullable:
// without it 3-D sweeps take the tile kernel) and a status word (nullable).
// Allocates nothing.
int split_sweep_counted(const fl_grid* grid, int dim, const void* in, void* out,
                        const fl_material* mat, double dtdh, uint32_t policy,
                        uint32_t boundary_mask, double* max_ws_out, unsigned int* walk_next,
                        int walk_slot, void* stream, void* scratch, int* status) {
  int rc = check_grid(grid);
  if (rc) return rc;
  if ((rc = check_policy(policy))) return rc;
  if (dim < 0 || dim >= grid->dims) return fail(kEInval, "dim %d out of range", dim);
  if (in == nullptr || out == nullptr) return fail(kEInval, "NULL state buffer");
  if (in == out) return fail(kEInval, "in and out must differ");
  if ((rc = check_material(mat))) return rc;
  if (boundary_mask >> grid->dims) return fail(kEInval, "boundary_mask has bits beyond dims");
  const Policy pol = decode(policy);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SweepParams p = make_params(grid, pol, mat->gamma, mat->p_inf, dtdh, boundary_mask);
  p.in = in;
  p.out = out;
  p.walk_next = walk_next;
  p.walk_slot = walk_slot;
  if (max_ws_out != nullptr) {
    cudaError_t e = cudaMemsetAsync(max_ws_out, 0, sizeof(double), st);
    if (e != cudaSuccess) return cuda_fail(e, "fl_split_sweep");
    p.ws_accum = reinterpret_cast<unsigned long long*>(max_ws_out);
  }
  p.scratch = (grid->dims == 3) ? scratch : nullptr;
  p.status = status;
  cudaError_t e = launch_sweep(p, pol, grid->dims, dim, st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_split_sweep");
  return kOk;
}

// The drop-in sweep with a caller's workspace: the counter it takes strips
// from is cleared on the stream first, so that calls need no parity of
// their own.
int split_sweep_ws(const fl_grid* grid, int dim, const void* in, void* out,
                   const fl_material* mat, double dtdh, uint32_t policy, uint32_t boundary_mask,
                   double* max_ws_out, void* workspace, void* stream) {
  if (workspace == nullptr) return fail(kEInval, "workspace is NULL");
  if (reinterpret_cast<uintptr_t>(workspace) & 255u)
    return fail(kEInval, "workspace must be 256-byte aligned");
  int rc = check_grid(grid);
  if (rc) return rc;
  auto* head = static_cast<WorkspaceHead*>(workspace);
  cudaError_t e = cudaMemsetAsync(&head->walk_next[0], 0, sizeof(unsigned int),
                                  static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "fl_split_sweep_ws");
  void* plane = (grid->dims == 3) ? static_cast<char*>(workspace) + kWsHead : nullptr;
  return split_sweep_counted(grid, dim, in, out, mat, dtdh, policy, boundary_mask, max_ws_out,
                             head->walk_next, 0, stream, plane, &head->status);
}

}  // namespace fl

extern "C" {

int fl_split_sweep(const fl_grid* grid, int dim, const void* in, void* out, double gamma,
                   double dtdh, uint32_t policy, uint32_t boundary_mask, double* max_ws_out,
                   void* stream) {
  const fl_material mat{gamma, 0.0};
  return fl_split_sweep_mat(grid, dim, in, out, &mat, dtdh, policy, boundary_mask, max_ws_out,
                            stream);
}

int fl_split_solve_mat(const fl_grid* grid, void** in, void** out, const fl_material* mat,
                       double dtdh, uint32_t policy, uint32_t boundary_mask, double* max_ws_out,
                       void* stream) {
  if (in == nullptr || out == nullptr) return fail(kEInval, "NULL buffer handle");
  int rc = check_grid(grid);
  if (rc) return rc;
  // split_solver.cuh:67-79: sweep x, y, z; swap between sweeps
  for (int d = 0; d < grid->dims; ++d) {
    double* ws = (d == grid->dims - 1) ? max_ws_out : nullptr;
    rc = fl_split_sweep_mat(grid, d, *in, *out, mat, dtdh, policy, boundary_mask, ws, stream);
    if (rc) return rc;
    if (grid->dims != 1 && d < grid->dims - 1) {
      void* t = *in;
      *in = *out;
      *out = t;
    }
  }
  return kOk;
}

int fl_split_solve(const fl_grid* grid, void** in, void** out, double gamma, double dtdh,
                   uint32_t policy, uint32_t boundary_mask, double* max_ws_out, void* stream) {
  const fl_material mat{gamma, 0.0};
  return fl_split_solve_mat(grid, in, out, &mat, dtdh, policy, boundary_mask, max_ws_out, stream);
}

int64_t fl_workspace_bytes(const fl_grid* grid, uint32_t policy) {
  if (check_grid(grid) != kOk || check_policy(policy) != kOk) return -1;
  int64_t bytes = (int64_t)kWsHead;
  if (grid->dims == 3)
    bytes += (grid->n[0] * grid->n[1] * grid->n[2] * (int64_t)elem_size(decode(policy)) + 255) /
             256 * 256;
  return bytes;
}

int fl_split_sweep_ws(const fl_grid* grid, int dim, const void* in, void* out,
                      const fl_material* mat, double dtdh, uint32_t policy,
                      uint32_t boundary_mask, double* max_ws_out, void* workspace,
                      void* stream) {
  return fl::split_sweep_ws(grid, dim, in, out, mat, dtdh, policy, boundary_mask, max_ws_out,
                            workspace, stream);
}

int fl_split_solve_ws(const fl_grid* grid, void** in, void** out, const fl_material* mat,
                      double dtdh, uint32_t policy, uint32_t boundary_mask, double* max_ws_out,
                      void* workspace, void* stream) {
  if (in == nullptr || out == nullptr) return fail(kEInval, "NULL buffer handle");
  int rc = check_grid(grid);
  if (rc) return rc;
  for (int d = 0; d < grid->dims; ++d) {
    double* ws = (d == grid->dims - 1) ? max_ws_out : nullptr;
    rc = fl::split_sweep_ws(grid, d, *in, *out, mat, dtdh, policy, boundary_mask, ws, workspace,
                            stream);
    if (rc) return rc;
    if (grid->dims != 1 && d < grid->dims - 1) {
      void* t = *in;
      *in = *out;
      *out = t;
    }
  }
  return kOk;
}

int fl_workspace_status(const void* workspace, void* stream, int* status) {
  if (workspace == nullptr || status == nullptr) return fail(kEInval, "NULL argument");
  int h = 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(&h, &static_cast<const WorkspaceHead*>(workspace)->status,
                                  sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_workspace_status");
  *status = h;
  return kOk;
}

int fl_max_wavespeed_mat(const fl_grid* grid, const void* in, const fl_material* mat,
                         uint32_t policy, double* max_ws_out, void* stream) {
  int rc = check_grid(grid);
  if (rc) return rc;
  if ((rc = check_policy(policy))) return rc;
  if ((rc = check_material(mat))) return rc;
  if (in == nullptr || max_ws_out == nullptr) return fail(kEInval, "NULL pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(max_ws_out, 0, sizeof(double), st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_max_wavespeed");
  auto* acc = reinterpret_cast<unsigned long long*>(max_ws_out);
  const double g = mat->gamma, pi = mat->p_inf;
  e = decode(policy).f32 ? launch_wavespeed<float>(grid, in, g, pi, acc, nullptr, st)
                         : launch_wavespeed<double>(grid, in, g, pi, acc, nullptr, st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_max_wavespeed");
  return kOk;
}

int fl_max_wavespeed(const fl_grid* grid, const void* in, double gamma, uint32_t policy,
                     double* max_ws_out, void* stream) {
  const fl_material mat{gamma, 0.0};
  return fl_max_wavespeed_mat(grid, in, &mat, policy, max_ws_out, stream);
}

int fl_fill_riemann_mat(const fl_grid* grid, const double* states_prim, const fl_material* mat,
                        uint32_t policy, void* out, void* stream) {
  int rc = check_grid(grid);
  if (rc) return rc;
  if ((rc = check_policy(policy))) return rc;
  if ((rc = check_material(mat))) return rc;
  if (states_prim == nullptr || out == nullptr) return fail(kEInval, "NULL pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double g = mat->gamma, pi = mat->p_inf;
  cudaError_t e = decode(policy).f32 ? launch_fill<float>(grid, states_prim, g, pi, out, st)
                                     : launch_fill<double>(grid, states_prim, g, pi, out, st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_fill_riemann");
  return kOk;
}

int fl_fill_riemann(const fl_grid* grid, const double* states_prim, double gamma,
                    uint32_t policy, void* out, void* stream) {
  const fl_material mat{gamma, 0.0};
  return fl_fill_riemann_mat(grid, states_prim, &mat, policy, out, stream);
}

int fl_aos_to_soa(const fl_grid* grid, uint32_t policy, const void* aos, void* soa,
                  void* stream) {
  int rc = check_grid(grid);
  if (rc) return rc;
  if (aos == nullptr || soa == nullptr) return fail(kEInval, "NULL pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = decode(policy).f32 ? launch_layout<float>(grid, aos, soa, 1, st)
                                     : launch_layout<double>(grid, aos, soa, 1, st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_aos_to_soa");
  return kOk;
}

int fl_soa_to_aos(const fl_grid* grid, uint32_t policy, const void* soa, void* aos,
                  void* stream) {
  int rc = check_grid(grid);
  if (rc) return rc;
  if (aos == nullptr || soa == nullptr) return fail(kEInval, "NULL pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = decode(policy).f32 ? launch_layout<float>(grid, soa, aos, 0, st)
                                     : launch_layout<double>(grid, soa, aos, 0, st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_soa_to_aos");
  return kOk;
}

int fl_sim_create(fl_sim** sim, const fl_grid* grid, double gamma, uint32_t policy,
                  uint32_t boundary_mask) {
  if (sim == nullptr) return fail(kEInval, "sim is NULL");
  *sim = nullptr;
  int rc = check_grid(grid);
  if (rc) return rc;
  if ((rc = check_policy(policy))) return rc;
  if (!(gamma > 1.0)) return fail(kEInval, "gamma must exceed 1");
  if (boundary_mask >> grid->dims) return fail(kEInval, "boundary_mask has bits beyond dims");
  fl_sim* s = new (std::nothrow) fl_sim;
  if (s == nullptr) return fail(kENoMem, "out of host memory");
  memset(s, 0, sizeof(*s));
  s->grid = *grid;
  s->pol = decode(policy);
  s->policy = policy;
  s->gamma = gamma;
  s->boundary = boundary_mask;
  cudaGetDevice(&s->device);
  cudaError_t e = cudaMalloc(&s->ctrl, sizeof(StepControl));
  if (e != cudaSuccess) {
    delete s;
    return fail(kENoMem, "cudaMalloc of the control block failed: %s", cudaGetErrorString(e));
  }
  if (grid->dims == 3) {
    const size_t bytes = (size_t)(grid->n[0] * grid->n[1] * grid->n[2]) * elem_size(s->pol);
    e = cudaMalloc(&s->scratch, bytes);
    if (e != cudaSuccess) {
      cudaFree(s->ctrl);
      delete s;
      return fail(kENoMem, "cudaMalloc of the 3-D scratch plane failed: %s",
                  cudaGetErrorString(e));
    }
  }
  e = cudaMemset(s->ctrl, 0, sizeof(StepControl));
  if (e != cudaSuccess) {
    cudaFree(s->ctrl);
    delete s;
    return cuda_fail(e, "fl_sim_create");
  }
  *sim = s;
  return kOk;
}

int fl_sim_destroy(fl_sim* sim) {
  if (sim == nullptr) return kOk;
  if (sim->scratch != nullptr) cudaFree(sim->scratch);
  cudaError_t e = cudaFree(sim->ctrl);
  delete sim;
  if (e != cudaSuccess) return cuda_fail(e, "fl_sim_destroy");
  return kOk;
}

int fl_sim_begin(fl_sim* sim, void* a, void* b, double cfl, double res, double sim_time,
                 int64_t max_iters, void* stream) {
  if (sim == nullptr || a == nullptr || b == nullptr || a == b)
    return fail(kEInval, "invalid sim or buffers");
  if (!(cfl > 0.0) || !(res > 0.0) || max_iters < 0)
    return fail(kEInval, "cfl and res must be positive, max_iters >= 0");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  sim->a = a;
  sim->b = b;
  sim->enqueued = 0;
  init_control_kernel<<<1, 32, 0, st>>>(sim->ctrl, cfl, res, sim_time, (long long)max_iters,
                                        sim->pol.f32 ? 1 : 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fl_sim_begin");
  sim->counters_dirty = 0;  // the control block's initialisation zeroes both counters
  sim->cursor = 0;
  if (sim->external && sim->ws_word == nullptr)
    return fail(kEInval, "external reduction needs fl_sim_set_ws_word");
  auto* acc = sim->external ? sim->ws_word : &sim->ctrl->ws_bits;
  if (sim->external) {
    e = cudaMemsetAsync(acc, 0, sizeof(*acc), st);
    if (e != cudaSuccess) return cuda_fail(e, "fl_sim_begin");
  }
  // own rows only: a view of the grid that starts at row own_lo
  fl_grid view = sim->grid;
  const void* base = a;
  if (sim->own_hi > sim->own_lo) {
    const int slow = sim->grid.dims - 1;
    int64_t row_cells = 1;
    for (int d = 0; d < slow; ++d) row_cells *= sim->grid.n[d];
    view.n[slow] = sim->own_hi - sim->own_lo;
    base = static_cast<const char*>(a) + sim->own_lo * row_cells * (int64_t)elem_size(sim->pol);
  }
  StepControl* fin = sim->external ? nullptr : sim->ctrl;
  e = sim->pol.f32 ? launch_wavespeed<float>(&view, base, sim->gamma, sim->pinf, acc, fin, st)
                   : launch_wavespeed<double>(&view, base, sim->gamma, sim->pinf, acc, fin, st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_sim_begin");
  return kOk;
}

int fl_sim_steps(fl_sim* sim, int64_t nsteps, void* stream) {
  if (sim == nullptr || sim->a == nullptr) return fail(kEInval, "fl_sim_begin not called");
  if (nsteps < 0) return fail(kEInval, "nsteps < 0");
  if (sim->external) return fail(kEInval, "external reduction: step with fl_sim_sweep");
  if (sim->cursor != 0) return fail(kEInval, "a step is half done (fl_sim_sweep)");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = settle_counters(sim, st, "fl_sim_steps");
  if (rc) return rc;
  const int D = sim->grid.dims;
  SweepParams p = make_params(&sim->grid, sim->pol, sim->gamma, sim->pinf, 0.0, sim->boundary);
  p.ctrl = sim->ctrl;
  p.ws_lo = sim->own_lo;
  p.ws_hi = sim->own_hi;
  p.scratch = sim->scratch;
  p.status = &sim->ctrl->status;
  if (D == 2 && nsteps > 0) {
    // The layout-alternating loop: the state goes from buffer a (x fastest)
    // into buffer b with y fastest; each x sweep reads b and writes a (x
    // fastest), each y sweep reads a and writes b (y fastest), so that both
    // sweeps walk along their input's slow dimension; after the last step
    // buffer a receives the state in the caller's layout again.
    SweepParams probe = p;
    probe.in = sim->a;
    probe.out = sim->b;
    const bool tl = sim->pol.f32 ? loop_transposes_f32(probe, sim->pol.flux)
                                 : loop_transposes_f64(probe, sim->pol.flux);
    if (tl) {
      const int64_t n0 = sim->grid.n[0], n1 = sim->grid.n[1], pt = sim->grid.pitch;
      cudaError_t e = sim->pol.f32 ? launch_transpose<float>(sim->a, sim->b, pt, n0, n1, st)
                                   : launch_transpose<double>(sim->a, sim->b, pt, n0, n1, st);
      if (e != cudaSuccess) return cuda_fail(e, "fl_sim_steps");
      p.transposed = 1;
      for (int64_t k = 0; k < nsteps; ++k) {
        for (int d = 0; d < 2; ++d) {
          p.in = (d == 0) ? sim->b : sim->a;
          p.out = (d == 0) ? sim->a : sim->b;
          p.walk_next = sim->ctrl->walk_next;
          p.walk_slot = (int)((sim->enqueued * 2 + d) & 1);
          p.ws_accum = (d == 1) ? &sim->ctrl->ws_bits : nullptr;
          p.finalize = (d == 1) ? 1 : 0;
          e = launch_sweep(p, sim->pol, 2, d, st);
          if (e != cudaSuccess) {
            sim->counters_dirty = 1;
            return cuda_fail(e, "fl_sim_steps");
          }
        }
        sim->enqueued += 1;
      }
      e = sim->pol.f32 ? launch_transpose<float>(sim->b, sim->a, pt, n1, n0, st)
                       : launch_transpose<double>(sim->b, sim->a, pt, n1, n0, st);
      if (e != cudaSuccess) return cuda_fail(e, "fl_sim_steps");
      return kOk;
    }
  }
  for (int64_t k = 0; k < nsteps; ++k) {
    // input of this step: for even D the state returns to buffer a every
    // step; for odd D it alternates a, b, a, ...
    const bool from_b = (D % 2 == 1) && ((sim->enqueued & 1) == 1);
    void* si = from_b ? sim->b : sim->a;
    void* so = from_b ? sim->a : sim->b;
    for (int d = 0; d < D; ++d) {
      p.in = si;
      p.out = so;
      p.walk_next = sim->ctrl->walk_next;
      p.walk_slot = (int)((sim->enqueued * D + d) & 1);
      const bool last = (d == D - 1);
      p.ws_accum = last ? &sim->ctrl->ws_bits : nullptr;
      p.finalize = last ? 1 : 0;
      cudaError_t e = launch_sweep(p, sim->pol, D, d, st);
      if (e != cudaSuccess) {
        sim->counters_dirty = 1;
        return cuda_fail(e, "fl_sim_steps");
      }
      if (D != 1 && d < D - 1) {
        void* t = si;
        si = so;
        so = t;
      }
    }
    sim->enqueued += 1;
  }
  return kOk;
}

int fl_sim_set_material(fl_sim* sim, const fl_material* mat) {
  if (sim == nullptr) return fail(kEInval, "sim is NULL");
  int rc = check_material(mat);
  if (rc) return rc;
  sim->gamma = mat->gamma;
  sim->pinf = mat->p_inf;
  return kOk;
}

int fl_sim_set_rows(fl_sim* sim, int64_t row_lo, int64_t row_hi) {
  if (sim == nullptr) return fail(kEInval, "sim is NULL");
  const int64_t n = sim->grid.n[sim->grid.dims - 1];
  if (!(row_lo == 0 && row_hi == 0) && !(0 <= row_lo && row_lo < row_hi && row_hi <= n))
    return fail(kEInval, "rows [%lld, %lld) outside [0, %lld)", (long long)row_lo,
                (long long)row_hi, (long long)n);
  sim->own_lo = row_lo;
  sim->own_hi = row_hi;
  return kOk;
}

int fl_sim_set_external_reduce(fl_sim* sim, int on) {
  if (sim == nullptr) return fail(kEInval, "sim is NULL");
  sim->external = on ? 1 : 0;
  return kOk;
}

int fl_sim_set_ws_word(fl_sim* sim, void* word) {
  if (sim == nullptr) return fail(kEInval, "sim is NULL");
  if (word != nullptr && (reinterpret_cast<uintptr_t>(word) & 7u))
    return fail(kEInval, "the wavespeed word must be 8-byte aligned");
  sim->ws_word = static_cast<unsigned long long*>(word);
  return kOk;
}

int fl_sim_sweep(fl_sim* sim, int dim, void* stream) {
  if (sim == nullptr || sim->a == nullptr) return fail(kEInval, "fl_sim_begin not called");
  const int D = sim->grid.dims;
  if (dim != sim->cursor) return fail(kEInval, "sweep %d expected, %d given", sim->cursor, dim);
  int rc = settle_counters(sim, static_cast<cudaStream_t>(stream), "fl_sim_sweep");
  if (rc) return rc;
  const bool from_b = (D % 2 == 1) && ((sim->enqueued & 1) == 1);
  void* si = from_b ? sim->b : sim->a;
  void* so = from_b ? sim->a : sim->b;
  if (D != 1 && (dim & 1)) {  // sweeps alternate direction between the buffers
    void* t = si;
    si = so;
    so = t;
  }
  SweepParams p = make_params(&sim->grid, sim->pol, sim->gamma, sim->pinf, 0.0, sim->boundary);
  p.ctrl = sim->ctrl;
  p.ws_lo = sim->own_lo;
  p.ws_hi = sim->own_hi;
  p.scratch = sim->scratch;
  p.walk_next = sim->ctrl->walk_next;
  p.walk_slot = (int)((sim->enqueued * D + dim) & 1);
  p.status = &sim->ctrl->status;
  p.in = si;
  p.out = so;
  const bool last = (dim == D - 1);
  p.ws_accum = last ? (sim->external ? sim->ws_word : &sim->ctrl->ws_bits) : nullptr;
  p.finalize = (last && !sim->external) ? 1 : 0;
  cudaError_t e = launch_sweep(p, sim->pol, D, dim, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    sim->counters_dirty = 1;
    return cuda_fail(e, "fl_sim_sweep");
  }
  if (last) {
    sim->cursor = 0;
    sim->enqueued += 1;
  } else {
    sim->cursor = dim + 1;
  }
  return kOk;
}

}  // extern "C"

namespace fl {

int sim_sweep_part(fl_sim* sim, int dim, int64_t row_lo, int64_t row_hi, unsigned int* counters,
                   int slot, int last_part, void* stream) {
  if (sim == nullptr || sim->a == nullptr) return fail(kEInval, "fl_sim_begin not called");
  if (sim->grid.dims != 2) return fail(kEInval, "sweep parts are 2-D");
  if (!sim->external) return fail(kEInval, "sweep parts need the external reduction");
  if (dim != sim->cursor) return fail(kEInval, "sweep %d expected, %d given", sim->cursor, dim);
  if (row_lo < 0 || row_hi > sim->grid.n[1])
    return fail(kEInval, "rows [%lld, %lld) outside the grid", (long long)row_lo,
                (long long)row_hi);
  if (row_lo < row_hi) {
    void* si = (dim & 1) ? sim->b : sim->a;
    void* so = (dim & 1) ? sim->a : sim->b;
    SweepParams p = make_params(&sim->grid, sim->pol, sim->gamma, sim->pinf, 0.0, sim->boundary);
    p.ctrl = sim->ctrl;
    p.ws_lo = sim->own_lo;
    p.ws_hi = sim->own_hi;
    p.walk_next = counters;
    p.walk_slot = slot;
    p.status = &sim->ctrl->status;
    p.in = si;
    p.out = so;
    p.row_lo = row_lo;
    p.row_hi = row_hi;
    p.ws_accum = (dim == 1) ? (sim->external ? sim->ws_word : &sim->ctrl->ws_bits) : nullptr;
    p.finalize = 0;
    cudaError_t e = launch_sweep(p, sim->pol, 2, dim, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "fl_slab sweep");
  }
  if (last_part) {
    if (dim == 1) {
      sim->cursor = 0;
      sim->enqueued += 1;
    } else {
      sim->cursor = dim + 1;
    }
  }
  return kOk;
}

}  // namespace fl

extern "C" {

int fl_sim_finalize(fl_sim* sim, int advance, void* stream) {
  if (sim == nullptr) return fail(kEInval, "sim is NULL");
  finalize_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(
      sim->ctrl, sim->external ? sim->ws_word : nullptr, advance);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fl_sim_finalize");
  return kOk;
}

int fl_sim_status(fl_sim* sim, void* stream, int64_t* iters, double* run_time, int* done,
                  void** result) {
  if (sim == nullptr) return fail(kEInval, "sim is NULL");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  StepControl h;
  cudaError_t e = cudaMemcpyAsync(&h, sim->ctrl, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "fl_sim_status");
  if (iters) *iters = h.iters;
  if (run_time) *run_time = h.run_time;
  if (done) *done = h.done;
  if (result) {
    const bool in_b = (sim->grid.dims % 2 == 1) && (h.iters & 1);
    *result = in_b ? sim->b : sim->a;
  }
  if (h.status == kENan) return fail(kENan, "non-finite wavespeed after step %lld", (long long)h.iters);
  if (h.status == kETimeout)
    return fail(kETimeout, "a sweep's wait for its staged copies gave up after step %lld",
                (long long)h.iters);
  return kOk;
}

int fl_simulate(fl_sim* sim, void* a, void* b, double cfl, double res, double sim_time,
                int64_t max_iters, void* stream, int64_t* iters, double* run_time,
                void** result) {
  int rc = fl_sim_begin(sim, a, b, cfl, res, sim_time, max_iters, stream);
  if (rc) return rc;
  int done = 0;
  int64_t it = 0;
  while (true) {
    rc = fl_sim_status(sim, stream, &it, run_time, &done, result);
    if (rc) return rc;
    if (done) break;
    const int64_t left = max_iters - sim->enqueued;
    const int64_t chunk = left < 64 ? left : 64;
    if (chunk <= 0) break;
    rc = fl_sim_steps(sim, chunk, stream);
    if (rc) return rc;
  }
  if (iters) *iters = it;
  return kOk;
}

// ---- fl_simulate_noalloc: the time loop without any allocation ------------
//
// For callers that cannot call cudaMalloc -- code running where the CUDA
// allocator is off limits (inside another framework's memory pool, a
// real-time thread, a pre-allocated embedded deployment) -- the loop's only
// scratch, its control block, lives in this file-scope device array instead
// of the block fl_sim_create allocates.  Size: one StepControl (96 bytes),
// whatever the grid: the loop never needs more.  Every GPU that loads the
// library holds it until the process exits.  All calls on a device share
// it and it keeps the last call's contents; fl_sim_begin's initialisation
// kernel clears everything that must start at zero.  Calls that overlap on
// the same GPU (two streams, two threads) race on it.
static __device__ __align__(256) fl::StepControl g_noalloc_control[1];

}  // extern "C"

extern "C" {

int fl_simulate_noalloc(const fl_grid* grid, double gamma, uint32_t policy,
                        uint32_t boundary_mask, void* a, void* b, double cfl, double res,
                        double sim_time, int64_t max_iters, void* stream, int64_t* iters,
                        double* run_time, void** result) {
  static_assert(sizeof(g_noalloc_control) >= sizeof(fl::StepControl),
                "the static scratch must hold one control block");
  int rc = check_grid(grid);
  if (rc) return rc;
  if ((rc = check_policy(policy))) return rc;
  if (!(gamma > 1.0)) return fail(kEInval, "gamma must exceed 1");
  if (boundary_mask >> grid->dims) return fail(kEInval, "boundary_mask has bits beyond dims");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "fl_simulate_noalloc");
  // The device address of the array, resolved on every call with the
  // caller's device current: the host-side name of the array is a stand-in,
  // not a device address, and a cached address would go stale when the
  // context is rebuilt (cudaDeviceReset reloads the module).  Resolving it is
  // a lookup, not an allocation; the first call on a device may load the
  // library's module there, so it should come before any stream capture.
  void* ctrl_addr = nullptr;
  e = cudaGetSymbolAddress(&ctrl_addr, g_noalloc_control);
  if (e != cudaSuccess) return cuda_fail(e, "fl_simulate_noalloc: cudaGetSymbolAddress");
  fl_sim sim;
  memset(&sim, 0, sizeof(sim));
  sim.grid = *grid;
  sim.pol = decode(policy);
  sim.policy = policy;
  sim.gamma = gamma;
  sim.boundary = boundary_mask;
  sim.device = dev;
  sim.ctrl = static_cast<fl::StepControl*>(ctrl_addr);
  return fl_simulate(&sim, a, b, cfl, res, sim_time, max_iters, stream, iters, run_time, result);
}

}  // extern "C"
