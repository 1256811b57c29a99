// fl_adjoint_api.cu -- C ABI of the discrete adjoint (include/fluidity_b200.h,
// fl_adjoint_sweep and fl_adj_*).  No reference counterpart: the reference
// has no differentiation.
//
// fl_adj runs the split-solver time loop forward, records the dt/dh of
// every step (the CFL step is then frozen: the adjoint treats it as a
// constant) and stores a checkpoint of the state every K steps
// (K = ceil(sqrt(nsteps)) unless the caller picks one).  Backward, each
// segment of K steps is recomputed from its checkpoint, the input of every
// sweep kept, and the adjoint sweeps run in reverse order.  Memory:
// (nsteps / K + 1) checkpoints + dims * K segment states + 4 work states;
// extra forward work: one recomputed forward pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/fluidity_b200.h"
#include "fl_adjoint_sweep.cuh"
#include "fl_internal.cuh"
#include "fl_launch.cuh"

namespace fl {
namespace {

template <typename T, int D, int S, int FLUX>
cudaError_t launch_adj_one(const AdjointParams& p, cudaStream_t st) {
  using G = AdjGeom<T, D, S>;
  auto k = adjoint_sweep_kernel<T, D, S, FLUX>;
  static bool configured[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 64 && !configured[dev]) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes);
    if (e != cudaSuccess) return e;
    configured[dev] = true;
  }
  const dim3 grid((unsigned)((p.n[0] + G::T0 - 1) / G::T0),
                  (unsigned)((p.n[1] + G::T1 - 1) / G::T1), 1);
  k<<<grid, G::THREADS, G::smem_bytes, st>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (p.chi_gz != nullptr && p.flatten && !p.basic) {
    // the chi terms, gathered per cell from the records the sweep left
    const int64_t cells = p.n[0] * (D >= 2 ? p.n[1] : 1);
    const int64_t blocks = (cells + 255) / 256;
    adj_chi_gather_kernel<T, D, S><<<(unsigned)(blocks < 148 * 8 ? blocks : 148 * 8), 256, 0,
                                     st>>>(static_cast<const T*>(p.u),
                                           static_cast<const T*>(p.chi_gz), p.chi_epoch_of,
                                           p.chi_sel, p.chi_flag, p.chi_epoch,
                                           static_cast<T*>(p.lam_in), p.pitch, p.n[0], p.n[1],
                                           (T)p.gamma - T(1));
    e = cudaGetLastError();
  }
  return e;
}

template <typename T, int FLUX>
cudaError_t launch_adj_t(const AdjointParams& p, int dims, int dim, cudaStream_t st) {
  switch (dims * 4 + dim) {
    case 4: return launch_adj_one<T, 1, 0, FLUX>(p, st);
    case 8: return launch_adj_one<T, 2, 0, FLUX>(p, st);
    case 9: return launch_adj_one<T, 2, 1, FLUX>(p, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_adj(const AdjointParams& p, bool f32, int flux, int dims, int dim,
                       cudaStream_t st) {
  if (f32)
    return flux == kForce ? launch_adj_t<float, kForce>(p, dims, dim, st)
                          : launch_adj_t<float, kHllc>(p, dims, dim, st);
  return flux == kForce ? launch_adj_t<double, kForce>(p, dims, dim, st)
                        : launch_adj_t<double, kHllc>(p, dims, dim, st);
}

int check_adj_args(const fl_grid* g, uint32_t policy, uint32_t boundary_mask, double gamma) {
  if (g == nullptr) return set_error(kEInval, "grid is NULL");
  if (g->dims < 1 || g->dims > 2) return set_error(kEInval, "the adjoint supports 1-D and 2-D grids");
  int64_t cells = 1;
  for (int d = 0; d < 3; ++d) {
    if (d < g->dims && g->n[d] < 4) return set_error(kEInval, "n[%d] must be >= 4", d);
    if (d >= g->dims && g->n[d] != 1) return set_error(kEInval, "n[%d] must be 1 beyond dims", d);
    cells *= g->n[d];
  }
  if (g->pitch < cells) return set_error(kEInval, "pitch smaller than the cell count");
  if (policy & ~0x3fu) return set_error(kEInval, "unknown policy bits (0x%x)", (unsigned)policy);
  const int flux = (int)((policy >> 1) & 3u);
  if (flux != kHllc && flux != kForce) return set_error(kEInval, "the adjoint supports HLLC and FORCE");
  if ((policy >> 3) & 1u) return set_error(kEInval, "the adjoint supports the van Leer limiter");
  if (boundary_mask >> g->dims) return set_error(kEInval, "boundary_mask has bits beyond dims");
  if (!(gamma > 1.0)) return set_error(kEInval, "gamma must exceed 1");
  return kOk;
}

int check_adj_material(const fl_material* m) {
  if (m == nullptr) return set_error(kEInval, "material is NULL");
  if (!(m->gamma > 1.0)) return set_error(kEInval, "gamma must exceed 1");
  if (!(m->p_inf >= 0.0) || m->p_inf > DBL_MAX)
    return set_error(kEInval, "p_inf must be finite and >= 0");
  return kOk;
}

// chi records for the widest sweep of the grid: (n_S + 2) * lines.
int64_t chi_record_count(const fl_grid* g) {
  if (g->dims == 1) return g->n[0] + 2;
  return std::max((g->n[0] + 2) * g->n[1], (g->n[1] + 2) * g->n[0]);
}

// Layout of count records: values (elem bytes each), epochs (4), selection
// bytes (1), then the two flag words, each part 16-byte aligned.
size_t chi_record_bytes(int64_t count, int elem) {
  auto al = [](size_t b) { return (b + 15) / 16 * 16; };
  return al((size_t)count * elem) + al((size_t)count * 4) + al((size_t)count) + 16;
}

void set_chi_records(AdjointParams& p, char* base, int64_t count, int elem, unsigned int epoch) {
  auto al = [](size_t b) { return (b + 15) / 16 * 16; };
  const size_t o1 = al((size_t)count * elem);
  const size_t o2 = o1 + al((size_t)count * 4);
  const size_t o3 = o2 + al((size_t)count);
  p.chi_gz = base;
  p.chi_epoch_of = reinterpret_cast<unsigned int*>(base + o1);
  p.chi_sel = reinterpret_cast<unsigned char*>(base + o2);
  p.chi_flag = reinterpret_cast<unsigned int*>(base + o3);
  p.chi_epoch = epoch;
}

AdjointParams make_adj_params(const fl_grid* g, uint32_t policy, double gamma, double pinf,
                              double dtdh, uint32_t boundary) {
  AdjointParams p;
  memset(&p, 0, sizeof(p));
  p.pitch = g->pitch;
  for (int d = 0; d < 3; ++d) p.n[d] = g->n[d];
  p.gamma = gamma;
  p.pinf = pinf;
  p.dtdh = dtdh;
  p.basic = (int)((policy >> 4) & 1u);
  p.flatten = ((policy >> 5) & 1u) ? 0 : 1;
  p.reflect = boundary;
  return p;
}

SweepParams make_fwd_params(const fl_grid* g, uint32_t policy, double gamma, double pinf,
                            double dtdh, uint32_t boundary) {
  SweepParams p;
  memset(&p, 0, sizeof(p));
  p.pitch = g->pitch;
  for (int d = 0; d < 3; ++d) p.n[d] = g->n[d];
  p.gamma = gamma;
  p.pinf = pinf;
  p.dtdh = dtdh;
  p.limiter = (int)((policy >> 3) & 1u);
  p.basic = (int)((policy >> 4) & 1u);
  p.flatten = ((policy >> 5) & 1u) ? 0 : 1;
  p.reflect = boundary;
  return p;
}

cudaError_t fwd_sweep(const fl_grid* g, uint32_t policy, const SweepParams& p, int dim,
                      cudaStream_t st) {
  const int flux = (int)((policy >> 1) & 3u);
  return (policy & 1u) ? launch_sweep_f32(p, g->dims, dim, flux, st)
                       : launch_sweep_f64(p, g->dims, dim, flux, st);
}

__global__ void record_dtdh_kernel(const StepControl* c, double* out) {
  if (threadIdx.x == 0) *out = c->done ? 0.0 : c->dtdh;
}

__global__ void adj_init_control_kernel(StepControl* c, double cfl, double res, long long max_iters,
                                        int is_f32) {
  if (threadIdx.x == 0) {
    memset(c, 0, sizeof(StepControl));
    c->sim_time = 1e300;
    c->cfl = is_f32 ? (double)(float)cfl : cfl;
    c->res = res;
    c->max_iters = max_iters;
    c->is_f32 = is_f32;
  }
}

template <typename T, int D, bool STIFF>
__global__ void adj_wavespeed_kernel(const T* in, int64_t pitch, int64_t cells, T gamma, T pinf,
                                     StepControl* ctrl) {
  __shared__ double s_red[8];
  const T gm1 = gamma - T(1);
  double local = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells;
       i += (int64_t)gridDim.x * blockDim.x) {
    Cons<T, D> u;
#pragma unroll
    for (int c = 0; c < D + 2; ++c) u.v[c] = in[c * pitch + i];
    ws_max(local, (double)max_wavespeed_q<STIFF>(derive(u, gm1), gamma, pinf));
  }
  cta_wavespeed_commit<256>(local, &ctrl->ws_bits, ctrl, 1, false, s_red);
}

}  // namespace
}  // namespace fl

using namespace fl;

struct fl_adj {
  fl_grid grid;
  uint32_t policy;
  uint32_t boundary;
  double gamma;
  double pinf = 0.0;        // stiffened fluid's p_inf; 0 for the ideal gas
  int64_t nsteps;
  int64_t interval;
  size_t state_bytes;
  char* ckpt = nullptr;     // (nsteps / interval + 1) states
  char* seg = nullptr;      // dims * interval states
  char* work = nullptr;     // 4 states: forward ping-pong, adjoint ping-pong
  char* chi_rec = nullptr;  // chi records of the widest sweep (chi_record_bytes)
  int64_t chi_count = 0;
  unsigned int chi_epoch = 0;  // adjoint sweeps run: names the records of each
  StepControl* ctrl = nullptr;
  double* d_dtdh = nullptr;
  std::vector<double> dtdh;
  bool have_forward = false;
  int64_t walk_launches = 0;  // forward sweeps launched: the strip counters' parity
  // a counted sweep failed to launch: it neither took its strips nor cleared
  // the other counter, so both are re-zeroed before the next pass
  bool counters_dirty = false;
};

namespace {

void* state_at(char* base, size_t bytes, int64_t i) { return base + (size_t)i * bytes; }

// Re-zeroes both strip counters on the stream after a failed counted sweep.
cudaError_t settle_adj_counters(fl_adj* a, cudaStream_t st) {
  if (!a->counters_dirty) return cudaSuccess;
  const cudaError_t e = cudaMemsetAsync(a->ctrl->walk_next, 0, sizeof(a->ctrl->walk_next), st);
  if (e == cudaSuccess) a->counters_dirty = false;
  return e;
}

}  // namespace

extern "C" {

int fl_adjoint_sweep_mat(const fl_grid* grid, int dim, const void* u_in,
                         const void* lambda_out, void* lambda_in, const fl_material* mat,
                         double dtdh, uint32_t policy, uint32_t boundary_mask, void* stream) {
  int rc = check_adj_material(mat);
  if (rc) return rc;
  const double gamma = mat->gamma;
  rc = check_adj_args(grid, policy, boundary_mask, gamma);
  if (rc) return rc;
  if (dim < 0 || dim >= grid->dims) return set_error(kEInval, "dim %d out of range", dim);
  if (!u_in || !lambda_out || !lambda_in) return set_error(kEInval, "NULL buffer");
  if (lambda_in == lambda_out) return set_error(kEInval, "lambda_in and lambda_out must differ");
  AdjointParams p = make_adj_params(grid, policy, gamma, mat->p_inf, dtdh, boundary_mask);
  p.u = u_in;
  p.lam_out = lambda_out;
  p.lam_in = lambda_in;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaSuccess;
  void* rec = nullptr;
  if (p.flatten && !p.basic) {
    // the chi terms need records for this call, epochs and flags at 0
    const int64_t count = chi_record_count(grid);
    const int elem = (policy & 1u) ? 4 : 8;
    const size_t bytes = chi_record_bytes(count, elem);
    e = cudaMallocAsync(&rec, bytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(rec, 0, bytes, st);
    set_chi_records(p, static_cast<char*>(rec), count, elem, 1u);
  }
  if (e == cudaSuccess)
    e = launch_adj(p, policy & 1u, (int)((policy >> 1) & 3u), grid->dims, dim, st);
  if (rec != nullptr) {
    const cudaError_t ef = cudaFreeAsync(rec, st);
    if (e == cudaSuccess) e = ef;
  }
  if (e != cudaSuccess) return set_error(kECuda, "fl_adjoint_sweep: %s", cudaGetErrorString(e));
  return kOk;
}

int fl_adjoint_sweep(const fl_grid* grid, int dim, const void* u_in, const void* lambda_out,
                     void* lambda_in, double gamma, double dtdh, uint32_t policy,
                     uint32_t boundary_mask, void* stream) {
  const fl_material mat{gamma, 0.0};
  return fl_adjoint_sweep_mat(grid, dim, u_in, lambda_out, lambda_in, &mat, dtdh, policy,
                              boundary_mask, stream);
}

int fl_adj_create(fl_adj** out, const fl_grid* grid, double gamma, uint32_t policy,
                  uint32_t boundary_mask, int64_t nsteps, int64_t interval) {
  if (out == nullptr) return set_error(kEInval, "handle pointer is NULL");
  *out = nullptr;
  int rc = check_adj_args(grid, policy, boundary_mask, gamma);
  if (rc) return rc;
  if (nsteps <= 0) return set_error(kEInval, "nsteps must be positive");
  if (interval <= 0) interval = (int64_t)std::ceil(std::sqrt((double)nsteps));
  fl_adj* a = new (std::nothrow) fl_adj;
  if (a == nullptr) return set_error(kENoMem, "out of host memory");
  a->grid = *grid;
  a->policy = policy;
  a->boundary = boundary_mask;
  a->gamma = gamma;
  a->nsteps = nsteps;
  a->interval = interval;
  a->state_bytes = (size_t)(grid->dims + 2) * grid->pitch * ((policy & 1u) ? 4 : 8);
  const int64_t nck = nsteps / interval + 1;
  cudaError_t e = cudaMalloc(&a->ckpt, a->state_bytes * nck);
  if (e == cudaSuccess) e = cudaMalloc(&a->seg, a->state_bytes * grid->dims * interval);
  if (e == cudaSuccess) e = cudaMalloc(&a->work, a->state_bytes * 4);
  a->chi_count = chi_record_count(grid);
  const size_t rec_bytes = chi_record_bytes(a->chi_count, (policy & 1u) ? 4 : 8);
  if (e == cudaSuccess) e = cudaMalloc(&a->chi_rec, rec_bytes);
  if (e == cudaSuccess) e = cudaMemset(a->chi_rec, 0, rec_bytes);   // epochs and flags 0
  if (e == cudaSuccess) e = cudaMalloc(&a->ctrl, sizeof(StepControl));
  if (e == cudaSuccess) e = cudaMemset(a->ctrl, 0, sizeof(StepControl));  // strip counters at 0
  if (e == cudaSuccess) e = cudaMalloc(&a->d_dtdh, sizeof(double) * nsteps);
  if (e != cudaSuccess) {
    fl_adj_destroy(a);
    return set_error(kENoMem, "fl_adj_create: %s", cudaGetErrorString(e));
  }
  a->dtdh.assign(nsteps, 0.0);
  *out = a;
  return kOk;
}

int fl_adj_set_material(fl_adj* a, const fl_material* mat) {
  if (a == nullptr) return set_error(kEInval, "adjoint handle is NULL");
  int rc = check_adj_material(mat);
  if (rc) return rc;
  a->gamma = mat->gamma;
  a->pinf = mat->p_inf;
  a->have_forward = false;  // a recorded forward pass belongs to the old material
  return kOk;
}

int fl_adj_destroy(fl_adj* a) {
  if (a == nullptr) return kOk;
  cudaFree(a->ckpt);
  cudaFree(a->seg);
  cudaFree(a->work);
  cudaFree(a->chi_rec);
  cudaFree(a->ctrl);
  cudaFree(a->d_dtdh);
  delete a;
  return kOk;
}

int fl_adj_forward(fl_adj* a, const void* u0, void* u_final, double cfl, double res,
                   const double* frozen_dtdh, void* stream) {
  if (a == nullptr || u0 == nullptr || u_final == nullptr) return set_error(kEInval, "NULL argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const fl_grid* g = &a->grid;
  const int D = g->dims;
  const size_t sb = a->state_bytes;
  void* cur = state_at(a->work, sb, 0);
  void* nxt = state_at(a->work, sb, 1);
  cudaError_t e = settle_adj_counters(a, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cur, u0, sb, cudaMemcpyDeviceToDevice, st);
  const bool record = frozen_dtdh == nullptr;
  if (record && e == cudaSuccess) {
    if (!(cfl > 0.0) || !(res > 0.0)) return set_error(kEInval, "cfl and res must be positive");
    adj_init_control_kernel<<<1, 32, 0, st>>>(a->ctrl, cfl, res, (long long)a->nsteps,
                                              (a->policy & 1u) ? 1 : 0);
    const int64_t cells = g->n[0] * g->n[1] * g->n[2];
    const unsigned blocks = (unsigned)std::min<int64_t>((cells + 255) / 256, 148 * 8);
    const bool f32 = (a->policy & 1u) != 0;
    const bool stiff = a->pinf != 0.0;
    if (D == 1) {
      if (f32 && stiff)
        adj_wavespeed_kernel<float, 1, true><<<blocks, 256, 0, st>>>(
            (const float*)cur, g->pitch, cells, (float)a->gamma, (float)a->pinf, a->ctrl);
      else if (f32)
        adj_wavespeed_kernel<float, 1, false><<<blocks, 256, 0, st>>>(
            (const float*)cur, g->pitch, cells, (float)a->gamma, 0.0f, a->ctrl);
      else if (stiff)
        adj_wavespeed_kernel<double, 1, true><<<blocks, 256, 0, st>>>(
            (const double*)cur, g->pitch, cells, a->gamma, a->pinf, a->ctrl);
      else
        adj_wavespeed_kernel<double, 1, false><<<blocks, 256, 0, st>>>(
            (const double*)cur, g->pitch, cells, a->gamma, 0.0, a->ctrl);
    } else {
      if (f32 && stiff)
        adj_wavespeed_kernel<float, 2, true><<<blocks, 256, 0, st>>>(
            (const float*)cur, g->pitch, cells, (float)a->gamma, (float)a->pinf, a->ctrl);
      else if (f32)
        adj_wavespeed_kernel<float, 2, false><<<blocks, 256, 0, st>>>(
            (const float*)cur, g->pitch, cells, (float)a->gamma, 0.0f, a->ctrl);
      else if (stiff)
        adj_wavespeed_kernel<double, 2, true><<<blocks, 256, 0, st>>>(
            (const double*)cur, g->pitch, cells, a->gamma, a->pinf, a->ctrl);
      else
        adj_wavespeed_kernel<double, 2, false><<<blocks, 256, 0, st>>>(
            (const double*)cur, g->pitch, cells, a->gamma, 0.0, a->ctrl);
    }
    e = cudaGetLastError();
  }
  for (int64_t k = 0; k < a->nsteps && e == cudaSuccess; ++k) {
    if (k % a->interval == 0)
      e = cudaMemcpyAsync(state_at(a->ckpt, sb, k / a->interval), cur, sb,
                          cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) break;
    if (record) {
      record_dtdh_kernel<<<1, 32, 0, st>>>(a->ctrl, a->d_dtdh + k);
      e = cudaGetLastError();
    }
    SweepParams p = make_fwd_params(g, a->policy, a->gamma, a->pinf,
                                    record ? 0.0 : frozen_dtdh[k], a->boundary);
    if (record) p.ctrl = a->ctrl;
    for (int d = 0; d < D && e == cudaSuccess; ++d) {
      p.in = cur;
      p.out = nxt;
      p.walk_next = a->ctrl->walk_next;
      p.walk_slot = (int)(a->walk_launches++ & 1);
      const bool last = (d == D - 1);
      p.ws_accum = (record && last) ? &a->ctrl->ws_bits : nullptr;
      p.finalize = (record && last) ? 1 : 0;
      e = fwd_sweep(g, a->policy, p, d, st);
      if (e != cudaSuccess) a->counters_dirty = true;
      void* t = cur;
      cur = nxt;
      nxt = t;
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(u_final, cur, sb, cudaMemcpyDeviceToDevice, st);
  if (record && e == cudaSuccess) {
    e = cudaMemcpyAsync(a->dtdh.data(), a->d_dtdh, sizeof(double) * a->nsteps,
                        cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  } else if (e == cudaSuccess) {
    a->dtdh.assign(frozen_dtdh, frozen_dtdh + a->nsteps);
  }
  if (e != cudaSuccess) return set_error(kECuda, "fl_adj_forward: %s", cudaGetErrorString(e));
  if (record) {
    for (int64_t k = 0; k < a->nsteps; ++k)
      if (!(a->dtdh[k] > 0.0)) return set_error(kENan, "step %lld: no finite CFL step", (long long)k);
  }
  a->have_forward = true;
  return kOk;
}

int fl_adj_dtdh(const fl_adj* a, double* out) {
  if (a == nullptr || out == nullptr) return set_error(kEInval, "NULL argument");
  if (!a->have_forward) return set_error(kEInval, "fl_adj_forward not called");
  memcpy(out, a->dtdh.data(), sizeof(double) * a->nsteps);
  return kOk;
}

int fl_adj_backward(fl_adj* a, const void* lambda_final, void* lambda_0, void* stream) {
  if (a == nullptr || lambda_final == nullptr || lambda_0 == nullptr)
    return set_error(kEInval, "NULL argument");
  if (!a->have_forward) return set_error(kEInval, "fl_adj_forward not called");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const fl_grid* g = &a->grid;
  const int D = g->dims;
  const size_t sb = a->state_bytes;
  const bool f32 = a->policy & 1u;
  const int flux = (int)((a->policy >> 1) & 3u);
  void* la = state_at(a->work, sb, 2);
  void* lb = state_at(a->work, sb, 3);
  cudaError_t e = settle_adj_counters(a, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(la, lambda_final, sb, cudaMemcpyDeviceToDevice, st);
  const int64_t nseg = (a->nsteps + a->interval - 1) / a->interval;
  for (int64_t j = nseg - 1; j >= 0 && e == cudaSuccess; --j) {
    const int64_t k0 = j * a->interval;
    const int64_t k1 = std::min(k0 + a->interval, a->nsteps);
    // recompute the segment, keeping the input of every sweep
    void* cur = state_at(a->seg, sb, 0);
    e = cudaMemcpyAsync(cur, state_at(a->ckpt, sb, j), sb, cudaMemcpyDeviceToDevice, st);
    for (int64_t k = k0; k < k1 && e == cudaSuccess; ++k) {
      SweepParams p = make_fwd_params(g, a->policy, a->gamma, a->pinf, a->dtdh[k], a->boundary);
      for (int d = 0; d < D && e == cudaSuccess; ++d) {
        const int64_t slot = (k - k0) * D + d;
        const bool last = (k == k1 - 1) && (d == D - 1);
        if (last) break;  // the final output of the segment is not needed
        p.in = state_at(a->seg, sb, slot);
        p.out = state_at(a->seg, sb, slot + 1);
        p.walk_next = a->ctrl->walk_next;
        p.walk_slot = (int)(a->walk_launches++ & 1);
        e = fwd_sweep(g, a->policy, p, d, st);
        if (e != cudaSuccess) a->counters_dirty = true;
      }
    }
    // adjoint sweeps in reverse order
    for (int64_t k = k1 - 1; k >= k0 && e == cudaSuccess; --k) {
      for (int d = D - 1; d >= 0 && e == cudaSuccess; --d) {
        AdjointParams p =
            make_adj_params(g, a->policy, a->gamma, a->pinf, a->dtdh[k], a->boundary);
        p.u = state_at(a->seg, sb, (k - k0) * D + d);
        p.lam_out = la;
        p.lam_in = lb;
        if (++a->chi_epoch == 0u) a->chi_epoch = 1u;   // 0 marks records never written
        set_chi_records(p, a->chi_rec, a->chi_count, f32 ? 4 : 8, a->chi_epoch);
        e = launch_adj(p, f32, flux, D, d, st);
        void* t = la;
        la = lb;
        lb = t;
      }
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(lambda_0, la, sb, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return set_error(kECuda, "fl_adj_backward: %s", cudaGetErrorString(e));
  return kOk;
}

}  // extern "C"
