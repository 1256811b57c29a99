// fl_batch_api.cu -- C ABI of the batched solver (include/fluidity_b200.h,
// fl_batch_*): descriptors, work lists, launches, CUDA-graph capture and the
// tile autotuner.  No reference counterpart (see fl_batch.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/fluidity_b200.h"
#include "fl_batch.cuh"

namespace fl {
namespace {

template <typename... A>
int bfail(int code, const char* fmt, A... args) {
  return set_error(code, fmt, args...);
}

// 1-D size classes: CTA width per class (autotuned), upper n per class.
constexpr int kClasses = 3;
constexpr int kClassThreads[3] = {128, 256, 512};

}  // namespace
}  // namespace fl

using namespace fl;

struct fl_batch {
  int count = 0;
  bool f32 = false;
  int flux = 0;
  int limiter = 0;
  int basic = 0;
  int flatten = 1;
  uint32_t reflect = 0;
  double gamma = 1.4;
  double pinf = 0.0;            // stiffened fluid's p_inf; 0 for the ideal gas
  std::vector<fl_batch_desc> desc;
  // device data
  BatchProblem* d_problems = nullptr;
  StepControl* d_ctrl = nullptr;
  BatchItem* d_items = nullptr;
  int* d_order = nullptr;       // 1-D problems grouped by class, largest first
  int* d_queue = nullptr;       // one queue head per class
  double* d_res = nullptr;
  int n_items = 0;
  // per 1-D class: [first, first + count) in d_order, max n
  int cls_first[kClasses] = {0, 0, 0};
  int cls_count[kClasses] = {0, 0, 0};
  int cls_nmax[kClasses] = {0, 0, 0};
  int cls_threads[kClasses] = {128, 256, 512};
  // autotuned: 1-D class boundaries (n <= bound -> class) and 2-D strip rows
  int bound1d[2] = {512, 2048};
  int ry_small = 32, ry_mid = 64, ry_large = 64;   // side <= 128, <= 256, larger
  void* arena_a = nullptr;
  void* arena_b = nullptr;
  cudaStream_t side = nullptr;
  cudaStream_t cap = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t graph = nullptr;
  int64_t graph_steps = 0;
};

namespace {

int cuda_berr(cudaError_t e, const char* where) {
  return set_error(kECuda, "%s: %s", where, cudaGetErrorString(e));
}

int pick_ry(const fl_batch* b, int64_t side) {
  return side <= 128 ? b->ry_small : (side <= 256 ? b->ry_mid : b->ry_large);
}

int pick_class(const fl_batch* b, int64_t n) {
  return n <= b->bound1d[0] ? 0 : (n <= b->bound1d[1] ? 1 : 2);
}

// (Re)builds descriptors, the 1-D queue order and the 2-D work items from the
// current tuning and uploads them.
int upload_plan(fl_batch* b) {
  const int n = b->count;
  std::vector<BatchProblem> pr(n);
  std::vector<BatchItem> items;
  std::vector<int> cls_lists[kClasses];
  for (int i = 0; i < n; ++i) {
    const fl_batch_desc& d = b->desc[i];
    BatchProblem& p = pr[i];
    memset(&p, 0, sizeof(p));
    p.n0 = d.n[0];
    p.n1 = d.dims == 2 ? d.n[1] : 1;
    p.offset = d.offset;
    p.pitch = d.pitch;
    p.dims = d.dims;
    if (d.dims == 1) {
      cls_lists[pick_class(b, d.n[0])].push_back(i);
    } else {
      const int ry = pick_ry(b, std::max(d.n[0], d.n[1]));
      p.ry = ry;
      using W = WalkCfg<float, 0>;   // the x sweep owns fewer columns: size by it
      const int64_t bx = (d.n[0] + W::OWN - 1) / W::OWN;
      const int64_t by = (d.n[1] + (int64_t)ry * W::WARPS - 1) / ((int64_t)ry * W::WARPS);
      p.items = (int)(bx * by);
      for (int64_t y = 0; y < by; ++y)
        for (int64_t x = 0; x < bx; ++x) items.push_back(BatchItem{i, (int)x, (int)y, 0});
    }
  }
  std::vector<int> order;
  for (int c = 0; c < kClasses; ++c) {
    std::sort(cls_lists[c].begin(), cls_lists[c].end(),
              [&](int x, int y) { return b->desc[x].n[0] > b->desc[y].n[0]; });
    b->cls_first[c] = (int)order.size();
    b->cls_count[c] = (int)cls_lists[c].size();
    b->cls_nmax[c] = cls_lists[c].empty() ? 0 : (int)b->desc[cls_lists[c][0]].n[0];
    order.insert(order.end(), cls_lists[c].begin(), cls_lists[c].end());
  }
  // Items of the 2-D y sweep must count per problem the same as the x sweep:
  // both launches use the same item list, and the y sweep's owned columns
  // (26) exceed the x sweep's (24), so the extra columns of the y sweep's
  // last group are simply out of range.
  cudaFree(b->d_items);
  cudaFree(b->d_order);
  b->d_items = nullptr;
  b->d_order = nullptr;
  b->n_items = (int)items.size();
  cudaError_t e = cudaSuccess;
  if (!items.empty()) {
    e = cudaMalloc(&b->d_items, items.size() * sizeof(BatchItem));
    if (e == cudaSuccess)
      e = cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(BatchItem),
                     cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !order.empty()) {
    e = cudaMalloc(&b->d_order, order.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpy(b->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_problems, pr.data(), n * sizeof(BatchProblem), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch plan upload");
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return kOk;
}

BatchArgs base_args(const fl_batch* b) {
  BatchArgs a;
  memset(&a, 0, sizeof(a));
  a.problems = b->d_problems;
  a.ctrl = b->d_ctrl;
  a.items = b->d_items;
  a.order = b->d_order;
  a.arena_a = b->arena_a;
  a.arena_b = b->arena_b;
  a.gamma = b->gamma;
  a.pinf = b->pinf;
  a.limiter = b->limiter;
  a.basic = b->basic;
  a.flatten = b->flatten;
  a.reflect = b->reflect;
  return a;
}

template <typename T, int FLUX, int THREADS>
cudaError_t set_attr_1d() {
  // the largest 1-D problem that fits
  const size_t smem = 2 * 3 * (size_t)(batch1d_max<T>() + 8) * sizeof(T);
  return cudaFuncSetAttribute(batch1d_kernel<T, FLUX, THREADS>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <typename T>
cudaError_t prepare(const fl_batch* b) {
  static bool done[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 64 && done[dev]) return cudaSuccess;
  constexpr int kSH = kHllc | kStiffEos, kSF = kForce | kStiffEos;
  const cudaError_t r[] = {
      set_attr_1d<T, kHllc, 64>(), set_attr_1d<T, kHllc, 128>(), set_attr_1d<T, kHllc, 256>(),
      set_attr_1d<T, kHllc, 512>(), set_attr_1d<T, kForce, 64>(), set_attr_1d<T, kForce, 128>(),
      set_attr_1d<T, kForce, 256>(), set_attr_1d<T, kForce, 512>(),
      set_attr_1d<T, kSH, 64>(), set_attr_1d<T, kSH, 128>(), set_attr_1d<T, kSH, 256>(),
      set_attr_1d<T, kSH, 512>(), set_attr_1d<T, kSF, 64>(), set_attr_1d<T, kSF, 128>(),
      set_attr_1d<T, kSF, 256>(), set_attr_1d<T, kSF, 512>()};
  for (cudaError_t x : r)
    if (x != cudaSuccess) return x;
  if (dev < 64) done[dev] = true;
  (void)b;
  return cudaSuccess;
}

template <typename T, int FLUX, int THREADS>
cudaError_t launch_1d(const fl_batch* b, int c, int64_t nsteps, cudaStream_t st) {
  BatchArgs a = base_args(b);
  a.order = b->d_order + b->cls_first[c];
  a.count = b->cls_count[c];
  a.queue = b->d_queue + c;
  const int ld = b->cls_nmax[c] + 8;
  const size_t smem = 2 * 3 * (size_t)ld * sizeof(T);
  auto k = batch1d_kernel<T, FLUX, THREADS>;
  cudaError_t e = prepare<T>(b);
  if (e != cudaSuccess) return e;
  batch_reset_queue_kernel<<<1, 1, 0, st>>>(a.queue);
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, THREADS, smem);
  int grid = sms * std::max(per_sm, 1);
  grid = std::min(grid, a.count);
  k<<<grid, THREADS, smem, st>>>(a, (long long)nsteps, ld);
  return cudaGetLastError();
}

template <typename T, int FLUX>
cudaError_t launch_1d_class(const fl_batch* b, int c, int64_t nsteps, cudaStream_t st) {
  switch (b->cls_threads[c]) {
    case 64: return launch_1d<T, FLUX, 64>(b, c, nsteps, st);
    case 128: return launch_1d<T, FLUX, 128>(b, c, nsteps, st);
    case 256: return launch_1d<T, FLUX, 256>(b, c, nsteps, st);
    default: return launch_1d<T, FLUX, 512>(b, c, nsteps, st);
  }
}

template <typename T, int FLUX>
cudaError_t launch_2d_step(const fl_batch* b, cudaStream_t st) {
  BatchArgs a = base_args(b);
  a.count = b->n_items;
  batch2d_kernel<T, 0, FLUX><<<b->n_items, WalkCfg<T, 0>::THREADS, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  batch2d_kernel<T, 1, FLUX><<<b->n_items, WalkCfg<T, 1>::THREADS, 0, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int FLUX>
cudaError_t enqueue_steps(fl_batch* b, int64_t nsteps, cudaStream_t st, bool do1d, bool do2d) {
  cudaError_t e = cudaSuccess;
  const bool has1d = do1d && (b->cls_count[0] + b->cls_count[1] + b->cls_count[2]) > 0;
  const bool has2d = do2d && b->n_items > 0;
  if (has1d && has2d) {
    // fork the resident 1-D launches onto the side stream
    if ((e = cudaEventRecord(b->ev_fork, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(b->side, b->ev_fork, 0)) != cudaSuccess) return e;
  }
  cudaStream_t s1 = (has1d && has2d) ? b->side : st;
  if (has1d)
    for (int c = 0; c < kClasses; ++c)
      if (b->cls_count[c] > 0 && (e = launch_1d_class<T, FLUX>(b, c, nsteps, s1)) != cudaSuccess)
        return e;
  if (has2d)
    for (int64_t s = 0; s < nsteps; ++s)
      if ((e = launch_2d_step<T, FLUX>(b, st)) != cudaSuccess) return e;
  if (has1d && has2d) {
    if ((e = cudaEventRecord(b->ev_join, b->side)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(st, b->ev_join, 0)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename T>
cudaError_t enqueue_t(fl_batch* b, int64_t nsteps, cudaStream_t st, bool do1d, bool do2d) {
  switch (b->flux | (b->pinf != 0.0 ? kStiffEos : 0)) {
    case kForce: return enqueue_steps<T, kForce>(b, nsteps, st, do1d, do2d);
    case kForce | kStiffEos: return enqueue_steps<T, kForce | kStiffEos>(b, nsteps, st, do1d, do2d);
    case kHllc | kStiffEos: return enqueue_steps<T, kHllc | kStiffEos>(b, nsteps, st, do1d, do2d);
    default: return enqueue_steps<T, kHllc>(b, nsteps, st, do1d, do2d);
  }
}

cudaError_t enqueue(fl_batch* b, int64_t nsteps, cudaStream_t st, bool do1d = true,
                    bool do2d = true) {
  return b->f32 ? enqueue_t<float>(b, nsteps, st, do1d, do2d)
                : enqueue_t<double>(b, nsteps, st, do1d, do2d);
}

int64_t arena_elems(const fl_batch* b) {
  int64_t m = 0;
  for (const auto& d : b->desc) m = std::max(m, d.offset + (int64_t)(d.dims + 2) * d.pitch);
  return m;
}

}  // namespace

extern "C" {

int fl_batch_create(fl_batch** out, const fl_batch_desc* problems, int32_t count, double gamma,
                    uint32_t policy, uint32_t boundary_mask) {
  if (out == nullptr) return bfail(kEInval, "batch handle pointer is NULL");
  *out = nullptr;
  if (problems == nullptr || count <= 0) return bfail(kEInval, "empty problem list");
  if (policy & ~0x3fu) return bfail(kEInval, "unknown policy bits (0x%x)", (unsigned)policy);
  const int flux = (int)((policy >> 1) & 3u);
  if (flux != kHllc && flux != kForce) return bfail(kEInval, "batched solver supports HLLC and FORCE");
  if (!(gamma > 1.0)) return bfail(kEInval, "gamma must exceed 1");
  if (boundary_mask > 3u) return bfail(kEInval, "boundary_mask has bits beyond 2-D");
  const bool f32 = (policy & 1u) != 0;
  const int nmax1d = f32 ? batch1d_max<float>() : batch1d_max<double>();
  for (int i = 0; i < count; ++i) {
    const fl_batch_desc& d = problems[i];
    if (d.dims != 1 && d.dims != 2) return bfail(kEInval, "problem %d: dims must be 1 or 2", i);
    if (d.n[0] < 4 || (d.dims == 2 && d.n[1] < 4))
      return bfail(kEInval, "problem %d: every dimension needs >= 4 cells", i);
    if (d.dims == 1 && d.n[0] > nmax1d)
      return bfail(kEInval, "problem %d: 1-D problems are limited to %d cells", i, nmax1d);
    const int64_t cells = d.n[0] * (d.dims == 2 ? d.n[1] : 1);
    if (d.pitch < cells || d.offset < 0) return bfail(kEInval, "problem %d: bad pitch/offset", i);
    if (!(d.res > 0.0)) return bfail(kEInval, "problem %d: res must be positive", i);
  }
  fl_batch* b = new (std::nothrow) fl_batch;
  if (b == nullptr) return bfail(kENoMem, "out of host memory");
  b->count = count;
  b->f32 = f32;
  b->flux = flux;
  b->limiter = (int)((policy >> 3) & 1u);
  b->basic = (int)((policy >> 4) & 1u);
  b->flatten = ((policy >> 5) & 1u) ? 0 : 1;
  b->reflect = boundary_mask;
  b->gamma = gamma;
  b->desc.assign(problems, problems + count);
  std::vector<double> res(count);
  for (int i = 0; i < count; ++i) res[i] = problems[i].res;
  cudaError_t e = cudaMalloc(&b->d_problems, count * sizeof(BatchProblem));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_ctrl, count * sizeof(StepControl));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, kClasses * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_res, count * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_res, res.data(), count * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->d_ctrl, 0, count * sizeof(StepControl));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    fl_batch_destroy(b);
    return bfail(kENoMem, "fl_batch_create: %s", cudaGetErrorString(e));
  }
  const int rc = upload_plan(b);
  if (rc) {
    fl_batch_destroy(b);
    return rc;
  }
  *out = b;
  return kOk;
}

int fl_batch_destroy(fl_batch* b) {
  if (b == nullptr) return kOk;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->d_problems);
  cudaFree(b->d_ctrl);
  cudaFree(b->d_items);
  cudaFree(b->d_order);
  cudaFree(b->d_queue);
  cudaFree(b->d_res);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  delete b;
  return kOk;
}

int fl_batch_set_material(fl_batch* b, const fl_material* mat) {
  if (b == nullptr) return bfail(kEInval, "batch handle is NULL");
  if (mat == nullptr) return bfail(kEInval, "material is NULL");
  if (!(mat->gamma > 1.0)) return bfail(kEInval, "gamma must exceed 1");
  if (!(mat->p_inf >= 0.0) || mat->p_inf > DBL_MAX)
    return bfail(kEInval, "p_inf must be finite and >= 0");
  b->gamma = mat->gamma;
  b->pinf = mat->p_inf;
  if (b->graph) {  // a captured graph holds the old material's kernels
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return kOk;
}

int fl_batch_begin(fl_batch* b, void* arena_a, void* arena_b, double cfl, double sim_time,
                   int64_t max_iters, void* stream) {
  if (b == nullptr || arena_a == nullptr) return bfail(kEInval, "NULL batch or arena");
  if (b->n_items > 0 && (arena_b == nullptr || arena_b == arena_a))
    return bfail(kEInval, "2-D problems need a second, distinct arena");
  if (!(cfl > 0.0) || max_iters < 0) return bfail(kEInval, "cfl must be positive, max_iters >= 0");
  if (b->arena_a != arena_a || b->arena_b != arena_b) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
  }
  b->arena_a = arena_a;
  b->arena_b = arena_b;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  BatchArgs a = base_args(b);
  if (b->f32)
    batch_init_kernel<float><<<b->count, 256, 0, st>>>(a, b->count, cfl, sim_time,
                                                       (long long)max_iters, b->d_res);
  else
    batch_init_kernel<double><<<b->count, 256, 0, st>>>(a, b->count, cfl, sim_time,
                                                        (long long)max_iters, b->d_res);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_begin");
  return kOk;
}

int fl_batch_steps(fl_batch* b, int64_t nsteps, void* stream) {
  if (b == nullptr || b->arena_a == nullptr) return bfail(kEInval, "fl_batch_begin not called");
  if (nsteps < 0) return bfail(kEInval, "nsteps < 0");
  cudaError_t e = enqueue(b, nsteps, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_steps");
  return kOk;
}

int fl_batch_capture(fl_batch* b, int64_t nsteps) {
  if (b == nullptr || b->arena_a == nullptr) return bfail(kEInval, "fl_batch_begin not called");
  if (nsteps < 0) return bfail(kEInval, "nsteps < 0");
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  // set shared-memory limits outside the capture
  cudaError_t e = b->f32 ? prepare<float>(b) : prepare<double>(b);
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_capture (prepare)");
  e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_capture (begin)");
  cudaError_t e2 = enqueue(b, nsteps, b->cap);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(b->cap, &g);
  if (e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cuda_berr(e2, "fl_batch_capture (enqueue)");
  }
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_capture (end)");
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_capture (instantiate)");
  b->graph_steps = nsteps;
  return kOk;
}

int fl_batch_launch(fl_batch* b, void* stream) {
  if (b == nullptr || b->graph == nullptr) return bfail(kEInval, "no captured graph");
  cudaError_t e = cudaGraphLaunch(b->graph, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_launch");
  return kOk;
}

int fl_batch_status(fl_batch* b, void* stream, int64_t* iters, double* run_time,
                    int32_t* done_count) {
  if (b == nullptr) return bfail(kEInval, "NULL batch");
  std::vector<StepControl> h(b->count);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(h.data(), b->d_ctrl, b->count * sizeof(StepControl),
                                  cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_status");
  int32_t done = 0;
  int nan = -1;
  for (int i = 0; i < b->count; ++i) {
    if (iters) iters[i] = h[i].iters;
    if (run_time) run_time[i] = h[i].run_time;
    done += h[i].done ? 1 : 0;
    if (h[i].status == kENan && nan < 0) nan = i;
  }
  if (done_count) *done_count = done;
  if (nan >= 0) return bfail(kENan, "problem %d: non-finite wavespeed", nan);
  return kOk;
}

int fl_batch_autotune(fl_batch* b, void* arena_a, void* arena_b, int64_t trial_steps,
                      void* stream) {
  if (b == nullptr || arena_a == nullptr) return bfail(kEInval, "NULL batch or arena");
  if (trial_steps <= 0) trial_steps = 8;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // trials run on scratch copies so that the caller's states are untouched
  const size_t bytes = (size_t)arena_elems(b) * (b->f32 ? 4 : 8);
  void* ta = nullptr;
  void* tb = nullptr;
  cudaError_t e = cudaMalloc(&ta, bytes);
  if (e == cudaSuccess && b->n_items > 0) e = cudaMalloc(&tb, bytes);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaFree(ta);
    cudaFree(tb);
    return bfail(kENoMem, "fl_batch_autotune: %s", cudaGetErrorString(e));
  }
  auto trial = [&](bool do1d, bool do2d) -> float {
    cudaMemcpyAsync(ta, arena_a, bytes, cudaMemcpyDeviceToDevice, st);
    void* sa = b->arena_a;
    void* sb = b->arena_b;
    fl_batch_begin(b, ta, tb ? tb : nullptr, 0.8, 1e30, trial_steps, stream);
    enqueue(b, 1, st, do1d, do2d);  // warm-up
    fl_batch_begin(b, ta, tb ? tb : nullptr, 0.8, 1e30, trial_steps, stream);
    cudaEventRecord(e0, st);
    enqueue(b, trial_steps, st, do1d, do2d);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    b->arena_a = sa;
    b->arena_b = sb;
    return ms;
  };
  // 1-D: CTA width per size class
  const int cand[4] = {64, 128, 256, 512};
  for (int c = 0; c < kClasses; ++c) {
    if (b->cls_count[c] == 0) continue;
    const int keep[kClasses] = {b->cls_count[0], b->cls_count[1], b->cls_count[2]};
    float best = 1e30f;
    int best_t = b->cls_threads[c];
    for (int t : cand) {
      for (int o = 0; o < kClasses; ++o) b->cls_count[o] = (o == c) ? keep[o] : 0;
      b->cls_threads[c] = t;
      const float ms = trial(true, false);
      if (ms < best) {
        best = ms;
        best_t = t;
      }
    }
    for (int o = 0; o < kClasses; ++o) b->cls_count[o] = keep[o];
    b->cls_threads[c] = best_t;
  }
  // 2-D: strip rows per size class (small / mid / large sides)
  if (b->n_items > 0) {
    int* slots[3] = {&b->ry_small, &b->ry_mid, &b->ry_large};
    for (int c = 0; c < 3; ++c) {
      float best = 1e30f;
      int best_ry = *slots[c];
      for (int ry : {16, 32, 64, 128}) {
        *slots[c] = ry;
        upload_plan(b);
        const float ms = trial(false, true);
        if (ms < best) {
          best = ms;
          best_ry = ry;
        }
      }
      *slots[c] = best_ry;
    }
    upload_plan(b);
  }
  cudaStreamSynchronize(st);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(ta);
  cudaFree(tb);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_berr(e, "fl_batch_autotune");
  return kOk;
}

int fl_batch_tuning(const fl_batch* b, int32_t* out, int32_t n) {
  // [threads of 1-D classes 0..2, 1-D class bounds 0..1, ry small/mid/large]
  if (b == nullptr || out == nullptr || n < 8) return bfail(kEInval, "need 8 slots");
  for (int c = 0; c < kClasses; ++c) out[c] = b->cls_threads[c];
  out[3] = b->bound1d[0];
  out[4] = b->bound1d[1];
  out[5] = b->ry_small;
  out[6] = b->ry_mid;
  out[7] = b->ry_large;
  return kOk;
}

}  // extern "C"
