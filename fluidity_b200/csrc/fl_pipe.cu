// fl_pipe.cu -- runs of the split solver whose initial states and results
// live in host memory, streamed through the GPU (fl_host_pipe_*).
//
// The reference's host flow is fill_data (host -> device), simulate, and
// write_results (device -> host), one simulation after another
// (simulator/simulator_impl.hpp:223-358).  Here a sequence of such jobs
// overlaps each job's copies with its neighbours' compute:
//   - the upload of job k + 1 runs while job k computes;
//   - the download of job k runs while job k + 1 computes.
// Uploads, compute and downloads use three streams.  `sets` pairs of device
// state buffers rotate; with 3 sets, a job's upload, its compute and the
// previous job's download never share a buffer.  Every copy is one
// cudaMemcpyAsync of a whole state.  The host buffers should be page-locked
// (cudaMallocHost / cudaHostRegister), otherwise the copies do not overlap.
#include <cuda_runtime.h>

#include <cstring>
#include <new>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"

using namespace fl;

struct fl_host_pipe {
  fl_grid grid;
  uint32_t policy;
  int sets;
  int64_t bytes;
  fl_sim* sim;
  void* a[4];
  void* b[4];
  cudaStream_t s_in, s_run, s_out;
  cudaEvent_t ev_in[4], ev_run[4], ev_free[4];
};

namespace {

constexpr int kMaxSets = 4;

int pipe_cuda(cudaError_t e, const char* where) {
  return set_error(kECuda, "%s: %s", where, cudaGetErrorString(e));
}

void release(fl_host_pipe* p) {
  if (p == nullptr) return;
  for (int i = 0; i < kMaxSets; ++i) {
    if (p->a[i]) cudaFree(p->a[i]);
    if (p->b[i]) cudaFree(p->b[i]);
    if (p->ev_in[i]) cudaEventDestroy(p->ev_in[i]);
    if (p->ev_run[i]) cudaEventDestroy(p->ev_run[i]);
    if (p->ev_free[i]) cudaEventDestroy(p->ev_free[i]);
  }
  if (p->s_in) cudaStreamDestroy(p->s_in);
  if (p->s_run) cudaStreamDestroy(p->s_run);
  if (p->s_out) cudaStreamDestroy(p->s_out);
  if (p->sim) fl_sim_destroy(p->sim);
  delete p;
}

}  // namespace

extern "C" {

int fl_host_pipe_create(fl_host_pipe** pipe, const fl_grid* grid, double gamma, uint32_t policy,
                        uint32_t boundary_mask, int sets) {
  if (pipe == nullptr) return set_error(kEInval, "pipe is NULL");
  *pipe = nullptr;
  if (sets < 2 || sets > kMaxSets) return set_error(kEInval, "sets must be 2..%d", kMaxSets);
  const int64_t bytes = fl_state_bytes(grid, policy);
  if (bytes < 0) return kEInval;   // fl_state_bytes recorded the reason
  fl_host_pipe* p = new (std::nothrow) fl_host_pipe;
  if (p == nullptr) return set_error(kENoMem, "out of host memory");
  memset(p, 0, sizeof(*p));
  p->grid = *grid;
  p->policy = policy;
  p->sets = sets;
  p->bytes = bytes;
  int rc = fl_sim_create(&p->sim, grid, gamma, policy, boundary_mask);
  if (rc) {
    release(p);
    return rc;
  }
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < sets && e == cudaSuccess; ++i) {
    e = cudaMalloc(&p->a[i], (size_t)bytes);
    if (e == cudaSuccess) e = cudaMalloc(&p->b[i], (size_t)bytes);
  }
  if (e != cudaSuccess) {
    release(p);
    return set_error(kENoMem, "fl_host_pipe_create: %s", cudaGetErrorString(e));
  }
  e = cudaStreamCreateWithFlags(&p->s_in, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->s_run, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->s_out, cudaStreamNonBlocking);
  for (int i = 0; i < sets && e == cudaSuccess; ++i) {
    e = cudaEventCreateWithFlags(&p->ev_in[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_run[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_free[i], cudaEventDisableTiming);
    // every set starts free
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_free[i], p->s_out);
  }
  if (e != cudaSuccess) {
    release(p);
    return pipe_cuda(e, "fl_host_pipe_create");
  }
  *pipe = p;
  return kOk;
}

int fl_host_pipe_destroy(fl_host_pipe* pipe) {
  if (pipe == nullptr) return kOk;
  cudaStreamSynchronize(pipe->s_in);
  cudaStreamSynchronize(pipe->s_run);
  cudaStreamSynchronize(pipe->s_out);
  release(pipe);
  return kOk;
}

int fl_host_pipe_set_material(fl_host_pipe* pipe, const fl_material* mat) {
  if (pipe == nullptr) return set_error(kEInval, "pipe is NULL");
  return fl_sim_set_material(pipe->sim, mat);
}

int fl_host_pipe_run(fl_host_pipe* pipe, int32_t njobs, const void* const* host_in,
                     void* const* host_out, double cfl, double res, double sim_time,
                     int64_t max_iters, int64_t* iters, double* run_times) {
  if (pipe == nullptr || host_in == nullptr || host_out == nullptr)
    return set_error(kEInval, "NULL argument");
  if (njobs < 0) return set_error(kEInval, "njobs < 0");
  for (int32_t k = 0; k < njobs; ++k)
    if (host_in[k] == nullptr || host_out[k] == nullptr)
      return set_error(kEInval, "host buffer %d is NULL", (int)k);
  fl_host_pipe* p = pipe;
  const size_t nb = (size_t)p->bytes;
  auto upload = [&](int32_t k) -> cudaError_t {
    const int s = k % p->sets;
    cudaError_t e = cudaStreamWaitEvent(p->s_in, p->ev_free[s], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->a[s], host_in[k], nb, cudaMemcpyHostToDevice,
                                              p->s_in);
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_in[s], p->s_in);
    return e;
  };
  cudaError_t e = njobs > 0 ? upload(0) : cudaSuccess;
  if (e != cudaSuccess) return pipe_cuda(e, "fl_host_pipe_run");
  for (int32_t k = 0; k < njobs; ++k) {
    if (k + 1 < njobs && (e = upload(k + 1)) != cudaSuccess) return pipe_cuda(e, "fl_host_pipe_run");
    const int s = k % p->sets;
    e = cudaStreamWaitEvent(p->s_run, p->ev_in[s], 0);
    if (e != cudaSuccess) return pipe_cuda(e, "fl_host_pipe_run");
    int64_t it = 0;
    double rt = 0.0;
    void* result = nullptr;
    // blocks this thread until job k's loop has finished; the copy streams
    // keep running meanwhile
    int rc = fl_simulate(p->sim, p->a[s], p->b[s], cfl, res, sim_time, max_iters, p->s_run, &it,
                         &rt, &result);
    if (rc) return rc;
    if (iters) iters[k] = it;
    if (run_times) run_times[k] = rt;
    e = cudaEventRecord(p->ev_run[s], p->s_run);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s_out, p->ev_run[s], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(host_out[k], result, nb, cudaMemcpyDeviceToHost, p->s_out);
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_free[s], p->s_out);
    if (e != cudaSuccess) return pipe_cuda(e, "fl_host_pipe_run");
  }
  e = cudaStreamSynchronize(p->s_out);
  if (e != cudaSuccess) return pipe_cuda(e, "fl_host_pipe_run");
  return kOk;
}

}  // extern "C"
