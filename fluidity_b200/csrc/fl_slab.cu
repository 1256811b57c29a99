// fl_slab.cu -- one 2-D grid decomposed into slabs of rows: the whole
// decomposed step enqueued below the host (include/fluidity_b200.h, fl_slab_*).
//
// A slab holds its own rows [own_lo, own_hi) of the local grid plus ghost
// rows facing its neighbours.  One step, on one stream:
//   exchange 3 ghost rows of buffer a -> sweep x (a -> b)
//   -> exchange 4 ghost rows of buffer b -> sweep y (b -> a, wavespeed of
//   own rows into the slab's word) -> MAX of the words over the slabs
//   -> finalize (dt, run time, stop test)
// The x sweep reads 3 rows across (the flattening coefficient takes the
// minimum over both dimensions), the y sweep 4 rows along (MUSCL-Hancock
// with flattening); a ghost row's own update is discarded, the next exchange
// overwrites it.  Nothing is read back to the host, so the steps can be
// captured in a CUDA graph.
//
// Transports:
//  * NCCL, one process (rank) per GPU: ncclSend / ncclRecv of each plane's
//    boundary rows into local ghost rows (no remote loads), and one 64-bit
//    MAX all-reduce of the wavespeed word per step.  libnccl.so.2 is loaded
//    at run time (the copy already in the process when there is one), so
//    the library loads without NCCL;
//  * in-process: several slabs held by one process, stepped together; the
//    exchange is a 2-D device copy from the neighbour's buffer and the
//    maximum a one-warp kernel over the slabs' words.  On one device this
//    runs every slab of a grid, in order, on one stream.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"

namespace {

constexpr int kRowsX = 3;           // ghost rows the x sweep reads
constexpr int kRowsY = 4;           // ghost rows the y sweep reads
constexpr int kMaxLocal = 16;       // slabs of one in-process group
constexpr int kParts = 6;           // sweep parts per step (3 per sweep)

// ---- NCCL, resolved at run time ---------------------------------------------
struct NcclApi {
  decltype(&ncclGetUniqueId) get_unique_id = nullptr;
  decltype(&ncclCommInitRank) comm_init_rank = nullptr;
  decltype(&ncclCommDestroy) comm_destroy = nullptr;
  decltype(&ncclGroupStart) group_start = nullptr;
  decltype(&ncclGroupEnd) group_end = nullptr;
  decltype(&ncclSend) send = nullptr;
  decltype(&ncclRecv) recv = nullptr;
  decltype(&ncclAllReduce) all_reduce = nullptr;
  decltype(&ncclGetErrorString) error_string = nullptr;
  bool ok = false;
};

const NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (h == nullptr) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (h == nullptr) return;
    NcclApi a;
    a.get_unique_id = reinterpret_cast<decltype(a.get_unique_id)>(dlsym(h, "ncclGetUniqueId"));
    a.comm_init_rank = reinterpret_cast<decltype(a.comm_init_rank)>(dlsym(h, "ncclCommInitRank"));
    a.comm_destroy = reinterpret_cast<decltype(a.comm_destroy)>(dlsym(h, "ncclCommDestroy"));
    a.group_start = reinterpret_cast<decltype(a.group_start)>(dlsym(h, "ncclGroupStart"));
    a.group_end = reinterpret_cast<decltype(a.group_end)>(dlsym(h, "ncclGroupEnd"));
    a.send = reinterpret_cast<decltype(a.send)>(dlsym(h, "ncclSend"));
    a.recv = reinterpret_cast<decltype(a.recv)>(dlsym(h, "ncclRecv"));
    a.all_reduce = reinterpret_cast<decltype(a.all_reduce)>(dlsym(h, "ncclAllReduce"));
    a.error_string = reinterpret_cast<decltype(a.error_string)>(dlsym(h, "ncclGetErrorString"));
    a.ok = a.get_unique_id && a.comm_init_rank && a.comm_destroy && a.group_start &&
           a.group_end && a.send && a.recv && a.all_reduce && a.error_string;
    api = a;
  });
  return api;
}

int nccl_fail(ncclResult_t r, const char* where) {
  const NcclApi& n = nccl();
  return fl::set_error(FL_ECUDA, "%s: %s", where, n.ok ? n.error_string(r) : "NCCL not loaded");
}

// The largest of the group's wavespeed words, written back to every word.
struct WordPtrs {
  unsigned long long* w[kMaxLocal];
};

__global__ void max_words_kernel(WordPtrs p, int count) {
  const int t = threadIdx.x;
  unsigned long long v = t < count ? *p.w[t] : 0ull;
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
    v = u > v ? u : v;
  }
  if (t < count) *p.w[t] = v;
}

}  // namespace

struct fl_slab {
  fl_sim* sim = nullptr;
  fl_grid grid{};
  int elem = 8;                      // bytes per value
  int64_t own_lo = 0, own_hi = 0;    // own rows of the local grid
  bool below = false, above = false;  // a neighbour below (lower rows) / above
  unsigned long long* word = nullptr;  // device wavespeed word
  // NCCL transport
  ncclComm_t comm = nullptr;
  int world = 1, rank = 0;
  bool nccl = false;
  // state buffers of the run in progress
  char* a = nullptr;
  char* b = nullptr;
  // the overlap: exchanges and collectives on a stream of the slab's own,
  // joined to the caller's stream by events
  cudaStream_t side = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // strip counters, a pair per sweep part (interior, lower edge, upper edge
  // of the x and the y sweep); each part takes slot `parity` and clears the
  // other, and parity flips every step
  unsigned int* counters = nullptr;
  int parity = 0;
  bool counters_dirty = false;
};

namespace {

int check_slab_args(const fl_grid* grid, int64_t own_lo, int64_t own_hi) {
  if (grid == nullptr || grid->dims != 2)
    return fl::set_error(FL_EINVAL, "slabs decompose 2-D grids");
  const int64_t ny = grid->n[1];
  if (!(0 <= own_lo && own_lo < own_hi && own_hi <= ny))
    return fl::set_error(FL_EINVAL, "own rows [%lld, %lld) outside [0, %lld)",
                         (long long)own_lo, (long long)own_hi, (long long)ny);
  if (own_hi - own_lo < kRowsY)
    return fl::set_error(FL_EINVAL, "a slab needs at least %d own rows", kRowsY);
  return FL_OK;
}

int make_slab(fl_slab** out, const fl_grid* grid, double gamma, uint32_t policy,
              uint32_t boundary_mask, int64_t own_lo, int64_t own_hi) {
  if (out == nullptr) return fl::set_error(FL_EINVAL, "slab is NULL");
  *out = nullptr;
  int rc = check_slab_args(grid, own_lo, own_hi);
  if (rc) return rc;
  fl_slab* s = new (std::nothrow) fl_slab();
  if (s == nullptr) return fl::set_error(FL_ENOMEM, "fl_slab");
  s->grid = *grid;
  s->elem = (policy & FL_DTYPE_F32) ? 4 : 8;
  s->own_lo = own_lo;
  s->own_hi = own_hi;
  rc = fl_sim_create(&s->sim, grid, gamma, policy, boundary_mask);
  if (rc == FL_OK) rc = fl_sim_set_rows(s->sim, own_lo, own_hi);
  if (rc == FL_OK) rc = fl_sim_set_external_reduce(s->sim, 1);
  if (rc == FL_OK) {
    const cudaError_t e = cudaMalloc(&s->word, sizeof(unsigned long long));
    if (e != cudaSuccess) rc = fl::set_error(FL_ENOMEM, "fl_slab: %s", cudaGetErrorString(e));
  }
  if (rc == FL_OK) rc = fl_sim_set_ws_word(s->sim, s->word);
  if (rc == FL_OK) {
    cudaError_t e = cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i)
      e = cudaEventCreateWithFlags(&s->ev[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&s->counters, kParts * 2 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(s->counters, 0, kParts * 2 * sizeof(unsigned int));
    if (e != cudaSuccess) rc = fl::set_error(FL_ECUDA, "fl_slab: %s", cudaGetErrorString(e));
  }
  if (rc != FL_OK) {
    fl_slab_destroy(s);
    return rc;
  }
  *out = s;
  return FL_OK;
}

// Ghost rows of `buf` (0: a, 1: b) of slab s from its neighbour's own rows,
// `rows` on each side.  In-process: neighbours are the adjacent slabs.
int exchange_local(fl_slab* const* g, int count, int buf, int rows, cudaStream_t st) {
  for (int i = 0; i < count; ++i) {
    fl_slab* s = g[i];
    char* dst = buf ? s->b : s->a;
    const size_t pitch = (size_t)s->grid.pitch * s->elem;
    const size_t width = (size_t)rows * s->grid.n[0] * s->elem;
    const int64_t nx = s->grid.n[0];
    if (i > 0) {
      const fl_slab* p = g[i - 1];
      const char* src = (buf ? p->b : p->a) + (size_t)(p->own_hi - rows) * nx * s->elem;
      const cudaError_t e = cudaMemcpy2DAsync(dst + (size_t)(s->own_lo - rows) * nx * s->elem,
                                              pitch, src, (size_t)p->grid.pitch * p->elem, width,
                                              4, cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return fl::set_error(FL_ECUDA, "fl_slab exchange: %s", cudaGetErrorString(e));
    }
    if (i < count - 1) {
      const fl_slab* q = g[i + 1];
      const char* src = (buf ? q->b : q->a) + (size_t)q->own_lo * nx * s->elem;
      const cudaError_t e = cudaMemcpy2DAsync(dst + (size_t)s->own_hi * nx * s->elem, pitch, src,
                                              (size_t)q->grid.pitch * q->elem, width, 4,
                                              cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return fl::set_error(FL_ECUDA, "fl_slab exchange: %s", cudaGetErrorString(e));
    }
  }
  return FL_OK;
}

int exchange_nccl(fl_slab* s, int buf, int rows, cudaStream_t st) {
  if (!s->below && !s->above) return FL_OK;
  const NcclApi& n = nccl();
  char* base = buf ? s->b : s->a;
  const int64_t nx = s->grid.n[0];
  const size_t bytes = (size_t)rows * nx * s->elem;
  ncclResult_t r = n.group_start();
  if (r != ncclSuccess) return nccl_fail(r, "ncclGroupStart");
  for (int c = 0; c < 4 && r == ncclSuccess; ++c) {
    char* plane = base + (size_t)c * s->grid.pitch * s->elem;
    if (s->below) {
      r = n.send(plane + (size_t)s->own_lo * nx * s->elem, bytes, ncclInt8, s->rank - 1, s->comm, st);
      if (r == ncclSuccess)
        r = n.recv(plane + (size_t)(s->own_lo - rows) * nx * s->elem, bytes, ncclInt8,
                   s->rank - 1, s->comm, st);
    }
    if (s->above && r == ncclSuccess) {
      r = n.send(plane + (size_t)(s->own_hi - rows) * nx * s->elem, bytes, ncclInt8, s->rank + 1,
                 s->comm, st);
      if (r == ncclSuccess)
        r = n.recv(plane + (size_t)s->own_hi * nx * s->elem, bytes, ncclInt8, s->rank + 1, s->comm,
                   st);
    }
  }
  const ncclResult_t r2 = n.group_end();
  if (r != ncclSuccess) return nccl_fail(r, "fl_slab exchange");
  if (r2 != ncclSuccess) return nccl_fail(r2, "ncclGroupEnd");
  return FL_OK;
}

int exchange(fl_slab* const* g, int count, int buf, int rows, cudaStream_t st) {
  return g[0]->nccl ? exchange_nccl(g[0], buf, rows, st) : exchange_local(g, count, buf, rows, st);
}

int reduce_words(fl_slab* const* g, int count, cudaStream_t st) {
  if (g[0]->nccl) {
    fl_slab* s = g[0];
    if (s->comm == nullptr) return FL_OK;
    const ncclResult_t r =
        nccl().all_reduce(s->word, s->word, 1, ncclUint64, ncclMax, s->comm, st);
    return r == ncclSuccess ? FL_OK : nccl_fail(r, "fl_slab all-reduce");
  }
  if (count == 1) return FL_OK;
  WordPtrs p{};
  for (int i = 0; i < count; ++i) p.w[i] = g[i]->word;
  max_words_kernel<<<1, 32, 0, st>>>(p, count);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FL_OK : fl::set_error(FL_ECUDA, "fl_slab reduce: %s", cudaGetErrorString(e));
}

// The group of one call: one NCCL slab, or in-process slabs bottom to top
// with matching row width and dtype and ghost rows where they meet.
int check_group(fl_slab* const* g, int count) {
  if (g == nullptr || count < 1) return fl::set_error(FL_EINVAL, "no slabs");
  for (int i = 0; i < count; ++i)
    if (g[i] == nullptr) return fl::set_error(FL_EINVAL, "slab %d is NULL", i);
  if (g[0]->nccl) {
    if (count != 1) return fl::set_error(FL_EINVAL, "an NCCL slab is stepped alone (one per rank)");
    return FL_OK;
  }
  if (count > kMaxLocal) return fl::set_error(FL_EINVAL, "at most %d in-process slabs", kMaxLocal);
  for (int i = 0; i < count; ++i) {
    const fl_slab* s = g[i];
    if (s->nccl) return fl::set_error(FL_EINVAL, "slab %d belongs to an NCCL group", i);
    if (s->grid.n[0] != g[0]->grid.n[0] || s->elem != g[0]->elem)
      return fl::set_error(FL_EINVAL, "slab %d differs in row width or dtype", i);
    if (i > 0 && s->own_lo < kRowsY)
      return fl::set_error(FL_EINVAL, "slab %d has %lld ghost rows below, %d needed", i,
                           (long long)s->own_lo, kRowsY);
    if (i < count - 1 && s->grid.n[1] - s->own_hi < kRowsY)
      return fl::set_error(FL_EINVAL, "slab %d has %lld ghost rows above, %d needed", i,
                           (long long)(s->grid.n[1] - s->own_hi), kRowsY);
  }
  return FL_OK;
}

}  // namespace

extern "C" {

int fl_slab_nccl_available(void) { return nccl().ok ? 1 : 0; }

int fl_slab_nccl_id(void* id) {
  if (id == nullptr) return fl::set_error(FL_EINVAL, "id is NULL");
  const NcclApi& n = nccl();
  if (!n.ok) return fl::set_error(FL_EINVAL, "libnccl.so.2 could not be loaded");
  ncclUniqueId u;
  const ncclResult_t r = n.get_unique_id(&u);
  if (r != ncclSuccess) return nccl_fail(r, "ncclGetUniqueId");
  std::memcpy(id, &u, sizeof(u));
  return FL_OK;
}

int fl_slab_create_nccl(fl_slab** slab, const fl_grid* grid, double gamma, uint32_t policy,
                        uint32_t boundary_mask, int64_t own_lo, int64_t own_hi,
                        const void* nccl_id, int world, int rank) {
  if (world < 1 || rank < 0 || rank >= world)
    return fl::set_error(FL_EINVAL, "rank %d of %d", rank, world);
  if (world > 1 && nccl_id == nullptr) return fl::set_error(FL_EINVAL, "nccl_id is NULL");
  if (nccl_id != nullptr && !nccl().ok)
    return fl::set_error(FL_EINVAL, "libnccl.so.2 could not be loaded");
  if (grid != nullptr && grid->dims == 2) {
    if (rank > 0 && own_lo < kRowsY)
      return fl::set_error(FL_EINVAL, "rank %d has %lld ghost rows below, %d needed", rank,
                           (long long)own_lo, kRowsY);
    if (rank < world - 1 && grid->n[1] - own_hi < kRowsY)
      return fl::set_error(FL_EINVAL, "rank %d has %lld ghost rows above, %d needed", rank,
                           (long long)(grid->n[1] - own_hi), kRowsY);
  }
  int rc = make_slab(slab, grid, gamma, policy, boundary_mask, own_lo, own_hi);
  if (rc) return rc;
  fl_slab* s = *slab;
  s->nccl = true;
  s->world = world;
  s->rank = rank;
  s->below = rank > 0;
  s->above = rank < world - 1;
  if (nccl_id != nullptr) {  // world 1 with an id: a communicator of one rank
    ncclUniqueId u;
    std::memcpy(&u, nccl_id, sizeof(u));
    const ncclResult_t r = nccl().comm_init_rank(&s->comm, world, u, rank);
    if (r != ncclSuccess) {
      rc = nccl_fail(r, "ncclCommInitRank");
      fl_slab_destroy(s);
      *slab = nullptr;
      return rc;
    }
  }
  return FL_OK;
}

int fl_slab_create_local(fl_slab** slab, const fl_grid* grid, double gamma, uint32_t policy,
                         uint32_t boundary_mask, int64_t own_lo, int64_t own_hi) {
  return make_slab(slab, grid, gamma, policy, boundary_mask, own_lo, own_hi);
}

int fl_slab_set_material(fl_slab* slab, const fl_material* mat) {
  if (slab == nullptr) return fl::set_error(FL_EINVAL, "slab is NULL");
  return fl_sim_set_material(slab->sim, mat);
}

int fl_slab_sim(fl_slab* slab, fl_sim** sim) {
  if (slab == nullptr || sim == nullptr) return fl::set_error(FL_EINVAL, "NULL argument");
  *sim = slab->sim;
  return FL_OK;
}

int fl_slab_begin(fl_slab* const* slabs, int count, void* const* a, void* const* b, double cfl,
                  double res, double sim_time, int64_t max_iters, void* stream) {
  int rc = check_group(slabs, count);
  if (rc) return rc;
  if (a == nullptr || b == nullptr) return fl::set_error(FL_EINVAL, "buffers are NULL");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int i = 0; i < count; ++i) {
    if (a[i] == nullptr || b[i] == nullptr) return fl::set_error(FL_EINVAL, "slab %d buffer NULL", i);
    slabs[i]->a = static_cast<char*>(a[i]);
    slabs[i]->b = static_cast<char*>(b[i]);
    rc = fl_sim_begin(slabs[i]->sim, a[i], b[i], cfl, res, sim_time, max_iters, stream);
    if (rc) return rc;
  }
  // below/above of in-process slabs follow their place in the group
  if (!slabs[0]->nccl)
    for (int i = 0; i < count; ++i) {
      slabs[i]->below = i > 0;
      slabs[i]->above = i < count - 1;
    }
  rc = reduce_words(slabs, count, st);
  for (int i = 0; i < count && rc == FL_OK; ++i) rc = fl_sim_finalize(slabs[i]->sim, 0, stream);
  return rc;
}

int fl_slab_steps(fl_slab* const* slabs, int count, int64_t nsteps, void* stream) {
  int rc = check_group(slabs, count);
  if (rc) return rc;
  for (int i = 0; i < count; ++i)
    if (slabs[i]->a == nullptr) return fl::set_error(FL_EINVAL, "fl_slab_begin not called");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  fl_slab* g0 = slabs[0];  // its side stream and events serve the group
  cudaStream_t side = g0->side;
  auto ok = [](cudaError_t e) {
    return e == cudaSuccess ? FL_OK : fl::set_error(FL_ECUDA, "fl_slab_steps: %s",
                                                    cudaGetErrorString(e));
  };
  // One sweep of every slab in three parts: the rows that need no ghost row
  // (the interior, launched while the exchange runs on the side stream),
  // then, once the exchange is in, the `reach` rows at each edge that faces
  // a neighbour.
  auto sweep = [&](int dim, int reach, cudaEvent_t exchanged) -> int {
    int r = FL_OK;
    for (int i = 0; i < count && r == FL_OK; ++i) {
      fl_slab* s = slabs[i];
      const int64_t lo = s->own_lo + (s->below ? reach : 0);
      const int64_t hi = s->own_hi - (s->above ? reach : 0);
      if (lo < hi)
        r = fl::sim_sweep_part(s->sim, dim, lo, hi, s->counters + (dim * 3 + 0) * 2, s->parity,
                               0, stream);
    }
    if (r == FL_OK) r = ok(cudaStreamWaitEvent(st, exchanged, 0));
    for (int i = 0; i < count && r == FL_OK; ++i) {
      fl_slab* s = slabs[i];
      const int64_t lo = s->own_lo + (s->below ? reach : 0);
      const int64_t hi = s->own_hi - (s->above ? reach : 0);
      const int64_t bot_hi = lo < s->own_hi ? lo : s->own_hi;
      const int64_t top_lo = hi > bot_hi ? hi : bot_hi;
      r = fl::sim_sweep_part(s->sim, dim, s->own_lo, bot_hi, s->counters + (dim * 3 + 1) * 2,
                             s->parity, 0, stream);
      if (r == FL_OK)
        r = fl::sim_sweep_part(s->sim, dim, top_lo, s->own_hi, s->counters + (dim * 3 + 2) * 2,
                               s->parity, 1, stream);
    }
    return r;
  };
  for (int64_t k = 0; k < nsteps; ++k) {
    for (int i = 0; i < count && rc == FL_OK; ++i)
      if (slabs[i]->counters_dirty) {
        rc = ok(cudaMemsetAsync(slabs[i]->counters, 0, kParts * 2 * sizeof(unsigned int), st));
        if (rc == FL_OK) slabs[i]->counters_dirty = false;
      }
    // x sweep: exchange 3 ghost rows of a on the side stream meanwhile
    if (rc == FL_OK) rc = ok(cudaEventRecord(g0->ev[0], st));
    if (rc == FL_OK) rc = ok(cudaStreamWaitEvent(side, g0->ev[0], 0));
    if (rc == FL_OK) rc = exchange(slabs, count, 0, kRowsX, side);
    if (rc == FL_OK) rc = ok(cudaEventRecord(g0->ev[1], side));
    if (rc == FL_OK) rc = sweep(0, kRowsX, g0->ev[1]);
    // y sweep: exchange 4 ghost rows of b (written by the x sweep's edges)
    if (rc == FL_OK) rc = ok(cudaEventRecord(g0->ev[2], st));
    if (rc == FL_OK) rc = ok(cudaStreamWaitEvent(side, g0->ev[2], 0));
    if (rc == FL_OK) rc = exchange(slabs, count, 1, kRowsY, side);
    if (rc == FL_OK) rc = ok(cudaEventRecord(g0->ev[3], side));
    if (rc == FL_OK) rc = sweep(1, kRowsY, g0->ev[3]);
    // the wavespeed maximum (NCCL on the side stream, after the y sweep),
    // then the step
    if (rc == FL_OK) {
      if (g0->nccl) {
        rc = ok(cudaEventRecord(g0->ev[0], st));
        if (rc == FL_OK) rc = ok(cudaStreamWaitEvent(side, g0->ev[0], 0));
        if (rc == FL_OK) rc = reduce_words(slabs, count, side);
        if (rc == FL_OK) rc = ok(cudaEventRecord(g0->ev[1], side));
        if (rc == FL_OK) rc = ok(cudaStreamWaitEvent(st, g0->ev[1], 0));
      } else {
        rc = reduce_words(slabs, count, st);
      }
    }
    for (int i = 0; i < count && rc == FL_OK; ++i) rc = fl_sim_finalize(slabs[i]->sim, 1, stream);
    if (rc) {
      for (int i = 0; i < count; ++i) slabs[i]->counters_dirty = true;
      return rc;
    }
    for (int i = 0; i < count; ++i) slabs[i]->parity ^= 1;
  }
  return FL_OK;
}

int fl_slab_destroy(fl_slab* slab) {
  if (slab == nullptr) return FL_OK;
  if (slab->comm != nullptr && nccl().ok) nccl().comm_destroy(slab->comm);
  for (int i = 0; i < 4; ++i)
    if (slab->ev[i] != nullptr) cudaEventDestroy(slab->ev[i]);
  if (slab->side != nullptr) cudaStreamDestroy(slab->side);
  if (slab->counters != nullptr) cudaFree(slab->counters);
  if (slab->word) cudaFree(slab->word);
  if (slab->sim) fl_sim_destroy(slab->sim);
  delete slab;
  return FL_OK;
}

}  // extern "C"
