// fl_tmap.cu -- tensor maps (TMA descriptors) of SoA state buffers.
//
// cuTensorMapEncodeTiled is a driver function; it is looked up once through
// the runtime (cudaGetDriverEntryPoint), so the library links only the CUDA
// runtime.  Encoding costs a few microseconds of host time, so maps are kept
// in a small cache keyed by buffer address, shape and box.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "fl_internal.cuh"

namespace fl {
namespace {

struct MapKey {
  const void* base;
  int64_t n0, n1, pitch;
  int planes, elem, box0, box1;
  bool operator==(const MapKey& o) const { return memcmp(this, &o, sizeof(MapKey)) == 0; }
};

struct MapEntry {
  MapKey key;
  CUtensorMap map;
  bool used;
};

constexpr int kCache = 32;
MapEntry g_cache[kCache];
int g_next = 0;
std::mutex g_mu;
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int resolve() {
  if (g_encode != nullptr) return kOk;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || fn == nullptr)
    return set_error(kECuda, "cuTensorMapEncodeTiled is not available from the driver");
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return kOk;
}

}  // namespace

int encode_state_map(void* map, const void* base, int64_t n0, int64_t n1, int64_t pitch,
                     int planes, int elem, int box0, int box1) {
  MapKey key;
  memset(&key, 0, sizeof(key));
  key.base = base;
  key.n0 = n0;
  key.n1 = n1;
  key.pitch = pitch;
  key.planes = planes;
  key.elem = elem;
  key.box0 = box0;
  key.box1 = box1;
  std::lock_guard<std::mutex> lock(g_mu);
  for (int i = 0; i < kCache; ++i) {
    if (g_cache[i].used && g_cache[i].key == key) {
      memcpy(map, &g_cache[i].map, sizeof(CUtensorMap));
      return kOk;
    }
  }
  int rc = resolve();
  if (rc) return rc;
  if ((reinterpret_cast<uintptr_t>(base) & 15u) || ((n0 * elem) & 15) || ((pitch * elem) & 15))
    return set_error(kEInval, "state buffer not 16-byte aligned for the staged sweep");
  CUtensorMap m;
  const cuuint64_t dims[3] = {(cuuint64_t)n0, (cuuint64_t)n1, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)(n0 * elem), (cuuint64_t)(pitch * elem)};
  const cuuint32_t box[3] = {(cuuint32_t)box0, (cuuint32_t)box1, (cuuint32_t)planes};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = g_encode(&m, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                        3, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(kECuda, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  MapEntry& slot = g_cache[g_next];
  g_next = (g_next + 1) % kCache;
  slot.key = key;
  slot.map = m;
  slot.used = true;
  memcpy(map, &m, sizeof(CUtensorMap));
  return kOk;
}

}  // namespace fl
