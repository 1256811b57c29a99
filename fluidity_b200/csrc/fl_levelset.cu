// fl_levelset.cu -- level-set kernels of the multimaterial path and their C
// ABI (include/fluidity_b200.h, fl_ls_*).
//
//  * fl_ls_velocity : interface-normal velocity from the first material
//    containing each cell (levelset/cuda/velocity_initialization.cuh:108-143);
//  * fl_ls_advect   : one TVD-RK3 step of phi_t + v |grad phi| = 0 with
//    WENO-HJ5 one-sided derivatives and the Godunov upwind Hamiltonian
//    (scheme/stencils/weno_hj_5.hpp, schemes/godunov_upwind.hpp,
//    evaluators/levelset_hamiltonian.hpp, updaters/runge_kutta_3.hpp); every
//    stage is one launch over the whole grid, so tile halos always hold the
//    current stage (the reference's single-launch RK3 keeps stale halos
//    between stages, scheme/cuda/evolve.cuh:51-157); the stages are in
//    fl_ls_rk3.cu, which is built with FMA contraction and agrees with the
//    reference's operation order to rounding;
//  * fl_ls_project  : two level sets without overlap or void
//    (levelset/cuda/levelset_projection.cuh:54-67);
//  * fl_ls_reinit   : signed-distance reinitialisation: sources next to the
//    interface keep |phi| (scheme/cuda/fast_iterative_method.cuh:48-89, which
//    seeds the signed value), every other cell
//    relaxes to the fixed point of the Godunov local eikonal solve
//    (schemes/godunov_upwind_scheme.hpp:44-53); 16x16 tiles relax in shared
//    memory, passes ping-pong between two buffers, only tiles stamped by a
//    changed neighbour relax in the next pass (a worklist: a changed tile
//    and those of its 4 edge neighbours whose shared edge changed; the
//    others hold the same values in both buffers), and the host checks
//    convergence once per 16 passes; the result takes the
//    input's sign (set_signs, :96-112).
// FP64 level sets on 2-D grids; out-of-domain reads mirror the domain.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"

namespace fl {
namespace {

__device__ __forceinline__ int64_t lmir(int64_t i, int64_t n) {
  if (i < 0) i = -1 - i;
  else if (i >= n) i = 2 * n - 1 - i;
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }

template <typename T>
__global__ void ls_velocity_kernel(int64_t nx, int64_t ny, int nmat, const double* phi0,
                                   const double* phi1, const T* u0, const T* u1, int64_t pitch,
                                   double h, double* vel) {
  const int64_t n = nx * ny;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = i % nx, y = i / nx;
    double v = 0.0;
    for (int m = 0; m < nmat; ++m) {
      const double* f = m == 0 ? phi0 : phi1;
      const T* u = m == 0 ? u0 : u1;
      if (!(f[i] <= 0.0 || f[i] <= -0.0)) continue;
      const double fact = 0.5 / h;
      const double g0 = fact * (f[y * nx + lmir(x + 1, nx)] - f[y * nx + lmir(x - 1, nx)]);
      const double g1 = fact * (f[lmir(y + 1, ny) * nx + x] - f[lmir(y - 1, ny) * nx + x]);
      const double s = sqrt(g0 * g0 + g1 * g1);
      const double rho = (double)u[i];
      v = ((double)u[2 * pitch + i] / rho) * (g0 / s) + ((double)u[3 * pitch + i] / rho) * (g1 / s);
      break;
    }
    vel[i] = v;
  }
}

__global__ void ls_project_kernel(int64_t n, double* a, double* b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double avg = __dmul_rn(0.5, a[i] + b[i]);  // no contraction into the subtraction
    a[i] -= avg;
    b[i] = -a[i];
  }
}

// ---- reinitialisation ------------------------------------------------------

#ifndef FL_FIM_TILE
#define FL_FIM_TILE 16
#endif
#ifndef FL_FIM_PERSIST
#define FL_FIM_PERSIST 1
#endif
constexpr int FT = FL_FIM_TILE;              // tile side
// In-tile relaxation rounds per pass.  2 * tile lets a front cross the tile
// (and back) within one pass: on the 2048 x 1024 shock-bubble level set the
// passes drop from 100 to 77 and a reinitialisation from 4.88 to 3.69 ms
// (1.5 * tile before; 40, 48 and 64 rounds keep 77 passes but cost more).
#ifndef FL_FIM_INNER
#define FL_FIM_INNER (2 * FL_FIM_TILE)
#endif
constexpr int FIM_INNER = FL_FIM_INNER;

__device__ __forceinline__ int dsgn(double v) { return (0.0 < v) - (v < 0.0); }

__global__ void fim_init_kernel(const double* phi, int64_t nx, int64_t ny, double* dist,
                                unsigned char* fixed) {
  const int64_t n = nx * ny;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = i % nx, y = i / nx;
    const double c = phi[i];
    bool s = false;
    for (int d = 0; d < 2 && !s; ++d)
      for (int k = -1; k <= 1 && !s; k += 2) {
        const int64_t xx = lmir(x + (d == 0 ? k : 0), nx), yy = lmir(y + (d == 1 ? k : 0), ny);
        const double o = phi[yy * nx + xx];
        if (dsgn(c) != dsgn(o) && fabs(c) < fabs(o)) s = true;
      }
    fixed[i] = s ? 1 : 0;
    dist[i] = s ? fabs(c) : DBL_MAX;
  }
}

// Godunov upwind local solve (godunov_upwind_scheme.hpp:44-53).
__device__ __forceinline__ double eik_local(double xm, double xp, double ym, double yp, double h) {
  const double a = dmin_(xm, xp), b = dmin_(ym, yp);
  const double fh = 1.0 * h;
  const double amb = a - b;
  if (fabs(amb) >= fh) return dmin_(a, b) + fh;
  return 0.5 * (a + b + sqrt(2.0 * fh * fh - (amb * amb)));
}

// Pass k over a worklist of tiles: reads src (the previous pass) and writes
// dst.  Pass 0 relaxes every tile; pass k > 0 relaxes the tiles that a tile
// which changed in pass k - 1 stamped (itself, and each of its 4 edge
// neighbours whose shared edge changed), each listed once.  A relaxing tile loads itself and a one-cell halo (+max
// outside the domain), relaxes FIM_INNER rounds in shared memory and writes
// its cells to dst.  A tile off the list holds the same values in both
// buffers: it last relaxed without a change (a tile that changes always
// relaxes again in the next pass), so it needs no copy.  Every pass depends
// only on the previous one, so the result is deterministic.
//   lists:  3 lists of up to `tiles` entries; pass k reads list k % 3,
//           appends to list (k + 1) % 3 and clears the count of list
//           (k + 2) % 3, which pass k - 1 has finished with.
//   counts: the 3 list lengths.
// A pass after one that changed nothing returns at once (last_change < k - 1).
__global__ void __launch_bounds__(FT * FT) fim_pass_kernel(
    const double* __restrict__ src, double* __restrict__ dst,
    const unsigned char* __restrict__ fixed, int64_t nx, int64_t ny, double h,
    int* __restrict__ stamp, int* __restrict__ lists, int* __restrict__ counts, int tiles_x,
    int tiles_y, int* __restrict__ last_change, int k) {
  if (k > 0 && *(volatile int*)last_change < k - 1) return;
  __shared__ double s[FT + 2][FT + 2];
  __shared__ int changed;
  const int lx = threadIdx.x % FT, ly = threadIdx.x / FT;
  const int tiles = tiles_x * tiles_y;
  const int* list = lists + (k % 3) * tiles;
  int* next = lists + ((k + 1) % 3) * tiles;
  int* next_count = counts + (k + 1) % 3;
  if (blockIdx.x == 0 && threadIdx.x == 0) counts[(k + 2) % 3] = 0;
  const int count = (k == 0) ? tiles : *(volatile int*)(counts + k % 3);
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const int t = (k == 0) ? i : list[i];
    const int tx0 = t % tiles_x, ty0 = t / tiles_x;
    const int64_t x = (int64_t)tx0 * FT + lx, y = (int64_t)ty0 * FT + ly;
    const bool in = x < nx && y < ny;
    const int64_t ci = y * nx + x;
    if (threadIdx.x == 0) changed = 0;
    // the cell's fixed flag is loaded with the tile, before the barrier
    const bool free_cell = in && !fixed[ci];
    for (int q = threadIdx.x; q < (FT + 2) * (FT + 2); q += FT * FT) {
      const int hx = q % (FT + 2), hy = q / (FT + 2);
      const int64_t gx = (int64_t)tx0 * FT + hx - 1, gy = (int64_t)ty0 * FT + hy - 1;
      s[hy][hx] = (gx >= 0 && gx < nx && gy >= 0 && gy < ny) ? src[gy * nx + gx] : DBL_MAX;
    }
    __syncthreads();
    bool mine = false;
    // up to FIM_INNER rounds; a round that changes no cell of the tile ends
    // them (the next round would see the same values: same result)
    for (int r = 0; r < FIM_INNER; ++r) {
      double q = 0.0;
      if (free_cell)
        q = eik_local(s[ly + 1][lx], s[ly + 1][lx + 2], s[ly][lx + 1], s[ly + 2][lx + 1], h);
      __syncthreads();
      const bool upd = free_cell && q < s[ly + 1][lx + 1];
      if (upd) {
        s[ly + 1][lx + 1] = q;
        mine = true;
      }
      if (!__syncthreads_or(upd)) break;
    }
    if (in) dst[ci] = s[ly + 1][lx + 1];
    // bit 0: a cell of the tile changed (the tile relaxes again next pass,
    // which also brings the other buffer up to date); bits 1-4: a changed
    // cell on the left, right, lower, upper edge.  The local solve reads the
    // 4 edge neighbours only, so only the edge-adjacent tiles whose shared
    // edge changed need the next pass.
    if (mine)
      atomicOr(&changed, 1 | (lx == 0 ? 2 : 0) | (lx == FT - 1 ? 4 : 0) | (ly == 0 ? 8 : 0) |
                             (ly == FT - 1 ? 16 : 0));
    __syncthreads();
    if (threadIdx.x == 0 && changed) {
      atomicMax(last_change, k);
      const int dxs[5] = {0, -1, 1, 0, 0}, dys[5] = {0, 0, 0, -1, 1};
      for (int q = 0; q < 5; ++q) {
        if (!(changed & (1 << q))) continue;
        const int ax = tx0 + dxs[q], ay = ty0 + dys[q];
        if (ax < 0 || ax >= tiles_x || ay < 0 || ay >= tiles_y) continue;
        const int nt = ay * tiles_x + ax;
        if (atomicMax(stamp + nt, k + 1) < k + 1) next[atomicAdd(next_count, 1)] = nt;
      }
    }
    __syncthreads();   // s and changed are reused by the next tile
  }
}

__global__ void fim_sign_kernel(const double* phi, double* out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)dsgn(phi[i]) * fabs(out[i]);
}

__global__ void fill_int_kernel(int* p, int n, int v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

int check_ls_grid(const fl_grid* g) {
  if (g == nullptr) return set_error(kEInval, "grid is NULL");
  if (g->dims != 2) return set_error(kEInval, "level-set kernels are 2-D");
  if (g->n[0] < 4 || g->n[1] < 4 || g->n[2] != 1)
    return set_error(kEInval, "level-set grid needs n[0], n[1] >= 4 and n[2] = 1");
  return kOk;
}

unsigned grid1d(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (unsigned)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace

// The three RK3 stages of fl_ls_advect (fl_ls_rk3.cu, built with FMA
// contraction; the kernels here are built without it).
cudaError_t launch_ls_rk3(const double* phi, const double* vel, double dt, double h, int64_t nx,
                          int64_t ny, double* s1, double* s2, double* out, cudaStream_t st);

}  // namespace fl

using namespace fl;

extern "C" {

int64_t fl_ls_workspace_bytes(const fl_grid* grid) {
  if (check_ls_grid(grid) != kOk) return -1;
  const int64_t n = grid->n[0] * grid->n[1];
  const int64_t tiles = ((grid->n[0] + FT - 1) / FT) * ((grid->n[1] + FT - 1) / FT);
  // two FP64 planes (RK3 stages; the first also the reinitialisation's
  // second buffer), its fixed-cell flags, tile stamps, three tile
  // worklists, and the change counter with the list counts, each 256-byte
  // aligned
  auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
  return al(2 * n * 8) + al(n) + al(tiles * 4) + al(3 * tiles * 4) + 256;
}

int fl_ls_velocity(const fl_grid* grid, int nmat, const double* const* phis,
                   const void* const* states, int64_t pitch, uint32_t policy, double h,
                   double* vel, void* stream) {
  int rc = check_ls_grid(grid);
  if (rc) return rc;
  if (nmat < 1 || nmat > 2) return set_error(kEInval, "nmat must be 1 or 2");
  if (!phis || !states || !vel) return set_error(kEInval, "NULL pointer");
  for (int m = 0; m < nmat; ++m)
    if (!phis[m] || !states[m]) return set_error(kEInval, "NULL material %d", m);
  if (pitch < grid->n[0] * grid->n[1]) return set_error(kEInval, "pitch below the cell count");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = grid->n[0] * grid->n[1];
  const double* p1 = nmat > 1 ? phis[1] : phis[0];
  if (policy & 1u) {
    const float* u1 = static_cast<const float*>(nmat > 1 ? states[1] : states[0]);
    ls_velocity_kernel<float><<<grid1d(n), 256, 0, st>>>(grid->n[0], grid->n[1], nmat, phis[0], p1,
                                                         static_cast<const float*>(states[0]), u1,
                                                         pitch, h, vel);
  } else {
    const double* u1 = static_cast<const double*>(nmat > 1 ? states[1] : states[0]);
    ls_velocity_kernel<double><<<grid1d(n), 256, 0, st>>>(grid->n[0], grid->n[1], nmat, phis[0],
                                                          p1, static_cast<const double*>(states[0]),
                                                          u1, pitch, h, vel);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(kECuda, "fl_ls_velocity: %s", cudaGetErrorString(e));
  return kOk;
}

int fl_ls_advect(const fl_grid* grid, const double* phi, const double* vel, double dt, double h,
                 double* out, void* workspace, void* stream) {
  int rc = check_ls_grid(grid);
  if (rc) return rc;
  if (!phi || !vel || !out || !workspace) return set_error(kEInval, "NULL pointer");
  if (out == phi) return set_error(kEInval, "out must differ from phi");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t nx = grid->n[0], ny = grid->n[1], n = nx * ny;
  double* s1 = static_cast<double*>(workspace);
  const cudaError_t e = launch_ls_rk3(phi, vel, dt, h, nx, ny, s1, s1 + n, out, st);
  if (e != cudaSuccess) return set_error(kECuda, "fl_ls_advect: %s", cudaGetErrorString(e));
  return kOk;
}

int fl_ls_project(int64_t cells, double* a, double* b, void* stream) {
  if (cells <= 0 || !a || !b) return set_error(kEInval, "bad arguments");
  ls_project_kernel<<<grid1d(cells), 256, 0, static_cast<cudaStream_t>(stream)>>>(cells, a, b);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(kECuda, "fl_ls_project: %s", cudaGetErrorString(e));
  return kOk;
}

int fl_ls_reinit(const fl_grid* grid, const double* phi, double h, double* out, void* workspace,
                 int max_passes, int* passes, void* stream) {
  int rc = check_ls_grid(grid);
  if (rc) return rc;
  if (!phi || !out || !workspace) return set_error(kEInval, "NULL pointer");
  if (out == phi) return set_error(kEInval, "out must differ from phi");
  if (max_passes <= 0) return set_error(kEInval, "max_passes must be positive");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t nx = grid->n[0], ny = grid->n[1], n = nx * ny;
  const int tiles_x = (int)((nx + FT - 1) / FT), tiles_y = (int)((ny + FT - 1) / FT);
  const int tiles = tiles_x * tiles_y;
  auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
  char* w = static_cast<char*>(workspace);
  unsigned char* fixed = reinterpret_cast<unsigned char*>(w + al(2 * n * 8));
  int* stamp = reinterpret_cast<int*>(w + al(2 * n * 8) + al(n));
  int* lists = reinterpret_cast<int*>(w + al(2 * n * 8) + al(n) + al(tiles * 4));
  int* last = reinterpret_cast<int*>(w + al(2 * n * 8) + al(n) + al(tiles * 4) +
                                     al(3 * tiles * 4));
  int* counts = last + 1;
  // passes ping-pong between `out` (even passes read it) and the first
  // workspace plane
  double* buf[2] = {out, reinterpret_cast<double*>(w)};
  fim_init_kernel<<<grid1d(n), 256, 0, st>>>(phi, nx, ny, out, fixed);
  fill_int_kernel<<<grid1d(tiles), 256, 0, st>>>(stamp, tiles, 0);
  fill_int_kernel<<<1, 32, 0, st>>>(last, 4, 0);   // last change, 3 list counts
  // passes are launched in chunks; the host reads the last pass that changed
  // anything after each chunk (passes past convergence return at once)
  constexpr int CHUNK = 16;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_sm = 2048 / (FT * FT);
  const int pass_ctas = (FL_FIM_PERSIST && tiles > sms * per_sm) ? sms * per_sm : tiles;
  int launched = 0, h_last = 0;
  bool converged = false;
  cudaError_t e = cudaGetLastError();
  while (e == cudaSuccess && !converged && launched < max_passes) {
    const int end = launched + CHUNK < max_passes ? launched + CHUNK : max_passes;
    for (int k = launched; k < end; ++k)
      fim_pass_kernel<<<pass_ctas, FT * FT, 0, st>>>(buf[k & 1], buf[(k + 1) & 1], fixed, nx, ny,
                                                     h, stamp, lists, counts, tiles_x, tiles_y,
                                                     last, k);
    launched = end;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_last, last, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    // converged once a pass after the last change has run
    converged = (e == cudaSuccess) && (h_last + 1 < launched);
  }
  // the last pass that ran (h_last + 1, which changed nothing) wrote
  // buf[(h_last + 2) & 1]
  if (e == cudaSuccess && converged && ((h_last + 2) & 1))
    e = cudaMemcpyAsync(out, buf[1], n * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess && !converged && (launched & 1))
    e = cudaMemcpyAsync(out, buf[1], n * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) {
    fim_sign_kernel<<<grid1d(n), 256, 0, st>>>(phi, out, n);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return set_error(kECuda, "fl_ls_reinit: %s", cudaGetErrorString(e));
  if (passes) *passes = converged ? h_last + 2 : launched;
  if (!converged)
    return set_error(kETimeout, "reinitialisation did not converge in %d passes", launched);
  return kOk;
}

}  // extern "C"
