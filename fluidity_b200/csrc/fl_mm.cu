// fl_mm.cu -- the two-material ghost-fluid path on one GPU: Riemann ghost-fluid
// star states, ghost-cell extrapolation, state initialisation inside a level
// set, the final merge, and the step loop that ties them to the split solver
// and the level-set kernels (include/fluidity_b200.h, fl_mm_*).
//
// One step (simulator/multimaterial_simulator.hpp:254-286):
//   1. interface scan (one launch, both materials): band cells of the
//      extrapolation go to a list; every cell that is the target of a GFM
//      source pulls its winning source (highest flat index among the up to 8
//      neighbours whose normal points at it), computes the star state from
//      the pre-pass states and appends (cell, state) to a list;
//   2. scatter of the star states (one launch);
//   3. extrapolation: one CTA per material iterates Jacobi sweeps over its band
//      list, ping-ponging band cells between the state and the material's
//      second buffer, until no cell moves by 1e-8 (one launch);
//   4. CFL time step from the max wavespeed of both materials (read back);
//   5. split MUSCL-Hancock step of each material with its own gamma;
//   6. level-set velocity, RK3 advection of both level sets, projection and,
//      every `reinit_every` steps, reinitialisation.
// Arithmetic of the GFM and the extrapolation is FP64 whatever the state
// precision; values are rounded to the state type when stored.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"

namespace fl {
// One dimensional sweep of the split step with strip counters (nullable) and
// the counters' parity slot: fl_split_sweep_mat for callers that own
// counters (the two-material loop).
int split_sweep_counted(const fl_grid* grid, int dim, const void* in, void* out,
                        const fl_material* mat, double dtdh, uint32_t policy,
                        uint32_t boundary_mask, double* max_ws_out, unsigned int* walk_next,
                        int walk_slot, void* stream, void* scratch = nullptr,
                        int* status = nullptr);

namespace {

struct MMCounters {
  int band[2];     // band cells per material
  int gfm[2];      // GFM targets per material
  int iters[2];    // Jacobi sweeps of the last extrapolation
  int stop[2];     // 1 once the material's extrapolation has converged
  // the extrapolation sweep in flight: max change (bits of a non-negative
  // double) and NaN flag per material and sweep parity, blocks arrived
  unsigned long long err[2][2];
  int nan[2][2];
  unsigned int arrive;
  int pad;
};

struct MMArgs {
  int64_t nx, ny, pitch;
  double h;
  double gamma[2];
  double pinf[2];       // stiffened fluids' p_inf (0: ideal gas)
  const void* u[2];     // states (read by the scan)
  void* w[2];           // states (written by scatter / extrapolation)
  void* x[2];           // second buffers (Jacobi ping-pong)
  const double* phi[2];
  MMCounters* cnt;
  int* band_list[2];
  int* gfm_idx[2];
  double* gfm_state[2];  // 4 doubles per target
  int max_iters;
};

__device__ __forceinline__ int64_t mir(int64_t i, int64_t n) {
  if (i < 0) i = -1 - i;
  else if (i >= n) i = 2 * n - 1 - i;
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}
__device__ __forceinline__ int64_t midx(int64_t nx, int64_t ny, int64_t x, int64_t y) {
  return mir(y, ny) * nx + mir(x, nx);
}
__device__ __forceinline__ int isgn(double v) { return (0.0 < v) - (v < 0.0); }
__device__ __forceinline__ double dmaxr(double a, double b) { return (a < b) ? b : a; }

template <typename T>
__device__ __forceinline__ void load4(const T* u, int64_t pitch, int64_t i, double* o) {
#pragma unroll
  for (int c = 0; c < 4; ++c) o[c] = (double)u[c * pitch + i];
}

// ideal gas (state/state_impl.hpp:117-128, material/ideal_gas.hpp:75-78)
__device__ __forceinline__ double pressure2(const double* u, double g) {
  const double r = u[0];
  const double vx = u[2] / r, vy = u[3] / r;
  return (g - 1.0) * (u[1] - 0.5 * r * (vx * vx + vy * vy));
}

__device__ __forceinline__ double wavespeed_slr(const double* u, double pstar, double a, double q,
                                                double g) {
  const double p = pressure2(u, g);
  const double vel = u[2] / u[0];
  if (pstar <= p) return vel + a;
  return vel + a * sqrt(1.0 + q * (pstar / p - 1.0));
}

// Hllc::solve_star_conservative_left (flux_method/flux_hllc.hpp:330-361) with
// two equations of state, normal direction x.  Sound speeds take each side's
// p_inf (stiff_fluid.hpp:92-96; 0 for the ideal gas: p + 0 = p).
__device__ void star_left(const double* ul, const double* ur, double gl, double gr, double il,
                          double ir, double* out) {
  const double pl = pressure2(ul, gl), pr = pressure2(ur, gr);
  const double al = sqrt(gl * (pl + il) / ul[0]), ar = sqrt(gr * (pr + ir) / ur[0]);
  const double vl = ul[2] / ul[0], vr = ur[2] / ur[0];
  const double p_pvrs = 0.5 * ((pl + pr) - (0.25 * (vr - vl) * (ur[0] + ul[0]) * (al + ar)));
  const double p_star = dmaxr(0.0, p_pvrs);
  const double ql = (gl + 1.0) / (2.0 * gl), qr = (gr + 1.0) / (2.0 * gr);
  const double wsl = wavespeed_slr(ul, p_star, -al, ql, gl);
  const double wsr = wavespeed_slr(ur, p_star, ar, qr, gr);
  const double fl = ul[0] * (wsl - vl), fr = ur[0] * (wsr - vr);
  const double s_star = (pr - pl + vl * fl - vr * fr) / (fl - fr);
  const double sf = wsl - vl;
  const double scale = sf / (wsl - s_star);
#pragma unroll
  for (int c = 0; c < 4; ++c) out[c] = scale * ul[c];
  out[2] = s_star * ul[0] * scale;
  out[1] = scale * (ul[1] + ul[0] * (s_star - vl) * (s_star + pl / (ul[0] * sf)));
}

// Probe of the state around (x, y) with offsets w in cells, with the
// arithmetic of the reference's 2-D math::interp (math/interp.hpp:120-167)
// as it computes: X0, X1 the cells offset by off_x and off_x + sign along x
// from the source, Y0, Y1 those offset along y; close = X0(1-fx) + X1 fx,
// far = Y0(1-fx) + Y1 fx, r = close(1-fy) + far fy.  (The function's comment
// documents a bilinear form over the four cells of the offset square, which
// its code does not compute.)
template <typename T>
__device__ void interp2(const T* u, int64_t pitch, int64_t nx, int64_t ny, int64_t x, int64_t y,
                        const double* w, double* out) {
  int64_t off[2];
  int sg[2];
  double f[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    sg[d] = isgn(w[d]);
    const double aw = fabs(w[d]);
    const double ao = floor(aw);
    off[d] = (int64_t)((double)sg[d] * ao);
    f[d] = aw - ao;
  }
  double X0[4], X1[4], Y0[4], Y1[4];
  load4(u, pitch, midx(nx, ny, x + off[0], y), X0);
  load4(u, pitch, midx(nx, ny, x + off[0] + sg[0], y), X1);
  load4(u, pitch, midx(nx, ny, x, y + off[1]), Y0);
  load4(u, pitch, midx(nx, ny, x, y + off[1] + sg[1]), Y1);
  const double factor = 1.0 - f[0];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double close = X0[c] * factor + X1[c] * f[0];
    const double far = Y0[c] * factor + Y1[c] * f[0];
    out[c] = close * (1.0 - f[1]) + far * f[1];
  }
}

// GFM source test (ghost_fluid/riemann_ghost_fluid.hpp:59-71,204-231) and
// the unit normal grad(phi)/|grad(phi)| (iterator/multidim_iterator.hpp
// :291-306 with dh = 1).
__device__ bool gfm_source(const double* pa, const double* pb, int64_t nx, int64_t ny, int64_t x,
                           int64_t y, double h, double* n) {
  const double phi = pa[y * nx + x];
  if (!((phi <= 0.0 || phi <= -0.0) && phi >= -h)) return false;
  const double xm = pa[midx(nx, ny, x - 1, y)], xp = pa[midx(nx, ny, x + 1, y)];
  const double ym = pa[midx(nx, ny, x, y - 1)], yp = pa[midx(nx, ny, x, y + 1)];
  if (xm == 0.0 || xp == 0.0 || ym == 0.0 || yp == 0.0) return false;
  const double ob = pb[y * nx + x];
  if (!((ob > 0.0 && ob < fabs(h)) || ob == 0.0)) return false;
  const double g0 = 0.5 * (xp - xm), g1 = 0.5 * (yp - ym);
  const double s = sqrt(g0 * g0 + g1 * g1);
  if (!(s > 0.0)) return false;
  n[0] = g0 / s;
  n[1] = g1 / s;
  return true;
}

// star state of a source (riemann_ghost_fluid.hpp:70-176)
template <typename T>
__device__ void gfm_star(const T* ua, const T* ub, int64_t pitch, int64_t nx, int64_t ny,
                         const double* pa, int64_t x, int64_t y, double h, const double* n,
                         double ga, double gb, double ia, double ib, double* star) {
  const double abs_phi = fabs(pa[y * nx + x]);
  const double h32 = 1.5 * h;
  double w[2], wl[4], wr[4];
#pragma unroll
  for (int d = 0; d < 2; ++d) w[d] = n[d] * (abs_phi - h32) / h;
  interp2(ua, pitch, nx, ny, x, y, w, wl);
#pragma unroll
  for (int d = 0; d < 2; ++d) w[d] = n[d] * (abs_phi + h32) / h;
  interp2(ub, pitch, nx, ny, x, y, w, wr);
  const double vl[2] = {wl[2] / wl[0], wl[3] / wl[0]};
  const double vr[2] = {wr[2] / wr[0], wr[3] / wr[0]};
  const double vl_n = vl[0] * n[0] + vl[1] * n[1];
  const double vr_n = vr[0] * n[0] + vr[1] * n[1];
  // set_velocity on a conservative state: m = v * rho, energy untouched
  wl[2] = vl_n * wl[0];
  wr[2] = vr_n * wr[0];
  wl[3] = 0.0 * wl[0];
  wr[3] = 0.0 * wr[0];
  star_left(wl, wr, ga, gb, ia, ib, star);
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const double sv = star[2 + d] / star[0];
    const double v = vl[d] + (sv - vl_n) * n[d];
    star[2 + d] = v * star[0];
  }
}

// band of the extrapolation (ghost_fluid/ghost_fluid_extrapolator.hpp:104-127)
__device__ __forceinline__ bool in_band(double phi, double h) {
  const double upper = (6.0 * h) * 0.70710678118654752440;
  return phi > 0.0 && phi <= upper && phi >= h;
}

// One thread per cell: x from blockIdx.x, rows from blockIdx.y (strided when
// the grid has more rows than a launch's y extent).
template <typename T>
__global__ void __launch_bounds__(256) mm_scan_kernel(MMArgs a) {
  const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.nx) return;
  for (int64_t y = blockIdx.y; y < a.ny; y += gridDim.y) {
    const int64_t t = y * a.nx + x;
#pragma unroll 1
    for (int m = 0; m < 2; ++m) {
      const double* pa = a.phi[m];
      const double* pb = a.phi[1 - m];
      if (in_band(pa[t], a.h)) {
        const int slot = atomicAdd(&a.cnt->band[m], 1);
        a.band_list[m][slot] = (int)t;
      }
      // pull: the last source in raster order whose target is this cell.
      // The 8 neighbours' level-set values are loaded together first; a cell
      // with no neighbour in [-h, 0] (almost every cell) is done after one
      // round trip.
      unsigned cand = 0u;
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        const int dx = 1 - q % 3, dy = 1 - q / 3;
        const int64_t cx = x + dx, cy = y + dy;
        if (q == 4 || cx < 0 || cx >= a.nx || cy < 0 || cy >= a.ny) continue;
        const double ps = pa[cy * a.nx + cx];
        if (ps <= 0.0 && ps >= -a.h) cand |= 1u << q;
      }
      bool found = false;
      double nrm[2] = {0.0, 0.0};
      int64_t sx = 0, sy = 0;
      for (int dy = 1; dy >= -1 && !found && cand; --dy) {
        for (int dx = 1; dx >= -1 && !found; --dx) {
          if (dx == 0 && dy == 0) continue;
          const int64_t cx = x + dx, cy = y + dy;
          if (!(cand & (1u << ((1 - dy) * 3 + (1 - dx))))) continue;
          double nn[2];
          if (!gfm_source(pa, pb, a.nx, a.ny, cx, cy, a.h, nn)) continue;
          if (cx + isgn(nn[0]) != x || cy + isgn(nn[1]) != y) continue;
          found = true;
          nrm[0] = nn[0];
          nrm[1] = nn[1];
          sx = cx;
          sy = cy;
        }
      }
      if (!found) continue;
      double star[4];
      gfm_star(static_cast<const T*>(a.u[m]), static_cast<const T*>(a.u[1 - m]), a.pitch, a.nx,
               a.ny, pa, sx, sy, a.h, nrm, a.gamma[m], a.gamma[1 - m], a.pinf[m], a.pinf[1 - m],
               star);
      const int slot = atomicAdd(&a.cnt->gfm[m], 1);
      a.gfm_idx[m][slot] = (int)t;
#pragma unroll
      for (int c = 0; c < 4; ++c) a.gfm_state[m][4 * (int64_t)slot + c] = star[c];
    }
  }
}

template <typename T>
__global__ void mm_scatter_kernel(MMArgs a) {
  for (int m = 0; m < 2; ++m) {
    const int cnt = a.cnt->gfm[m];
    T* u = static_cast<T*>(a.w[m]);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
      const int64_t t = a.gfm_idx[m][k];
#pragma unroll
      for (int c = 0; c < 4; ++c) u[c * a.pitch + t] = (T)a.gfm_state[m][4 * (int64_t)k + c];
    }
  }
}

// Ghost-cell extrapolation (ghost_fluid_extrapolator.hpp:99-196) as Jacobi
// sweeps over the band lists of both materials, one launch per sweep, one
// thread per band cell.  Sweep `it` (counted from `base`, the sweeps done
// before this chunk) reads the iterate from U (even) or X (odd) and writes
// the other buffer; neighbours outside the band read U.  The last block to
// finish a sweep closes it: a material whose largest change is below 1e-8
// with no NaN stops (later sweeps skip it), and its sweep count is recorded.
// mm_extrap_finish_kernel then moves a final iterate left in X back to U.
template <typename T>
__global__ void __launch_bounds__(256) mm_extrap_sweep_kernel(MMArgs a, int it, int base) {
  MMCounters* c = a.cnt;
  const int n0 = c->band[0], n1 = c->band[1];
  const int par = (it - base) & 1;
  const int64_t nx = a.nx, ny = a.ny, pitch = a.pitch;
  const double h = a.h;
  double worst[2] = {0.0, 0.0};
  int nan_seen[2] = {0, 0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n0 + n1; k += gridDim.x * blockDim.x) {
    const int m = k < n0 ? 0 : 1;
    if (*(volatile int*)&c->stop[m]) continue;
    const int64_t i = a.band_list[m][m == 0 ? k : k - n0];
    const double* phi = a.phi[m];
    T* U = static_cast<T*>(a.w[m]);
    T* X = static_cast<T*>(a.x[m]);
    const T* src = par ? X : U;
    T* dst = par ? U : X;
    const int64_t x = i % nx, y = i / nx;
    const double fact = 0.5 / h;
    double g[2];
    g[0] = fact * (phi[midx(nx, ny, x + 1, y)] - phi[midx(nx, ny, x - 1, y)]);
    g[1] = fact * (phi[midx(nx, ny, x, y + 1)] - phi[midx(nx, ny, x, y - 1)]);
    const double sq = sqrt(g[0] * g[0] + g[1] * g[1]);
    const double sign = (double)isgn(phi[i]);
    double nrm[2], l1 = 0.0;
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      nrm[d] = -sign * (g[d] / sq);
      l1 += fabs(nrm[d]);
    }
    const bool use_n = l1 > 1e-2;
    double pv[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const int64_t qm = d == 0 ? midx(nx, ny, x - 1, y) : midx(nx, ny, x, y - 1);
      const int64_t qp = d == 0 ? midx(nx, ny, x + 1, y) : midx(nx, ny, x, y + 1);
      const int64_t q = phi[qm] < phi[qp] ? qm : qp;
      const T* from = in_band(phi[q], h) ? src : U;
      const double wgt = use_n ? fabs(nrm[d]) : 0.5;
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) pv[cc] += (double)from[cc * pitch + q] * wgt;
    }
    if (use_n) {
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) pv[cc] = pv[cc] / l1;
    }
    bool has_nan = false;
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) has_nan |= isnan(pv[cc]);
    double err = 0.0;
    if (has_nan) {
      nan_seen[m] = 1;
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) dst[cc * pitch + i] = src[cc * pitch + i];
    } else {
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const T v = (T)pv[cc];
        err += fabs((double)v - (double)src[cc * pitch + i]);
        dst[cc * pitch + i] = v;
      }
    }
    worst[m] = (err > worst[m]) ? err : worst[m];
  }
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    if (worst[m] > 0.0)
      atomicMax(&c->err[m][par], (unsigned long long)__double_as_longlong(worst[m]));
    if (nan_seen[m]) atomicOr(&c->nan[m][par], 1);
  }
  __threadfence();   // this thread's writes and atomics, before the block arrives
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(&c->arrive, 1u);
    if (prev == gridDim.x - 1) {
      __threadfence();
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        volatile MMCounters* vc = c;
        if (vc->stop[m]) continue;
        const double mx = __longlong_as_double((long long)vc->err[m][par]);
        vc->iters[m] = it + 1;
        if (!(mx >= 1e-8) && !vc->nan[m][par]) vc->stop[m] = 1;
        vc->err[m][1 - par] = 0ull;
        vc->nan[m][1 - par] = 0;
      }
      c->arrive = 0u;
    }
  }
}

// After a chunk of sweeps: a material whose last iterate is in X (an odd
// number of sweeps in the chunk since U held the iterate) gets its band
// cells copied back to U.
template <typename T>
__global__ void __launch_bounds__(256) mm_extrap_finish_kernel(MMArgs a, int base) {
  MMCounters* c = a.cnt;
  const int n0 = c->band[0], n1 = c->band[1];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n0 + n1; k += gridDim.x * blockDim.x) {
    const int m = k < n0 ? 0 : 1;
    if (((c->iters[m] - base) & 1) == 0 || c->iters[m] <= base) continue;
    const int64_t i = a.band_list[m][m == 0 ? k : k - n0];
    T* U = static_cast<T*>(a.w[m]);
    const T* X = static_cast<const T*>(a.x[m]);
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) U[cc * a.pitch + i] = X[cc * a.pitch + i];
  }
}

__global__ void negate_kernel(int64_t n, const double* __restrict__ src, double* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = -src[i];
}

template <typename T>
__global__ void set_states_kernel(T* u, int64_t pitch, int64_t n, const double* phi, T c0, T c1,
                                  T c2, T c3) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!(phi[i] <= 0.0 || phi[i] <= -0.0)) continue;
    u[i] = c0;
    u[pitch + i] = c1;
    u[2 * pitch + i] = c2;
    u[3 * pitch + i] = c3;
  }
}

template <typename T>
__global__ void combine_kernel(T* u0, const T* u1, int64_t pitch, int64_t n, const double* phi1) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!(phi1[i] <= 0.0 || phi1[i] <= -0.0)) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) u0[c * pitch + i] = u1[c * pitch + i];
  }
}

unsigned grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (unsigned)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

int check_mm_grid(const fl_grid* g) {
  if (g == nullptr) return set_error(kEInval, "grid is NULL");
  if (g->dims != 2) return set_error(kEInval, "the multimaterial path is 2-D");
  if (g->n[0] < 4 || g->n[1] < 4 || g->n[2] != 1)
    return set_error(kEInval, "grid needs n[0], n[1] >= 4 and n[2] = 1");
  if (g->n[0] * g->n[1] > (int64_t)0x7fffffff) return set_error(kEInval, "grid too large");
  if (g->pitch < g->n[0] * g->n[1]) return set_error(kEInval, "pitch below the cell count");
  return kOk;
}

}  // namespace
}  // namespace fl

using namespace fl;

struct fl_mm {
  fl_grid grid;
  // strip counters of the split sweeps, a pair per material (4, device)
  unsigned int* walk_next = nullptr;
  int64_t walk_launches = 0;          // sweeps launched per material: the parity slot
  bool counters_dirty = false;        // a counted sweep failed: re-zero them first
  // material 1's split step runs on a stream of its own, beside material 0's
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  uint32_t policy;
  bool f32;
  double gamma[2];
  double pinf[2];   // stiffened fluids' p_inf (0: ideal gas)
  double h;
  // owned device workspace
  MMCounters* cnt;
  int* band_list[2];
  int* gfm_idx[2];
  double* gfm_state[2];
  double* vel;
  double* ws_dev;   // 2 doubles
  void* ls_ws;
  // loop state (caller buffers)
  void* u[2][2];       // [material][buffer]; the state is in buffer 0 between steps
  double* phi[2][2];   // [material][buffer]
  int phi_cur[2];
  double cfl, sim_time;
  int64_t max_iters, iters;
  double run_time;
  int reinit_every;
  int done, status;
  int extrap_iters;
  int stats[8];
  MMArgs ghost_args;   // the last ghost pass, for its extrapolation's continuation
  int ex_launched;     // extrapolation sweeps launched in the last ghost pass
  int ex_max;          // its sweep limit
};

namespace {

void free_mm(fl_mm* m) {
  if (!m) return;
  cudaFree(m->cnt);
  cudaFree(m->walk_next);
  if (m->fork) cudaEventDestroy(m->fork);
  if (m->join) cudaEventDestroy(m->join);
  if (m->side) cudaStreamDestroy(m->side);
  for (int k = 0; k < 2; ++k) {
    cudaFree(m->band_list[k]);
    cudaFree(m->gfm_idx[k]);
    cudaFree(m->gfm_state[k]);
  }
  cudaFree(m->vel);
  cudaFree(m->ws_dev);
  cudaFree(m->ls_ws);
  delete m;
}

int cuda_err(cudaError_t e, const char* where) {
  return set_error(kECuda, "%s: %s", where, cudaGetErrorString(e));
}

constexpr int kExChunk = 8;   // extrapolation sweeps launched before the host looks

// One chunk of extrapolation sweeps, starting at sweep m->ex_launched with the
// iterate in U, then the copy-back of iterates left in X.
cudaError_t extrap_chunk(fl_mm* m, cudaStream_t st) {
  const MMArgs& a = m->ghost_args;
  const int base = m->ex_launched;
  const int end = base + kExChunk < m->ex_max ? base + kExChunk : m->ex_max;
  const unsigned blocks = 148 * 2;
  for (int it = base; it < end; ++it) {
    if (m->f32) mm_extrap_sweep_kernel<float><<<blocks, 256, 0, st>>>(a, it, base);
    else mm_extrap_sweep_kernel<double><<<blocks, 256, 0, st>>>(a, it, base);
  }
  if (m->f32) mm_extrap_finish_kernel<float><<<blocks, 256, 0, st>>>(a, base);
  else mm_extrap_finish_kernel<double><<<blocks, 256, 0, st>>>(a, base);
  m->ex_launched = end;
  return cudaGetLastError();
}

// Whether the last ghost pass's extrapolation still has sweeps to run
// (reads the counters; the caller has synchronised the stream).
bool extrap_unfinished(const fl_mm* m, const MMCounters& c) {
  return m->ex_launched < m->ex_max && (!c.stop[0] || !c.stop[1]);
}

// Runs the remaining chunks of the last ghost pass's extrapolation, waiting
// for the stream after each.
int extrap_complete(fl_mm* m, cudaStream_t st) {
  for (;;) {
    MMCounters c;
    cudaError_t e = cudaMemcpyAsync(&c, m->cnt, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(e, "fl_mm extrapolation");
    if (!extrap_unfinished(m, c)) return kOk;
    if ((e = extrap_chunk(m, st)) != cudaSuccess) return cuda_err(e, "fl_mm extrapolation");
  }
}

// GFM + the first chunk of the extrapolation on states u[m] with second
// buffers x[m].
int ghost_pass(fl_mm* m, void* const* u, void* const* x, const double* const* phi, int max_iters,
               cudaStream_t st) {
  MMArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = m->grid.n[0];
  a.ny = m->grid.n[1];
  a.pitch = m->grid.pitch;
  a.h = m->h;
  for (int k = 0; k < 2; ++k) {
    a.gamma[k] = m->gamma[k];
    a.pinf[k] = m->pinf[k];
    a.u[k] = u[k];
    a.w[k] = u[k];
    a.x[k] = x[k];
    a.phi[k] = phi[k];
    a.band_list[k] = m->band_list[k];
    a.gfm_idx[k] = m->gfm_idx[k];
    a.gfm_state[k] = m->gfm_state[k];
  }
  a.cnt = m->cnt;
  a.max_iters = max_iters;
  cudaError_t e = cudaMemsetAsync(m->cnt, 0, sizeof(MMCounters), st);
  if (e != cudaSuccess) return cuda_err(e, "fl_mm ghost");
  const dim3 scan_grid((unsigned)((a.nx + 255) / 256), (unsigned)(a.ny < 65535 ? a.ny : 65535));
  if (m->f32) {
    mm_scan_kernel<float><<<scan_grid, 256, 0, st>>>(a);
    mm_scatter_kernel<float><<<148, 256, 0, st>>>(a);
  } else {
    mm_scan_kernel<double><<<scan_grid, 256, 0, st>>>(a);
    mm_scatter_kernel<double><<<148, 256, 0, st>>>(a);
  }
  m->ghost_args = a;
  m->ex_launched = 0;
  m->ex_max = max_iters;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = extrap_chunk(m, st);
  if (e != cudaSuccess) return cuda_err(e, "fl_mm ghost");
  return kOk;
}

}  // namespace

extern "C" {

int fl_mm_create(fl_mm** out, const fl_grid* grid, const double* gammas, uint32_t policy,
                 double res) {
  if (out == nullptr) return set_error(kEInval, "out is NULL");
  *out = nullptr;
  int rc = check_mm_grid(grid);
  if (rc) return rc;
  if (gammas == nullptr || !(gammas[0] > 1.0) || !(gammas[1] > 1.0))
    return set_error(kEInval, "both gammas must exceed 1");
  if (!(res > 0.0)) return set_error(kEInval, "res must be positive");
  fl_mm* m = new (std::nothrow) fl_mm;
  if (m == nullptr) return set_error(kENoMem, "out of host memory");
  memset(m, 0, sizeof(*m));
  m->grid = *grid;
  m->policy = policy;
  m->f32 = (policy & 1u) != 0;
  m->gamma[0] = gammas[0];
  m->gamma[1] = gammas[1];
  m->h = res;
  m->reinit_every = 1;
  const int64_t n = grid->n[0] * grid->n[1];
  const int64_t lsb = fl_ls_workspace_bytes(grid);
  cudaError_t e = cudaMalloc(&m->cnt, sizeof(MMCounters));
  if (e == cudaSuccess) e = cudaMalloc(&m->walk_next, 4 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(m->walk_next, 0, 4 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->join, cudaEventDisableTiming);
  for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
    e = cudaMalloc(&m->band_list[k], n * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&m->gfm_idx[k], n * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&m->gfm_state[k], n * 4 * sizeof(double));
  }
  if (e == cudaSuccess) e = cudaMalloc(&m->vel, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&m->ws_dev, 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&m->ls_ws, (size_t)lsb);
  if (e != cudaSuccess) {
    free_mm(m);
    return set_error(kENoMem, "fl_mm_create: %s", cudaGetErrorString(e));
  }
  *out = m;
  return kOk;
}

int fl_mm_destroy(fl_mm* m) {
  free_mm(m);
  return kOk;
}

int fl_mm_ghost(fl_mm* m, void* u0, void* u1, void* scratch0, void* scratch1, const double* phi0,
                const double* phi1, int max_iters, void* stream) {
  if (m == nullptr) return set_error(kEInval, "mm is NULL");
  if (!u0 || !u1 || !scratch0 || !scratch1 || !phi0 || !phi1)
    return set_error(kEInval, "NULL pointer");
  if (max_iters <= 0) return set_error(kEInval, "max_iters must be positive");
  void* u[2] = {u0, u1};
  void* x[2] = {scratch0, scratch1};
  const double* p[2] = {phi0, phi1};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int rc = ghost_pass(m, u, x, p, max_iters, st);
  return rc ? rc : extrap_complete(m, st);
}

int fl_mm_stats(const fl_mm* m, int32_t* out, int32_t n) {
  if (m == nullptr || out == nullptr || n < 8) return set_error(kEInval, "bad arguments");
  MMCounters c;
  cudaError_t e = cudaMemcpy(&c, m->cnt, sizeof(c), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_err(e, "fl_mm_stats");
  out[0] = c.gfm[0];
  out[1] = c.gfm[1];
  out[2] = c.band[0];
  out[3] = c.band[1];
  out[4] = c.iters[0];
  out[5] = c.iters[1];
  out[6] = m->stats[6];
  out[7] = m->stats[7];
  return kOk;
}

int fl_mm_set_states_mat(const fl_grid* grid, uint32_t policy, void* state, const double* phi,
                         const double* prim, const fl_material* mat, void* stream) {
  int rc = check_mm_grid(grid);
  if (rc) return rc;
  if (!state || !phi || !prim || !mat) return set_error(kEInval, "NULL pointer");
  const double gamma = mat->gamma, pinf = mat->p_inf;
  if (!(gamma > 1.0)) return set_error(kEInval, "gamma must exceed 1");
  if (!(pinf >= 0.0) || pinf > DBL_MAX) return set_error(kEInval, "p_inf must be finite and >= 0");
  const int64_t n = grid->n[0] * grid->n[1];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // prim -> cons in the state's precision (state/state_impl.hpp:390-406)
  if (policy & 1u) {
    const float r = (float)prim[0], p = (float)prim[1], vx = (float)prim[2], vy = (float)prim[3];
    const float g = (float)gamma, pi = (float)pinf;
    float v2 = 0.0f;
    v2 += vx * vx;
    v2 += vy * vy;
    // e from the eos (ideal_gas.hpp:59-63; stiff_fluid.hpp:76-80)
    const float e = (p + g * pi) / ((g - 1.0f) * r);
    set_states_kernel<float><<<grid_for(n), 256, 0, st>>>(static_cast<float*>(state), grid->pitch,
                                                          n, phi, r, r * (0.5f * v2 + e), vx * r,
                                                          vy * r);
  } else {
    const double r = prim[0], p = prim[1], vx = prim[2], vy = prim[3];
    double v2 = 0.0;
    v2 += vx * vx;
    v2 += vy * vy;
    const double e = (p + gamma * pinf) / ((gamma - 1.0) * r);
    set_states_kernel<double><<<grid_for(n), 256, 0, st>>>(static_cast<double*>(state),
                                                           grid->pitch, n, phi, r,
                                                           r * (0.5 * v2 + e), vx * r, vy * r);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "fl_mm_set_states");
  return kOk;
}

int fl_mm_set_states(const fl_grid* grid, uint32_t policy, void* state, const double* phi,
                     const double* prim, double gamma, void* stream) {
  const fl_material mat{gamma, 0.0};
  return fl_mm_set_states_mat(grid, policy, state, phi, prim, &mat, stream);
}

int fl_mm_set_materials(fl_mm* m, const fl_material* mats) {
  if (m == nullptr || mats == nullptr) return set_error(kEInval, "NULL pointer");
  for (int k = 0; k < 2; ++k) {
    if (!(mats[k].gamma > 1.0)) return set_error(kEInval, "gamma of material %d must exceed 1", k);
    if (!(mats[k].p_inf >= 0.0) || mats[k].p_inf > DBL_MAX)
      return set_error(kEInval, "p_inf of material %d must be finite and >= 0", k);
  }
  for (int k = 0; k < 2; ++k) {
    m->gamma[k] = mats[k].gamma;
    m->pinf[k] = mats[k].p_inf;
  }
  return kOk;
}

int fl_mm_combine(const fl_grid* grid, uint32_t policy, void* u0, const void* u1,
                  const double* phi1, void* stream) {
  int rc = check_mm_grid(grid);
  if (rc) return rc;
  if (!u0 || !u1 || !phi1) return set_error(kEInval, "NULL pointer");
  const int64_t n = grid->n[0] * grid->n[1];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (policy & 1u)
    combine_kernel<float><<<grid_for(n), 256, 0, st>>>(static_cast<float*>(u0),
                                                       static_cast<const float*>(u1), grid->pitch,
                                                       n, phi1);
  else
    combine_kernel<double><<<grid_for(n), 256, 0, st>>>(static_cast<double*>(u0),
                                                        static_cast<const double*>(u1),
                                                        grid->pitch, n, phi1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "fl_mm_combine");
  return kOk;
}

int fl_mm_begin(fl_mm* m, void* u0a, void* u0b, void* u1a, void* u1b, double* phi0a,
                double* phi0b, double* phi1a, double* phi1b, double cfl, double sim_time,
                int64_t max_iters, int reinit_every) {
  if (m == nullptr) return set_error(kEInval, "mm is NULL");
  if (!u0a || !u0b || !u1a || !u1b || !phi0a || !phi0b || !phi1a || !phi1b)
    return set_error(kEInval, "NULL buffer");
  if (!(cfl > 0.0) || max_iters < 0 || reinit_every < 0)
    return set_error(kEInval, "cfl must be positive, max_iters and reinit_every >= 0");
  m->u[0][0] = u0a;
  m->u[0][1] = u0b;
  m->u[1][0] = u1a;
  m->u[1][1] = u1b;
  m->phi[0][0] = phi0a;
  m->phi[0][1] = phi0b;
  m->phi[1][0] = phi1a;
  m->phi[1][1] = phi1b;
  m->phi_cur[0] = m->phi_cur[1] = 0;
  m->cfl = cfl;
  m->sim_time = sim_time;
  m->max_iters = max_iters;
  m->iters = 0;
  m->run_time = 0.0;
  m->reinit_every = reinit_every;
  m->done = (0.0 < sim_time && 0 < max_iters) ? 0 : 1;
  m->status = kOk;
  m->extrap_iters = 64;
  return kOk;
}

int fl_mm_steps(fl_mm* m, int64_t nsteps, void* stream) {
  if (m == nullptr || m->u[0][0] == nullptr) return set_error(kEInval, "fl_mm_begin not called");
  if (nsteps < 0) return set_error(kEInval, "nsteps < 0");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const fl_grid* g = &m->grid;
  const int64_t n = g->n[0] * g->n[1];
  for (int64_t k = 0; k < nsteps && !m->done; ++k) {
    // 1-2: ghost cells (the second state buffers are free until the sweeps)
    void* u[2] = {m->u[0][0], m->u[1][0]};
    void* x[2] = {m->u[0][1], m->u[1][1]};
    const double* p[2] = {m->phi[0][m->phi_cur[0]], m->phi[1][m->phi_cur[1]]};
    int rc = ghost_pass(m, u, x, p, m->extrap_iters, st);
    if (rc) return rc;
    // 3: time step over both materials (multimaterial_simulator.hpp:384-404).
    // The host reads the wavespeeds and, with them, whether the ghost pass's
    // extrapolation converged within its first chunk of sweeps; if not, the
    // remaining sweeps run and the wavespeeds are taken again.
    double ws[2];
    cudaError_t e = cudaSuccess;
    for (;;) {
      for (int mat = 0; mat < 2; ++mat) {
        const fl_material mm{m->gamma[mat], m->pinf[mat]};
        rc = fl_max_wavespeed_mat(g, u[mat], &mm, m->policy, m->ws_dev + mat, stream);
        if (rc) return rc;
      }
      MMCounters cnt;
      e = cudaMemcpyAsync(ws, m->ws_dev, sizeof(ws), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(&cnt, m->cnt, sizeof(cnt), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return cuda_err(e, "fl_mm_steps");
      if (!extrap_unfinished(m, cnt)) break;
      if ((rc = extrap_complete(m, st))) return rc;
    }
    const double w = (ws[0] < ws[1]) ? ws[1] : ws[0];
    if (!(w > 0.0) || !(w <= DBL_MAX)) {
      m->done = 1;
      m->status = kENan;
      return set_error(kENan, "non-finite wavespeed after step %lld", (long long)m->iters);
    }
    const double dt = m->cfl * m->h / w;
    const double dtdh = dt / m->h;
    // 4: each material's split step with its own gamma; state returns to buffer 0
    // split_solver.cuh:67-79 per material: sweep x into the second buffer,
    // y back into the first, with strip counters of their own.  The two
    // materials' steps are independent: material 1's runs on the side
    // stream while material 0's runs on the loop's, which fills the GPU
    // better than one 2.1M-cell sweep at a time.
    if (m->counters_dirty) {
      const cudaError_t ce = cudaMemsetAsync(m->walk_next, 0, 4 * sizeof(unsigned int), st);
      if (ce != cudaSuccess) return cuda_err(ce, "fl_mm_steps");
      m->counters_dirty = false;
    }
    {
      cudaError_t ce = cudaEventRecord(m->fork, st);
      if (ce == cudaSuccess) ce = cudaStreamWaitEvent(m->side, m->fork, 0);
      if (ce != cudaSuccess) return cuda_err(ce, "fl_mm_steps");
    }
    for (int d = 0; d < 2 && rc == 0; ++d) {
      const int slot = (int)(m->walk_launches & 1);
      for (int mat = 0; mat < 2 && rc == 0; ++mat) {
        const fl_material mm{m->gamma[mat], m->pinf[mat]};
        rc = split_sweep_counted(g, d, m->u[mat][d], m->u[mat][1 - d], &mm, dtdh, m->policy, 0u,
                                 nullptr, m->walk_next + 2 * mat, slot,
                                 mat == 0 ? stream : static_cast<void*>(m->side));
      }
      m->walk_launches += 1;
    }
    {
      cudaError_t ce = cudaEventRecord(m->join, m->side);
      if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, m->join, 0);
      if (ce != cudaSuccess && rc == 0) rc = cuda_err(ce, "fl_mm_steps");
    }
    if (rc) {
      m->counters_dirty = true;
      return rc;
    }
    // 5: level sets (multimaterial_simulator.hpp:428-477)
    const double* phis[2] = {m->phi[0][m->phi_cur[0]], m->phi[1][m->phi_cur[1]]};
    const void* sts[2] = {m->u[0][0], m->u[1][0]};
    rc = fl_ls_velocity(g, 2, phis, sts, g->pitch, m->policy, m->h, m->vel, stream);
    if (rc) return rc;
    for (int mat = 0; mat < 2; ++mat) {
      const int c = m->phi_cur[mat];
      rc = fl_ls_advect(g, m->phi[mat][c], m->vel, dt, m->h, m->phi[mat][1 - c], m->ls_ws, stream);
      if (rc) return rc;
      m->phi_cur[mat] = 1 - c;
    }
    rc = fl_ls_project(n, m->phi[0][m->phi_cur[0]], m->phi[1][m->phi_cur[1]], stream);
    if (rc) return rc;
    const bool reinit = m->reinit_every > 0 && ((m->iters + 1) % m->reinit_every) == 0;
    if (reinit) {
      // The projection has just set phi1 = -phi0 exactly, and the
      // reinitialisation is odd bit for bit (sources keep |phi|, the passes
      // see only distances, the sign is applied last): reinit(phi1) is the
      // negation of reinit(phi0), so material 1 takes that instead of a
      // second run.
      const int c0 = m->phi_cur[0], c1 = m->phi_cur[1];
      int passes = 0;
      rc = fl_ls_reinit(g, m->phi[0][c0], m->h, m->phi[0][1 - c0], m->ls_ws, 1 << 20, &passes,
                        stream);
      if (rc) return rc;
      negate_kernel<<<grid_for(n), 256, 0, st>>>(n, m->phi[0][1 - c0], m->phi[1][1 - c1]);
      cudaError_t ne = cudaGetLastError();
      if (ne != cudaSuccess) return cuda_err(ne, "fl_mm_steps");
      m->stats[6] = m->stats[7] = passes;
      m->phi_cur[0] = 1 - c0;
      m->phi_cur[1] = 1 - c1;
    }
    // 6: time bookkeeping (sim/parameters.hpp:60-77)
    m->run_time += dt;
    m->iters += 1;
    if (!(m->run_time < m->sim_time && m->iters < m->max_iters)) m->done = 1;
  }
  return kOk;
}

int fl_mm_status(fl_mm* m, void* stream, int64_t* iters, double* run_time, int* done,
                 double** phi0, double** phi1) {
  if (m == nullptr) return set_error(kEInval, "mm is NULL");
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_err(e, "fl_mm_status");
  if (iters) *iters = m->iters;
  if (run_time) *run_time = m->run_time;
  if (done) *done = m->done;
  if (phi0) *phi0 = m->phi[0][m->phi_cur[0]];
  if (phi1) *phi1 = m->phi[1][m->phi_cur[1]];
  return m->status;
}

}  // extern "C"
