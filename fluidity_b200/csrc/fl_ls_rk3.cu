// fl_ls_rk3.cu -- the three TVD-RK3 stages of fl_ls_advect: phi_t + v |grad phi| = 0
// with WENO-HJ5 one-sided derivatives (scheme/stencils/weno_hj_5.hpp:85-144),
// the Godunov upwind Hamiltonian (scheme/schemes/godunov_upwind.hpp:94-166,
// scheme/evaluators/levelset_hamiltonian.hpp:63-98) and the RK3 combination
// (scheme/updaters/runge_kutta_3.hpp:110-148).
//
// This file is compiled with FMA contraction and evaluates the WENO weights
// in a rearranged form, so its results agree with the reference's operation
// order to rounding (a few ulp of the derivative), not bit for bit:
//
//  * a window of five differences d1..d5 = D(j-2..j+2), D(k) = (phi(k+1) -
//    phi(k)) / h, gives two one-sided derivatives: read forward it is the
//    backward derivative of cell j+1, read in reverse the forward derivative
//    of cell j.  The two readings share the epsilon and their smoothness
//    indicators (beta_1 and beta_3 trade places), so each window is evaluated
//    once and the backward value is handed to the next cell through shared
//    memory;
//  * the weights alpha_k = c_k / (beta_k + eps)^2 are normalised by one
//    product instead of three divisions: with s_k = (beta_k + eps) 2^-E,
//    2^E the power of two at or below eps (an exact scaling that keeps
//    s_k in [1, 7e6] whatever the magnitude of the differences), the
//    weights are proportional to c_1 s_2^2 s_3^2, c_2 s_1^2 s_3^2 and
//    c_3 s_1^2 s_2^2, and one reciprocal per reading divides them out;
//  * reciprocals start from rcp.approx.ftz.f64 and take one third-order
//    step (y += y (e + e^2), e = 1 - x y), correct to about an ulp.
#include <cuda_runtime.h>

#include <cstdint>

#include "fl_internal.cuh"

namespace fl {
namespace {

constexpr int LX = 32, LY = 8, LH = 3;
constexpr int SX = LX + 2 * LH, SY = LY + 2 * LH;

__device__ __forceinline__ int64_t lmir(int64_t i, int64_t n) {
  if (i < 0) i = -1 - i;
  else if (i >= n) i = 2 * n - 1 - i;
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

__device__ __forceinline__ double dmax_(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }

__device__ __forceinline__ double rcp_f64(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
}

// 2^-E for the power of two 2^E at or below e > 0 (a normal number): built
// from e's exponent field, so multiplying by it is exact.
__device__ __forceinline__ double pow2_below_inv(double e) {
  const int biased = (__double2hiint(e) >> 20) & 0x7ff;
  int k = 2046 - biased;            // biased exponent of 2^-(biased - 1023)
  k = k < 1 ? 1 : (k > 2046 ? 2046 : k);
  return __hiloint2double(k << 20, 0);
}

// Both readings of one window.  fwd: weno_hj_5 of (d1, d2, d3, d4, d5);
// rev: of (d5, d4, d3, d2, d1).  With kFwdOnly the reverse reading is skipped.
template <bool kFwdOnly>
__device__ __forceinline__ void weno_window(double d1, double d2, double d3, double d4, double d5,
                                            double& fwd, double& rev) {
  const double f1 = 13.0 / 12.0, f2 = 1.0 / 4.0;
  const double t1 = d1 - 2.0 * d2 + d3, t2 = d1 - 4.0 * d2 + 3.0 * d3;
  const double t3 = d2 - 2.0 * d3 + d4, t4 = d2 - d4;
  const double t5 = d3 - 2.0 * d4 + d5, t6 = 3.0 * d3 - 4.0 * d4 + d5;
  const double b1 = f1 * (t1 * t1) + f2 * (t2 * t2);
  const double b2 = f1 * (t3 * t3) + f2 * (t4 * t4);
  const double b3 = f1 * (t5 * t5) + f2 * (t6 * t6);
  const double eps =
      10.0e-6 * dmax_(dmax_(dmax_(dmax_(d1 * d1, d2 * d2), d3 * d3), d4 * d4), d5 * d5) + 10.0e-99;
  const double sc = pow2_below_inv(eps);
  const double s1 = (b1 + eps) * sc, s2 = (b2 + eps) * sc, s3 = (b3 + eps) * sc;
  const double q1 = s1 * s1, q2 = s2 * s2, q3 = s3 * s3;
  const double p23 = q2 * q3, p13 = q1 * q3, p12 = q1 * q2;
  const double wb = 0.6 * p13;
  {
    const double wa = 0.1 * p23, wc = 0.3 * p12;
    const double c1 = 2.0 * d1 - 7.0 * d2 + 11.0 * d3;
    const double c2 = -d2 + 5.0 * d3 + 2.0 * d4;
    const double c3 = 2.0 * d3 + 5.0 * d4 - d5;
    fwd = (wa * c1 + wb * c2 + wc * c3) * rcp_f64((wa + wb + wc) * 6.0);
  }
  if (!kFwdOnly) {
    const double wa = 0.1 * p12, wc = 0.3 * p23;
    const double c1 = 2.0 * d5 - 7.0 * d4 + 11.0 * d3;
    const double c2 = -d4 + 5.0 * d3 + 2.0 * d2;
    const double c3 = 2.0 * d3 + 5.0 * d2 - d1;
    rev = (wa * c1 + wb * c2 + wc * c3) * rcp_f64((wa + wb + wc) * 6.0);
  }
}

// The window centred on tile position c along a row (kStride 1) or a
// column (kStride = the tile's row length) of the staged tile.
template <bool kFwdOnly, int kStride>
__device__ __forceinline__ void tile_window(const double* c, double h1, double& fwd, double& rev) {
  const double p0 = c[-2 * kStride], p1 = c[-kStride], p2 = c[0], p3 = c[kStride],
               p4 = c[2 * kStride], p5 = c[3 * kStride];
  weno_window<kFwdOnly>(h1 * (p1 - p0), h1 * (p2 - p1), h1 * (p3 - p2), h1 * (p4 - p3),
                        h1 * (p5 - p4), fwd, rev);
}

// One RK3 stage on a 32 x 8 tile staged with a 3-cell halo.
//   stage 1: out = phi_n - dt H(phi_n)
//   stage 2: out = 0.75 phi_n + 0.25 (s - dt H(s))
//   stage 3: out = (1/3) phi_n + (2/3) (s - dt H(s))
// Every thread evaluates the x and the y window centred on its own cell; the
// windows centred one cell before the tile (one per row and one per column)
// are evaluated by the first 40 threads, forward reading only.
#ifndef FL_LS_RK3_CTAS
#define FL_LS_RK3_CTAS 4
#endif
template <int STAGE>
__global__ void __launch_bounds__(LX * LY, FL_LS_RK3_CTAS)
    ls_rk3_kernel(const double* __restrict__ phi_n, const double* __restrict__ s,
                  const double* __restrict__ vel, double dt, double h, int64_t nx, int64_t ny,
                  double* __restrict__ out) {
  constexpr int kRow = SX + 1;
  __shared__ double tile[SY][kRow];
  __shared__ double bkx[LY][LX + 1];  // bkx[r][k]: backward x derivative of tile cell (k, r)
  __shared__ double bky[LY + 1][LX];  // bky[k][c]: backward y derivative of tile cell (c, k)
  const int64_t x0 = (int64_t)blockIdx.x * LX, y0 = (int64_t)blockIdx.y * LY;
  const double* src = (STAGE == 1) ? phi_n : s;
  for (int i = threadIdx.x; i < SX * SY; i += LX * LY) {
    const int lx = i % SX, ly = i / SX;
    tile[ly][lx] = src[lmir(y0 - LH + ly, ny) * nx + lmir(x0 - LH + lx, nx)];
  }
  __syncthreads();
  const int tx = threadIdx.x % LX, ty = threadIdx.x / LX;
  const int cx = tx + LH, cy = ty + LH;
  const double h1 = 1.0 / h;
  double fwx, fwy, bk, unused;
  tile_window<false, 1>(&tile[cy][cx], h1, bk, fwx);
  bkx[ty][tx + 1] = bk;
  tile_window<false, kRow>(&tile[cy][cx], h1, bk, fwy);
  bky[ty + 1][tx] = bk;
  if (threadIdx.x < LX) {  // column tx: the window centred on row y0 - 1
    tile_window<true, kRow>(&tile[LH - 1][cx], h1, bk, unused);
    bky[0][tx] = bk;
  } else if (threadIdx.x < LX + LY) {  // row threadIdx.x - 32: the window centred on x0 - 1
    const int r = threadIdx.x - LX;
    tile_window<true, 1>(&tile[r + LH][LH - 1], h1, bk, unused);
    bkx[r][0] = bk;
  }
  __syncthreads();
  const int64_t x = x0 + tx, y = y0 + ty;
  if (x >= nx || y >= ny) return;
  const int64_t i = y * nx + x;
  const double v = vel[i];
  double r = 0.0;
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const double bkd = d == 0 ? bkx[ty][tx] : bky[ty][tx];
    const double fwd = d == 0 ? fwx : fwy;
    double b, w;
    if (v <= 0.0) {
      b = dmax_(bkd, 0.0);
      w = dmin_(fwd, 0.0);
    } else {
      b = dmin_(bkd, 0.0);
      w = dmax_(fwd, 0.0);
    }
    r += dmax_(b * b, w * w);
  }
  const double H = v * sqrt(r);
  const double cur = tile[cy][cx];
  if (STAGE == 1) {
    out[i] = cur - dt * H;
  } else if (STAGE == 2) {
    out[i] = 0.75 * phi_n[i] + 0.25 * (cur - dt * H);
  } else {
    const double f13 = 1.0 / 3.0, f23 = 2.0 * f13;
    out[i] = (f13 * phi_n[i]) + (f23 * (cur - dt * H));
  }
}

}  // namespace

cudaError_t launch_ls_rk3(const double* phi, const double* vel, double dt, double h, int64_t nx,
                          int64_t ny, double* s1, double* s2, double* out, cudaStream_t st) {
  const dim3 g((unsigned)((nx + LX - 1) / LX), (unsigned)((ny + LY - 1) / LY));
  ls_rk3_kernel<1><<<g, LX * LY, 0, st>>>(phi, nullptr, vel, dt, h, nx, ny, s1);
  ls_rk3_kernel<2><<<g, LX * LY, 0, st>>>(phi, s1, vel, dt, h, nx, ny, s2);
  ls_rk3_kernel<3><<<g, LX * LY, 0, st>>>(phi, s2, vel, dt, h, nx, ny, out);
  return cudaGetLastError();
}

}  // namespace fl
