// Guard band of the sync threshold decisions.
//
// The reference decides in FP64 whether a sync sample lies at or below the
// pulse threshold (src/pipeline/sync_pulses.cu:35-55; the VSYNC widths of
// src/pipeline/vsync_discover.cu:5-45 and the threshold crossings of
// src/pipeline/hsync_refine.cu:21-65 make the same decision).  This decoder
// computes sync in FP32, within a few Hz of FP64.  K1b lists every sync sample
// it writes within kGuardHz of the threshold; guard_kernel re-evaluates each
// listed sample in FP64 straight from the raw capture and writes it back on the
// side of the FP32 threshold its FP64 value lies on, so every later threshold
// decision (edges, VSYNC widths, pulses, hsync crossings) is the FP64 one.
//
// The FP64 value follows the reference's tile arithmetic exactly, with the
// circular kernels truncated only where their taps fall below 1e-13 of the
// peak (Design::ga64 / hs64):
//   sync[s]  = sum_k hs[k] * dem[c(J - k)],   J = 2048 + s - f*spp, s in tile f,
//   dem[c]   = wrap(arg z(J') - arg z(J' - 1)) * fs / 2pi   (c in tile f', J' = 2048 + c - f'*spp),
//   z(j)     = sum_m g[m] * x_f'(j - m),
// where tile positions wrap mod the tile length and chunk positions clamp to
// the demodulated range (src/pipeline/fm_demod.cu:133-169, 396-485).
//
// Work: one flagged sample is split over `parts` CTAs, each CTA evaluating 256
// of the 2*hb + 1 demod samples of the sync window.  Where those positions
// lie inside one tile away from its wrap and the chunk ends (nearly always),
// the CTA stages their raw window once in shared memory as FP64 and computes
// each analytic-signal value once (one FP64 dot product of 2*ha + 1 taps per
// position); elsewhere each thread evaluates its position with the tile wrap
// and chunk clamp (two dot products).  Each CTA writes its
// partial sum; the CTA that finishes a sample last (an atomic count, no
// waiting) adds the partials in part order, so the result is deterministic.
#include <cuda_runtime.h>

#include <algorithm>

#include "chain.cuh"
#include "cuvhs_internal.h"
#include "raw_input.cuh"

namespace cuvhs {
namespace {

constexpr int kGuardThreads = 256;
constexpr double kPi64 = 3.14159265358979323846;
constexpr double kTau64 = 2.0 * kPi64;

__device__ __forceinline__ long long wrap_pos(long long q, long long tile) {
  return q < 0 ? q + tile : (q >= tile ? q - tile : q);
}

// Converted sample at chunk position p (already clamped to the chunk): 0 past
// the samples read, DC removed.
template <int FMT>
__device__ __forceinline__ double raw64(const GuardArgs& g, long long p, double dc) {
  if (p >= g.n_read) return 0.0;
  return (double)raw_convert<FMT>(g.raw, (int)p) - dc;
}

// z(J) of tile f2 at tile positions J for the kGuardThreads demod positions
// of one CTA, when they are consecutive inside one tile and their raw windows
// need no wrap, clamp or zero fill: the raw window is staged once as FP64
// (converted, DC removed) and each analytic-signal value is computed once.
// Returns false (nothing written) when the CTA's positions are not of that
// kind; the caller then evaluates every position on its own.
struct GuardSmem {
  double2* taps;  // [2*ha + 3]
  double* xs;     // [kGuardThreads + 2*ha + 2] staged raw
  double2* z;     // [kGuardThreads + 1]
};

template <int FMT>
__device__ bool stage_interior(const GuardArgs& g, const GuardSmem& sm, long long c_first, int count, double dc) {
  // positions c_first, c_first - 1, ..., c_first - count + 1 and one more for z(J2 - 1)
  const long long c_last = c_first - count;  // the extra position (z only)
  const long long last = g.total - 1;
  if (c_last < 0) return false;
  const long long f2 = c_first / g.spp;
  if (c_last / g.spp != f2 || c_last - f2 * g.spp < 0) return false;
  const long long tile0 = f2 * g.spp - kOverlap;
  const long long J_hi = c_first - tile0, J_lo = c_last - tile0;  // tile positions
  const long long u_lo = J_lo - g.ha, u_hi = J_hi + g.ha;
  if (u_lo < 0 || u_hi >= g.tile || tile0 + u_lo < 0 || tile0 + u_hi > last || tile0 + u_hi >= g.n_read)
    return false;
  const int nx = (int)(u_hi - u_lo + 1);
  for (int i = threadIdx.x; i < nx; i += kGuardThreads)
    sm.xs[i] = (double)raw_convert<FMT>(g.raw, (int)(tile0 + u_lo + i)) - dc;
  __syncthreads();
  // thread t: z at tile position J_hi - t; z(J) = sum_m g[m] x(J - m)
  const int t = threadIdx.x;
  auto zdot = [&](long long J, int m0, int m1) {
    double2 acc = make_double2(0.0, 0.0);
    const double* xp = sm.xs + (J - u_lo);
    for (int m = m0; m < m1; m++) {
      const double2 a = sm.taps[m + g.ha + 1];
      const double x = xp[-m];
      acc.x = fma(a.x, x, acc.x);
      acc.y = fma(a.y, x, acc.y);
    }
    return acc;
  };
  if (t < count) sm.z[t] = zdot(J_hi - t, -g.ha, g.ha + 1);
  // the extra position, split over the first warp
  if (t < 32) {
    const int per = (2 * g.ha + 1 + 31) / 32;
    const int m0 = -g.ha + t * per, m1 = min(m0 + per, g.ha + 1);
    double2 acc = m0 < m1 ? zdot(J_lo, m0, m1) : make_double2(0.0, 0.0);
    for (int off = 16; off > 0; off >>= 1) {
      acc.x += __shfl_down_sync(0xffffffffu, acc.x, off);
      acc.y += __shfl_down_sync(0xffffffffu, acc.y, off);
    }
    if (t == 0) sm.z[count] = acc;
  }
  __syncthreads();
  return true;
}

template <int FMT>
__global__ void __launch_bounds__(kGuardThreads) guard_kernel(GuardArgs g) {
  chain_wait();
  extern __shared__ double2 smem2[];
  __shared__ double red[kGuardThreads / 32];
  const int n_listed = min(*g.count, g.cap);
  if ((int)blockIdx.y >= n_listed) return;  // whole CTA
  const int t = threadIdx.x, part = blockIdx.x;
  const int nt = 2 * g.ha + 3;
  GuardSmem sm;
  sm.taps = smem2;
  sm.z = smem2 + nt;
  sm.xs = reinterpret_cast<double*>(smem2 + nt + kGuardThreads + 1);
  for (int i = t; i < nt; i += kGuardThreads)
    sm.taps[i] = (i == 0 || i == nt - 1) ? make_double2(0.0, 0.0)
                                         : make_double2(g.ga64[2 * (i - 1)], g.ga64[2 * (i - 1) + 1]);
  __syncthreads();
  const double dc = g.dc ? (double)*g.dc : 0.0;
  const int W = 2 * g.hb + 1;
  const long long last = g.total - 1;
  for (int y = blockIdx.y; y < n_listed; y += gridDim.y) {
    const long long s = g.list[y];
    const long long f = s / g.spp;
    const long long J = kOverlap + (s - f * g.spp);
    const int kk0 = part * kGuardThreads, kk = kk0 + t;
    const int count = min(kGuardThreads, W - kk0);
    // demod sample at tile position J - k of tile f (k = kk - hb), chunk position c
    auto chunk_pos = [&](int k_index) {
      const long long q = wrap_pos(J - (k_index - g.hb), g.tile);
      return min(max(f * g.spp + q - kOverlap, 0LL), last);
    };
    // the CTA's positions are consecutive (decreasing) when neither the tile
    // wrap nor the chunk clamp falls inside them
    const long long q_first = J - (kk0 - g.hb), q_end = J - (kk0 + count - 1 - g.hb);
    const bool consecutive = q_end >= 0 && q_first < g.tile && f * g.spp + q_end - kOverlap >= 0 &&
                             f * g.spp + q_first - kOverlap <= last;
    const long long c_first = chunk_pos(kk0);
    double contrib = 0.0;
    if (consecutive && stage_interior<FMT>(g, sm, c_first, count, dc)) {
      if (t < count) {
        const double2 z0 = sm.z[t], z1 = sm.z[t + 1];
        double d = atan2(z0.y, z0.x) - atan2(z1.y, z1.x);  // k_unwrap_to_hz (fm_demod.cu:222-244)
        if (d > kPi64) d -= kTau64;
        if (d < -kPi64) d += kTau64;
        contrib = g.hs64[kk] * (d * g.scale);
      }
    } else if (kk < W) {
      const long long c = chunk_pos(kk);
      const long long f2 = c / g.spp;
      const long long J2 = kOverlap + (c - f2 * g.spp);
      const long long tile0 = f2 * g.spp - kOverlap;  // chunk position of tile position 0
      // raw tile positions J2 + ha down to J2 - 1 - ha feed z(J2) and z(J2 - 1)
      const long long u_hi = J2 + g.ha;
      double2 z0 = make_double2(0.0, 0.0), z1 = make_double2(0.0, 0.0);
      const int nu = 2 * g.ha + 2;
      for (int n = 0; n < nu; n++) {
        const long long p = min(max(tile0 + wrap_pos(u_hi - n, g.tile), 0LL), last);
        const double x = raw64<FMT>(g, p, dc);
        const double2 a = sm.taps[n + 1], b = sm.taps[n];
        z0.x = fma(a.x, x, z0.x);
        z0.y = fma(a.y, x, z0.y);
        z1.x = fma(b.x, x, z1.x);
        z1.y = fma(b.y, x, z1.y);
      }
      double d = atan2(z0.y, z0.x) - atan2(z1.y, z1.x);
      if (d > kPi64) d -= kTau64;
      if (d < -kPi64) d += kTau64;
      contrib = g.hs64[kk] * (d * g.scale);
    }
    // fixed-order reduction: warp shuffle tree, then the warps in order
    for (int off = 16; off > 0; off >>= 1) contrib += __shfl_down_sync(0xffffffffu, contrib, off);
    if ((t & 31) == 0) red[t >> 5] = contrib;
    __syncthreads();
    if (t == 0) {
      double ps = 0.0;
      for (int w = 0; w < kGuardThreads / 32; w++) ps += red[w];
      g.part[(size_t)y * kGuardMaxParts + part] = ps;
      __threadfence();
      const int parts = (int)gridDim.x;
      if (atomicAdd(&g.done[y], 1) == parts - 1) {
        // every part of sample y is in: add them in part order
        __threadfence();
        double x64 = 0.0;
        for (int p = 0; p < parts; p++) x64 += __ldcg(&g.part[(size_t)y * kGuardMaxParts + p]);
        const bool in_pulse = x64 <= g.thr_hz;  // the reference's FP64 decision
        float r = (float)(x64 - g.ire0);
        if (in_pulse && !(r <= g.thr_rel)) r = g.thr_rel;
        if (!in_pulse && r <= g.thr_rel) r = nextafterf(g.thr_rel, 3.0e38f);
        g.sync[s] = r;
        if (g.values) g.values[y] = x64;
      }
    }
    __syncthreads();  // red, z and xs are reused by the next sample
  }
}

}  // namespace

int guard_parts(int hb) { return (2 * hb + 1 + kGuardThreads - 1) / kGuardThreads; }

cudaError_t launch_sync_guard(const GuardArgs& g, cudaStream_t st) {
  const int parts = guard_parts(g.hb);
  if (parts > kGuardMaxParts || g.cap <= 0) return cudaErrorInvalidValue;
  const size_t smem = (size_t)(2 * g.ha + 3 + kGuardThreads + 1) * sizeof(double2) +
                      (size_t)(kGuardThreads + 2 * g.ha + 2) * sizeof(double);
  // enough rows to spread a typical chunk's few flagged samples over the GPU;
  // rows past the listed count leave at once
  const int rows = std::max(1, std::min(g.cap, (148 * 8 + parts - 1) / parts));
  auto go = [&](auto kernel) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return launch_chained(kernel, dim3(parts, rows), dim3(kGuardThreads), smem, st, g);
  };
  if (g.in_fmt == kInS16) return go(guard_kernel<kInS16>);
  if (g.in_fmt == kInU16) return go(guard_kernel<kInU16>);
  return go(guard_kernel<kInU8>);
}

}  // namespace cuvhs
