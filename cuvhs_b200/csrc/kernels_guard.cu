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
// of the 2*hb + 1 demod samples of the sync window (two FP64 analytic-signal
// dot products of 2*ha + 1 taps each per demod sample).  Each CTA writes its
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

template <int FMT>
__global__ void __launch_bounds__(kGuardThreads) guard_kernel(GuardArgs g) {
  chain_wait();
  extern __shared__ double2 taps[];  // [2*ha + 3]: 0, g[-ha..ha], 0
  __shared__ double red[kGuardThreads / 32];
  const int n_listed = min(*g.count, g.cap);
  if ((int)blockIdx.y >= n_listed) return;  // whole CTA
  const int t = threadIdx.x, part = blockIdx.x;
  const int nt = 2 * g.ha + 3;
  for (int i = t; i < nt; i += kGuardThreads)
    taps[i] = (i == 0 || i == nt - 1) ? make_double2(0.0, 0.0)
                                      : make_double2(g.ga64[2 * (i - 1)], g.ga64[2 * (i - 1) + 1]);
  __syncthreads();
  const double dc = g.dc ? (double)*g.dc : 0.0;
  const int W = 2 * g.hb + 1;
  const long long last = g.total - 1;
  for (int y = blockIdx.y; y < n_listed; y += gridDim.y) {
    const long long s = g.list[y];
    const long long f = s / g.spp;
    const long long J = kOverlap + (s - f * g.spp);
    const int kk = part * kGuardThreads + t;
    double contrib = 0.0;
    if (kk < W) {
      // demod sample at tile position J - k of tile f (k = kk - hb)
      const long long q = wrap_pos(J - (kk - g.hb), g.tile);
      const long long c = min(max(f * g.spp + q - kOverlap, 0LL), last);
      const long long f2 = c / g.spp;
      const long long J2 = kOverlap + (c - f2 * g.spp);
      const long long tile0 = f2 * g.spp - kOverlap;  // chunk position of tile position 0
      // raw tile positions J2 + ha down to J2 - 1 - ha feed z(J2) and z(J2 - 1)
      const long long u_hi = J2 + g.ha, u_lo = J2 - 1 - g.ha;
      double2 z0 = make_double2(0.0, 0.0), z1 = make_double2(0.0, 0.0);
      const int nu = 2 * g.ha + 2;
      if (u_lo >= 0 && u_hi < g.tile && tile0 + u_lo >= 0 && tile0 + u_hi <= last && tile0 + u_hi < g.n_read) {
        const long long p0 = tile0 + u_hi;  // interior: no wrap, no clamp, no zero fill
#pragma unroll 4
        for (int n = 0; n < nu; n++) {
          const double x = (double)raw_convert<FMT>(g.raw, (int)(p0 - n)) - dc;
          const double2 a = taps[n + 1], b = taps[n];
          z0.x = fma(a.x, x, z0.x);
          z0.y = fma(a.y, x, z0.y);
          z1.x = fma(b.x, x, z1.x);
          z1.y = fma(b.y, x, z1.y);
        }
      } else {
        for (int n = 0; n < nu; n++) {
          const long long p = min(max(tile0 + wrap_pos(u_hi - n, g.tile), 0LL), last);
          const double x = raw64<FMT>(g, p, dc);
          const double2 a = taps[n + 1], b = taps[n];
          z0.x = fma(a.x, x, z0.x);
          z0.y = fma(a.y, x, z0.y);
          z1.x = fma(b.x, x, z1.x);
          z1.y = fma(b.y, x, z1.y);
        }
      }
      double d = atan2(z0.y, z0.x) - atan2(z1.y, z1.x);  // k_unwrap_to_hz (fm_demod.cu:222-244)
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
    __syncthreads();  // red is reused by the next sample
  }
}

}  // namespace

int guard_parts(int hb) { return (2 * hb + 1 + kGuardThreads - 1) / kGuardThreads; }

cudaError_t launch_sync_guard(const GuardArgs& g, cudaStream_t st) {
  const int parts = guard_parts(g.hb);
  if (parts > kGuardMaxParts || g.cap <= 0) return cudaErrorInvalidValue;
  const size_t smem = (size_t)(2 * g.ha + 3) * sizeof(double2);
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
