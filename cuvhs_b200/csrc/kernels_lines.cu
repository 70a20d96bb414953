// Line-geometry kernels: hsync refinement (reference K4,
// src/pipeline/hsync_refine.cu:21-239) and the luma TBC resampler (reference
// K5, src/pipeline/tbc_resample.cu:19-133).
//
// Signals are FP32 and stored relative to ire0; every sample position, window
// bound and crossing interpolation is FP64, as the reference computes them, so
// the integer window truncations match.
#include <cuda_runtime.h>

#include <cstdint>

#include "chain.cuh"
#include "cuvhs_internal.h"

namespace cuvhs {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kHsyncWarps = 4;   // lines per 128-thread CTA
constexpr int kLumaThreads = 128;

__device__ __forceinline__ double shfl_d(double v, int src) { return __shfl_sync(kFull, v, src); }

// A line's sync samples: the window the refinement reads is staged in shared
// memory (one coalesced burst per warp instead of a dependent global load per
// scan step); a position outside the staged range reads global memory, so the
// result never depends on the staging.
struct SyncWindow {
  const float* g;   // the chunk's sync signal
  const float* sm;  // staged samples [lo, lo + n)
  long long lo;
  int n;
  __device__ __forceinline__ float operator()(long long i) const {
    const long long k = i - lo;
    return (unsigned long long)k < (unsigned long long)n ? sm[k] : __ldg(g + i);
  }
};

// Samples a line's refinement can read, relative to floor(line start): from
// 2 us before (the second falling scan) to 3 hsync widths + 1 us after (the
// rising scan, its re-centred porch median) or 10 us after (the falling
// edge's porch median), with a margin for the integer truncations.  0 means
// no staging (a window that would not fit the CTA's shared memory).
constexpr int kHsyncWinMax = 2816;  // floats per warp: 4 warps in 44 KiB
__host__ __device__ inline int hsync_lead(double us) { return 2 * (int)(us + 0.5) + 8; }
__host__ __device__ inline int hsync_window(double us, double hw) {
  const double tail = fmax(3.0 * hw + us, 10.0 * us + 1.0);
  const int n = ((hsync_lead(us) + (int)ceil(tail) + 16) + 3) & ~3;
  return n <= kHsyncWinMax ? n : 0;
}

// First sample pair (i-1, i) in [start, start+count) with prev >= target > cur;
// returns the linearly interpolated crossing or -1.  The warp tests 32 pairs
// per step and takes the lowest hit, so the result is the sequential scan's.
__device__ double falling_cross(const SyncWindow& s, int start, int count, double target, long long total,
                                int lane) {
  if (start < 0 || (long long)start + count > total || count < 2) return -1.0;
  for (int base = start + 1; base < start + count; base += 32) {
    const int i = base + lane;
    double p = 0.0, q = 0.0;
    bool hit = false;
    if (i < start + count) {
      p = s(i - 1);
      q = s(i);
      hit = p >= target && q < target;
    }
    const unsigned m = __ballot_sync(kFull, hit);
    if (m) {
      const int src = __ffs(m) - 1;
      double r = 0.0;
      if (lane == src) {
        const double a = p - target, b = q - target;
        const double fr = (a - b != 0.0) ? (a / (a - b)) : 0.0;
        r = (double)(i - 1) + fr;
      }
      return shfl_d(r, src);
    }
  }
  return -1.0;
}

__device__ double rising_cross(const SyncWindow& s, int start, int count, double target, long long total,
                               int lane) {
  if (start < 0 || (long long)start + count > total || count < 2) return -1.0;
  if ((double)s(start) > target) return -1.0;
  for (int base = start + 1; base < start + count; base += 32) {
    const int i = base + lane;
    double p = 0.0, q = 0.0;
    bool hit = false;
    if (i < start + count) {
      p = s(i - 1);
      q = s(i);
      hit = p < target && q >= target;
    }
    const unsigned m = __ballot_sync(kFull, hit);
    if (m) {
      const int src = __ffs(m) - 1;
      double r = 0.0;
      if (lane == src) {
        const double a = target - p, b = target - q;
        const double fr = (a + b != 0.0) ? (a / (a - b)) : 0.0;
        r = (double)(i - 1) + fr;
      }
      return shfl_d(r, src);
    }
  }
  return -1.0;
}

// One compare-exchange stage of a warp bitonic sort: element e (value x) and
// element e ^ j (lane ^ j), ascending within blocks of k elements whose
// index bit k is clear, descending in the others.
__device__ __forceinline__ float bitonic_stage(float x, int e, int j, int k) {
  const float y = __shfl_xor_sync(kFull, x, j);
  const bool keep_min = ((e & k) == 0) == ((e & j) == 0);
  return keep_min ? fminf(x, y) : fmaxf(x, y);
}

// Order statistic n/2 of the window (the upper median for even n), n <= 64:
// the window, padded with +inf, is sorted across the warp by a bitonic
// network (32 elements, one per lane, when n <= 32; else 64, lane l holding
// elements l and l + 32), and element n/2 is read from its lane.  Ties hold
// equal values, so the result is the window's order statistic whichever
// duplicate lands there.
__device__ double window_median(const SyncWindow& s, int start, int count, long long total, int lane) {
  if (start < 0 || (long long)start + count > total || count <= 0) return 0.0;
  const int n = min(count, 64);
  const int mid = n / 2;
  float x0 = lane < n ? s(start + lane) : INFINITY;
  if (n <= 32) {
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) x0 = bitonic_stage(x0, lane, j, k);
    return (double)__shfl_sync(kFull, x0, mid);
  }
  float x1 = lane + 32 < n ? s(start + lane + 32) : INFINITY;
#pragma unroll
  for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j == 32) {  // partners in the same lane; k = 64 sorts ascending
        const float lo = fminf(x0, x1), hi = fmaxf(x0, x1);
        x0 = lo;
        x1 = hi;
      } else {
        x0 = bitonic_stage(x0, lane, j, k);
        x1 = bitonic_stage(x1, lane + 32, j, k);
      }
    }
  }
  return (double)__shfl_sync(kFull, mid < 32 ? x0 : x1, mid & 31);
}

// One warp per line location (lines from the first active line to the end of
// the frame table).  The warp first stages the line's sync window.
template <class Src>
__global__ void __launch_bounds__(32 * kHsyncWarps) hsync_kernel(const __grid_constant__ Src src) {
  const LineArgs& a = src.get();
  extern __shared__ __align__(16) float hs_win[];
  chain_wait();
  const int lane = threadIdx.x & 31;
  const int idx = blockIdx.x * kHsyncWarps + (threadIdx.x >> 5);
  if (idx >= a.fields * a.lines_per_frame) return;  // whole warp
  const int line = idx % a.lines_per_frame;
  if (line < a.active_line_start) return;
  const double thr = (double)a.thr_rel;
  const double us = a.one_us, hw = a.hsync_width;
  const double orig = a.ll[idx];
  const int ou = (int)(us + 0.5);
  const int nw = hsync_window(us, hw);
  SyncWindow s{a.sync, hs_win + (threadIdx.x >> 5) * nw, 0, 0};
  if (nw > 0 && orig > -1e15 && orig < 1e15) {
    long long lo = ((long long)floor(orig) - hsync_lead(us)) & ~3LL;
    long long hi = min(lo + nw, a.total);
    if (lo < 0) lo = 0;
    if (hi > lo) {
      const int n = (int)(hi - lo);
      float* w = const_cast<float*>(s.sm);
      const bool vec = (reinterpret_cast<uintptr_t>(a.sync) & 15) == 0;
      const int n4 = vec ? n >> 2 : 0;
      const float4* g4 = reinterpret_cast<const float4*>(a.sync + lo);
      for (int k = lane; k < n4; k += 32) reinterpret_cast<float4*>(w)[k] = __ldg(g4 + k);
      for (int k = 4 * n4 + lane; k < n; k += 32) w[k] = __ldg(a.sync + lo + k);
      s.lo = lo;
      s.n = n;
    }
    __syncwarp();
  }
  // leading (falling) edge
  const double zc = falling_cross(s, (int)(orig - ou), ou * 2, thr, a.total, lane);
  double left = -1.0;
  if (zc >= 0.0) {
    const int zi = (int)(zc + 0.5);
    const double sync_lv = window_median(s, zi + (int)(1.0 * us), (int)(1.5 * us), a.total, lane);
    const double porch_lv = window_median(s, zi + (int)(8.0 * us), (int)(1.0 * us), a.total, lane);
    if (porch_lv > sync_lv) {
      const double mid = (sync_lv + porch_lv) / 2.0;
      const double zc2 = falling_cross(s, (int)(orig - ou * 2), (int)(us * 4), mid, a.total, lane);
      if (zc2 >= 0.0 && fabs(zc2 - zc) <= us * 0.5) left = zc2;
    }
  }
  // trailing (rising) edge
  double right = -1.0;
  const double rx = rising_cross(s, (int)(orig + hw - us), (int)(hw * 2), thr, a.total, lane);
  if (rx >= 0.0) {
    const int zfi = (int)(rx - hw + 0.5);
    const double rs = window_median(s, zfi + (int)(1.0 * us), (int)(1.5 * us), a.total, lane);
    const double rp = window_median(s, zfi + (int)(hw + 1.0 * us), (int)(1.0 * us), a.total, lane);
    if (rp > rs) {
      const double rmid = (rs + rp) / 2.0;
      const double zc2r = rising_cross(s, (int)(orig + hw - us), (int)(hw * 2), rmid, a.total, lane);
      if (zc2r >= 0.0 && fabs(zc2r - rx) <= us * 0.5) {
        const double cand = rx - hw + a.right_edge_offset;
        const double ref = (left >= 0.0) ? left : orig;
        if (fabs(cand - ref) <= us * 2.0) right = cand;
      }
    }
  }
  if (lane == 0) {
    if (right >= 0.0) a.ll[idx] = right;
    else if (left >= 0.0) a.ll[idx] = left;
  }
}

// One CTA per output row: the row's two line starts are read once, the column
// fractions col/W come from a table (the same FP64 quotient), and consecutive
// threads write consecutive pixels.  The row's source window -- the samples
// from just before the line start to just past the next line's -- is first
// staged in shared memory with coalesced 16-byte loads (each sample feeds two
// to three output columns), then every Catmull-Rom tap reads shared memory.
// A row whose window would not fit (line locations of a lost signal) reads
// global memory directly, with the same arithmetic.
constexpr int kLumaWindow = 4096;  // staged samples per row (a line is 1780 at 28 MHz, 2560 at 40 MHz PAL)

__device__ __forceinline__ uint16_t luma_pixel(const LineArgs& a, float p0, float p1, float p2, float p3, float x,
                                               bool ok) {
  const float c1 = p2 - p0;
  const float c2 = 2.0f * p0 - 5.0f * p1 + 4.0f * p2 - p3;
  const float c3 = 3.0f * (p1 - p2) + p3 - p0;
  const float hz = p1 + 0.5f * x * (c1 + x * (c2 + x * c3));
  float v = hz * a.luma_gain + a.luma_offset;
  v = fminf(fmaxf(v, 0.0f), 65535.0f);
  return ok ? (uint16_t)(v + 0.5f) : a.oob_value;
}

template <class Src>
__global__ void __launch_bounds__(kLumaThreads) luma_kernel(const __grid_constant__ Src src) {
  const LineArgs& a = src.get();
  const int W = a.out_w, H = a.out_h;
  const int grow = blockIdx.x;  // field * H + row
  const int field = grow / H, row = grow % H;
  if (field >= a.fields) return;  // whole CTA: a batched capture with fewer fields
  chain_wait();
  __shared__ __align__(16) float win[kLumaWindow];
  uint16_t* out = a.luma + (size_t)grow * W;
  if (row + 1 >= a.lines_per_frame) {
    for (int col = threadIdx.x; col < W; col += kLumaThreads) out[col] = a.oob_value;
    return;
  }
  const double a0 = a.ll[(size_t)field * a.lines_per_frame + row];
  const double a1 = a.ll[(size_t)field * a.lines_per_frame + row + 1];
  const double span = a1 - a0;
  // staged window [lo, lo + n): the taps ci-1 .. ci+2 of every in-range
  // column, ci = floor(coordinate) between the two line starts (a coordinate
  // may round a few ulp past either one, so the window reaches one more
  // sample each way)
  const double cmin = fmin(a0, a1), cmax = fmax(a0, a1);
  bool staged = cmin >= -4.0 && cmax < (double)a.total && cmax - cmin < (double)(kLumaWindow - 16);
  long long lo = 0;
  int n = 0;
  if (staged) {
    lo = ((long long)floor(cmin) - 2) & ~3LL;  // 16-byte aligned start
    if (lo < 0) lo = 0;
    const long long hi = min((long long)floor(cmax) + 4, a.total);
    n = (int)(hi - lo);
    staged = n > 0 && n <= kLumaWindow;
  }
  if (staged) {
    const float* src = a.video + lo;
    const bool vec = (reinterpret_cast<uintptr_t>(a.video) & 15) == 0;
    const int n4 = vec ? n >> 2 : 0;
    for (int i = threadIdx.x; i < n4; i += kLumaThreads)
      reinterpret_cast<float4*>(win)[i] = __ldg(reinterpret_cast<const float4*>(src) + i);
    for (int i = 4 * n4 + threadIdx.x; i < n; i += kLumaThreads) win[i] = __ldg(&src[i]);
    __syncthreads();
#pragma unroll 4
    for (int col = threadIdx.x; col < W; col += kLumaThreads) {
      const double coord = a0 + __ldg(&a.col_frac[col]) * span;
      const int ci = (int)coord;
      const bool ok = ci >= 1 && (long long)ci + 2 < a.total;
      const int k = ok ? (int)((long long)ci - lo) : 1;  // in-range taps lie in the window
      const float x = (float)(coord - (double)ci);
      out[col] = luma_pixel(a, win[k - 1], win[k], win[k + 1], win[k + 2], x, ok);
    }
    return;
  }
  // The loads do not depend on the range test (an out-of-range column reads
  // the first samples and writes the out-of-range value), so the unrolled
  // loop keeps several columns' loads in flight.
#pragma unroll 4
  for (int col = threadIdx.x; col < W; col += kLumaThreads) {
    const double coord = a0 + __ldg(&a.col_frac[col]) * span;
    const int ci = (int)coord;
    const bool ok = ci >= 1 && (long long)ci + 2 < a.total;
    const int cl = ok ? ci : 1;
    const float x = (float)(coord - (double)ci);
    out[col] = luma_pixel(a, __ldg(&a.video[cl - 1]), __ldg(&a.video[cl]), __ldg(&a.video[cl + 1]),
                          __ldg(&a.video[cl + 2]), x, ok);
  }
}

}  // namespace

void launch_hsync_refine(const LineArgs& a, cudaStream_t st) {
  const int n = a.fields * a.lines_per_frame;
  if (n <= 0) return;
  using S = ArgsOne<LineArgs>;
  const size_t smem = (size_t)kHsyncWarps * hsync_window(a.one_us, a.hsync_width) * sizeof(float);
  launch_chained(hsync_kernel<S>, dim3((n + kHsyncWarps - 1) / kHsyncWarps), dim3(32 * kHsyncWarps), smem, st, S{a});
}

void launch_luma(const LineArgs& a, cudaStream_t st) {
  const int rows = a.fields * a.out_h;
  if (rows <= 0) return;
  using S = ArgsOne<LineArgs>;
  launch_chained(luma_kernel<S>, dim3(rows), dim3(kLumaThreads), 0, st, S{a});
}

void launch_hsync_refine_many(const ArgsMany<LineArgs>& p, int portions, int max_fields, cudaStream_t st) {
  const int n = max_fields * p.a[0].lines_per_frame;
  if (n <= 0 || portions <= 0) return;
  const size_t smem = (size_t)kHsyncWarps * hsync_window(p.a[0].one_us, p.a[0].hsync_width) * sizeof(float);
  launch_chained(hsync_kernel<ArgsMany<LineArgs>>, dim3((n + kHsyncWarps - 1) / kHsyncWarps, 1, portions),
                 dim3(32 * kHsyncWarps), smem, st, p);
}

void launch_luma_many(const ArgsMany<LineArgs>& p, int portions, int max_fields, cudaStream_t st) {
  const int rows = max_fields * p.a[0].out_h;
  if (rows <= 0 || portions <= 0) return;
  launch_chained(luma_kernel<ArgsMany<LineArgs>>, dim3(rows, 1, portions), dim3(kLumaThreads), 0, st, p);
}

}  // namespace cuvhs
