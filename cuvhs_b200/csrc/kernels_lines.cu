// Line-geometry kernels: hsync refinement (reference K4,
// src/pipeline/hsync_refine.cu:21-239) and the luma TBC resampler (reference
// K5, src/pipeline/tbc_resample.cu:19-133).
//
// Signals are FP32 and stored relative to ire0; every sample position, window
// bound and crossing interpolation is FP64, as the reference computes them, so
// the integer window truncations match.
#include <cuda_runtime.h>

#include "cuvhs_internal.h"

namespace cuvhs {
namespace {

// First sample pair (i-1, i) in [start, start+count) with prev >= target > cur;
// returns the linearly interpolated crossing or -1.
__device__ double falling_cross(const float* __restrict__ s, int start, int count, double target, long long total) {
  if (start < 0 || (long long)start + count > total || count < 2) return -1.0;
  for (int i = start + 1; i < start + count; i++) {
    const double p = s[i - 1], q = s[i];
    if (p >= target && q < target) {
      const double a = p - target, b = q - target;
      const double fr = (a - b != 0.0) ? (a / (a - b)) : 0.0;
      return (double)(i - 1) + fr;
    }
  }
  return -1.0;
}

__device__ double rising_cross(const float* __restrict__ s, int start, int count, double target, long long total) {
  if (start < 0 || (long long)start + count > total || count < 2) return -1.0;
  if ((double)s[start] > target) return -1.0;
  for (int i = start + 1; i < start + count; i++) {
    const double p = s[i - 1], q = s[i];
    if (p < target && q >= target) {
      const double a = target - p, b = target - q;
      const double fr = (a + b != 0.0) ? (a / (a - b)) : 0.0;
      return (double)(i - 1) + fr;
    }
  }
  return -1.0;
}

// Order statistic n/2 of the window (the upper median for even n), n <= 64.
__device__ double window_median(const float* __restrict__ s, int start, int count, long long total) {
  if (start < 0 || (long long)start + count > total || count <= 0) return 0.0;
  const int n = min(count, 64);
  float buf[64];
  for (int i = 0; i < n; i++) buf[i] = s[start + i];
  const int mid = n / 2;
  for (int i = 0; i <= mid; i++) {
    int m = i;
    for (int j = i + 1; j < n; j++)
      if (buf[j] < buf[m]) m = j;
    const float t = buf[i];
    buf[i] = buf[m];
    buf[m] = t;
  }
  return (double)buf[mid];
}

__global__ void hsync_kernel(LineArgs a) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.fields * a.lines_per_frame) return;
  const int line = idx % a.lines_per_frame;
  if (line < a.active_line_start) return;
  const float* s = a.sync;
  const double thr = (double)a.thr_rel;
  const double us = a.one_us, hw = a.hsync_width;
  const double orig = a.ll[idx];
  const int ou = (int)(us + 0.5);
  // leading (falling) edge
  const double zc = falling_cross(s, (int)(orig - ou), ou * 2, thr, a.total);
  double left = -1.0;
  if (zc >= 0.0) {
    const int zi = (int)(zc + 0.5);
    const double sync_lv = window_median(s, zi + (int)(1.0 * us), (int)(1.5 * us), a.total);
    const double porch_lv = window_median(s, zi + (int)(8.0 * us), (int)(1.0 * us), a.total);
    if (porch_lv > sync_lv) {
      const double mid = (sync_lv + porch_lv) / 2.0;
      const double zc2 = falling_cross(s, (int)(orig - ou * 2), (int)(us * 4), mid, a.total);
      if (zc2 >= 0.0 && fabs(zc2 - zc) <= us * 0.5) left = zc2;
    }
  }
  // trailing (rising) edge
  double right = -1.0;
  const double rx = rising_cross(s, (int)(orig + hw - us), (int)(hw * 2), thr, a.total);
  if (rx >= 0.0) {
    const int zfi = (int)(rx - hw + 0.5);
    const double rs = window_median(s, zfi + (int)(1.0 * us), (int)(1.5 * us), a.total);
    const double rp = window_median(s, zfi + (int)(hw + 1.0 * us), (int)(1.0 * us), a.total);
    if (rp > rs) {
      const double rmid = (rs + rp) / 2.0;
      const double zc2r = rising_cross(s, (int)(orig + hw - us), (int)(hw * 2), rmid, a.total);
      if (zc2r >= 0.0 && fabs(zc2r - rx) <= us * 0.5) {
        const double cand = rx - hw + a.right_edge_offset;
        const double ref = (left >= 0.0) ? left : orig;
        if (fabs(cand - ref) <= us * 2.0) right = cand;
      }
    }
  }
  if (right >= 0.0) a.ll[idx] = right;
  else if (left >= 0.0) a.ll[idx] = left;
}

__global__ void luma_kernel(LineArgs a) {
  const int W = a.out_w, H = a.out_h;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)a.fields * H * W) return;
  const int field = (int)(idx / (H * W));
  const int rem = (int)(idx % (H * W));
  const int row = rem / W, col = rem % W;
  uint16_t out;
  if (row + 1 >= a.lines_per_frame) {
    out = 1024;
  } else {
    const double a0 = a.ll[(size_t)field * a.lines_per_frame + row];
    const double a1 = a.ll[(size_t)field * a.lines_per_frame + row + 1];
    const double coord = a0 + ((double)col / (double)W) * (a1 - a0);
    const int ci = (int)coord;
    if (ci < 1 || (long long)ci + 2 >= a.total) {
      out = 1024;
    } else {
      const float x = (float)(coord - (double)ci);
      const float p0 = __ldg(&a.video[ci - 1]), p1 = __ldg(&a.video[ci]);
      const float p2 = __ldg(&a.video[ci + 1]), p3 = __ldg(&a.video[ci + 2]);
      const float c1 = p2 - p0;
      const float c2 = 2.0f * p0 - 5.0f * p1 + 4.0f * p2 - p3;
      const float c3 = 3.0f * (p1 - p2) + p3 - p0;
      const float hz = p1 + 0.5f * x * (c1 + x * (c2 + x * c3));
      float v = hz * a.luma_gain + a.luma_offset;
      v = fminf(fmaxf(v, 0.0f), 65535.0f);
      out = (uint16_t)(v + 0.5f);
    }
  }
  a.luma[idx] = out;
}

}  // namespace

void launch_hsync_refine(const LineArgs& a, cudaStream_t st) {
  const int n = a.fields * a.lines_per_frame;
  if (n <= 0) return;
  hsync_kernel<<<(n + 127) / 128, 128, 0, st>>>(a);
}

void launch_luma(const LineArgs& a, cudaStream_t st) {
  const long long n = (long long)a.fields * a.out_h * a.out_w;
  if (n <= 0) return;
  luma_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a);
}

}  // namespace cuvhs
