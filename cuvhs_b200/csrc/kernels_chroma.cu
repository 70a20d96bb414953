// Colour-under chroma kernels (reference K6, src/pipeline/chroma_decode.cu:526-1002).
//
//  * prefilter: the reference band-passes each zero-padded tile (60 kHz - 1.2 MHz,
//    |Butterworth order 4|^2) with one FP64 FFT pair per field in a serial loop
//    (chroma_decode.cu:596-633).  Here: overlap-save over the same circular
//    zero-padded tile, 16384-point shared-memory transforms; the kernel is real,
//    so two output blocks ride in the real and imaginary parts of one transform.
//  * lines: Catmull-Rom resample of the prefiltered signal on the line grid,
//    times the heterodyne carrier with the per-line track rotation
//    (chroma_decode.cu:75-157), 1024-point transform, keep bins fsc +/- 500 kHz
//    (chroma_decode.cu:163-182), inverse, then burst RMS -> ACC gain -> u16
//    (chroma_decode.cu:188-231).  One warp transforms two lines at once.
//  * metric: adjacent-line burst cancellation per field (chroma_decode.cu:242-296).
#include <cuda_runtime.h>

#include "chain.cuh"
#include "cuvhs_internal.h"
#include "raw_input.cuh"
#include "reg_fft.cuh"

namespace cuvhs {
namespace {

// 16 elements per thread, 1024 threads at 64 registers each (spill-free since
// the inverse transform takes an opaque thread index); 32 elements with 512
// threads at 128 registers is also spill-free but measured 9% slower.
constexpr int kElemsC = 16;
constexpr int kThreadsC = Design::kNc / kElemsC;
// Line kernel geometry: a line pair (two lines in one complex transform) per
// group of line_tp threads with a padded N-point buffer (NTSC 1024, PAL 2048
// points), line_pairs groups per CTA.  NTSC pairs take two warps, so each
// thread holds one radix-16 butterfly per pass and the kernel fits 64
// registers (32 warps per SM to cover the gathers' latency).
template <int N>
__host__ __device__ constexpr int line_tp() { return N <= 1024 ? 64 : 32; }
template <int N>
__host__ __device__ constexpr int line_pairs() { return 2; }  // at most 4 (the two-warp barriers)
template <int N>
__host__ __device__ constexpr int line_threads() { return line_tp<N>() * line_pairs<N>(); }
template <int N>
__host__ __device__ constexpr int line_min_ctas() { return N <= 1024 ? 8 : 1; }

// Barrier of one line pair's threads (the transform's barrier).
template <int TP>
__device__ __forceinline__ void pair_sync() {
  static_assert(TP == 32 || TP == 64, "one or two warps per line pair");
  fft_sync<TP>();
}

// Two adjacent output blocks ride in the real and imaginary parts of one
// transform (the kernel is real).  Thread t holds block samples t + T*q, q < kElemsC.
template <int FMT, class Src>
__global__ void __launch_bounds__(kThreadsC, 1) prefilter_kernel(const __grid_constant__ Src src) {
  const ChromaArgs& a = src.get();
  if ((int)blockIdx.y >= a.fields) return;  // whole CTA: a batched capture with fewer tiles
  chain_wait();
  constexpr int N = Design::kNc, T = kThreadsC, E = kElemsC;
  extern __shared__ float2 sm[];
  const int t = threadIdx.x;
  const int f = blockIdx.y;
  const int i0 = blockIdx.x * 2 * a.c_out;  // first output of the real half
  const int tile = f * a.spp;               // chunk position of the tile
  const float dc = a.dc ? *a.dc : 0.0f;
  float2 v[E];
  const int base = i0 - a.c_half;  // tile position of block sample 0 (before the wrap)
  if (base >= 0 && base + N + a.c_out <= a.spp && tile + base + N + a.c_out <= a.n_read) {
    // interior: no wrap, inside the tile's samples and the samples read
    const int p = tile + base + t;
#pragma unroll
    for (int q = 0; q < E; q++)
      v[q] = make_float2(raw_convert<FMT>(a.raw, p + T * q) - dc, raw_convert<FMT>(a.raw, p + T * q + a.c_out) - dc);
  } else {
    // the zero-padded tile wraps at most once (ctile > N + c_out)
#pragma unroll
    for (int q = 0; q < E; q++) {
      int q0 = base + t + T * q;
      if (q0 < 0) q0 += a.ctile;
      else if (q0 >= a.ctile) q0 -= a.ctile;
      int q1 = q0 + a.c_out;
      if (q1 >= a.ctile) q1 -= a.ctile;
      const float v0 = q0 < a.spp ? raw_sample<FMT>(a.raw, tile + q0, a.n_read, dc) : 0.0f;
      const float v1 = q1 < a.spp ? raw_sample<FMT>(a.raw, tile + q1, a.n_read, dc) : 0.0f;
      v[q] = make_float2(v0, v1);
    }
  }
  RegFFT<N, E>::run<false>(v, sm, a.tw_c, t);
#pragma unroll
  for (int q = 0; q < E; q++) {
    const float g = __ldg(&a.gc[t + T * q]);
    v[q] = make_float2(v[q].x * g, v[q].y * g);
  }
  RegFFT<N, E>::run<true>(v, sm, a.tw_c_inv, opaque_index(t));
  float* out = a.pre + (size_t)f * a.spp;
#pragma unroll
  for (int q = 0; q < E; q++) {
    const int i = t + T * q - a.c_half;
    if (i >= 0 && i < a.c_out) {
      const int p0 = i0 + i, p1 = i0 + a.c_out + i;
      if (p0 < a.spp) out[p0] = v[q].x;
      if (p1 < a.spp) out[p1] = v[q].y;
    }
  }
}

// Per-line constants of the heterodyne resampler: the line's start and length
// (chunk samples), its first output index and the track's quarter-turn
// carrier rotation.  ok is false for lines past the line-location table.
struct HetLine {
  double a0, span;
  int ubase;  // row * out_w
  float lpf;  // 0.5 * ((row * rot) & 3): the rotation in half turns
  bool ok;
};

__device__ __forceinline__ HetLine het_line(const ChromaArgs& a, int gl) {
  HetLine L;
  const int field = gl / a.out_h, row = gl % a.out_h;
  L.ok = row + 1 < a.lines_per_frame;
  L.a0 = 0.0;
  L.span = 0.0;
  if (L.ok) {
    const double a0 = a.ll[(size_t)field * a.lines_per_frame + row];
    const double a1 = a.ll[(size_t)field * a.lines_per_frame + row + 1];
    L.a0 = a0;
    L.span = a1 - a0;
  }
  const int rot = a.track[field] ? 1 : 3;
  L.lpf = 0.5f * (float)((row * rot) & 3);
  L.ubase = row * a.out_w;
  return L;
}

// Heterodyned, resampled chroma sample of line L at column c (frac = c / out_w).
// The loads do not depend on the range test (an out-of-range column reads
// the first samples and is zeroed at the end), so an unrolled caller keeps
// several columns' loads in flight.
__device__ __forceinline__ float het_at(const ChromaArgs& a, const HetLine& L, double frac, int c) {
  const double coord = L.a0 + frac * L.span;
  const int ci = (int)coord;
  const bool ok = L.ok && ci >= 1 && (long long)ci + 2 < a.total;
  const int cl = ok ? ci : 1;
  const float x = (float)(coord - (double)ci);
  const float p0 = __ldg(&a.pre[cl - 1]), p1 = __ldg(&a.pre[cl]);
  const float p2 = __ldg(&a.pre[cl + 1]), p3 = __ldg(&a.pre[cl + 2]);
  const float c1 = p2 - p0;
  const float c2 = 2.0f * p0 - 5.0f * p1 + 4.0f * p2 - p3;
  const float c3 = 3.0f * (p1 - p2) + p3 - p0;
  const float v = p1 + 0.5f * x * (c1 + x * (c2 + x * c3));
  // carrier phase in FP64 turns, reduced before the FP32 cosine
  const double u = a.het_scale * (double)(L.ubase + c);
  const float fr = (float)(u - floor(u));
  const float het = -cospif(2.0f * fr + L.lpf);
  return ok ? v * het : 0.0f;
}

// nlines < 0: every line of the capture's a.fields fields (a batched round).
template <int N, class Src>
__global__ void __launch_bounds__(line_threads<N>(), line_min_ctas<N>())
    lines_kernel(const __grid_constant__ Src src, int line0, int nlines, int write_output) {
  const ChromaArgs& a = src.get();
  if (nlines < 0) nlines = a.fields * a.out_h;
  chain_wait();
  constexpr int TP = line_tp<N>(), P = line_pairs<N>();
  static_assert(TP == 32 || P <= 4, "two-warp pairs use named barriers 1..4");
  __shared__ float2 sm_all[P][fft_pad(N)];
  __shared__ float acc_sh[P][2];
  const int g = threadIdx.x / TP, tid = threadIdx.x % TP, lane = threadIdx.x & 31;
  float2* sm = sm_all[g];
  const int pair = blockIdx.x * P + g;
  const int la = 2 * pair, lb = la + 1;  // relative to line0
  if (la >= nlines) return;               // the pair's warps leave together
  const bool has_b = lb < nlines;
  const HetLine A = het_line(a, line0 + la);
  HetLine B = A;
  if (has_b) B = het_line(a, line0 + lb);
  B.ok = B.ok && has_b;
  // the gather is latency bound: unrolled so that several columns' loads are
  // in flight (the FFT below sets the register budget, not this loop)
#pragma unroll 4
  for (int c = tid; c < N; c += TP) {
    float va = 0.0f, vb = 0.0f;
    if (c < a.out_w) {
      const double frac = __ldg(&a.col_frac[c]);
      va = het_at(a, A, frac, c);
      vb = het_at(a, B, frac, c);
    }
    sm[pidx(c)] = make_float2(va, vb);
  }
  pair_sync<TP>();
  smem_fft<N, TP, false>(sm, a.tw_line, tid);
  const int lo = a.fsc_bin - a.bw_bins, hi = a.fsc_bin + a.bw_bins;
  const float scale = 1.0f / (float)N;
  for (int k = tid; k < N; k += TP) {
    const int kk = k <= N / 2 ? k : N - k;
    const float m = (kk >= lo && kk <= hi) ? scale : 0.0f;
    const float2 x = sm[pidx(k)];
    sm[pidx(k)] = make_float2(x.x * m, x.y * m);
  }
  pair_sync<TP>();
  smem_fft<N, TP, true>(sm, a.tw_line_inv, opaque_index(tid));
  // burst RMS per line -> ACC gain, summed by the pair's first warp in a
  // fixed order (lane sums i = lane, lane + 32, ..., then a butterfly)
  if (tid < 32) {
    const int bl = a.burst_len;
    float ssa = 0.0f, ssb = 0.0f;
    for (int i = lane; i < bl; i += 32) {
      const float2 v = sm[pidx(a.burst_start + i)];
      ssa += v.x * v.x;
      ssb += v.y * v.y;
      a.burst[(size_t)(line0 + la) * bl + i] = v.x;
      if (has_b) a.burst[(size_t)(line0 + lb) * bl + i] = v.y;
    }
    for (int off = 16; off > 0; off >>= 1) {
      ssa += __shfl_xor_sync(0xffffffffu, ssa, off);
      ssb += __shfl_xor_sync(0xffffffffu, ssb, off);
    }
    const float rms_a = sqrtf(ssa / (float)bl), rms_b = sqrtf(ssb / (float)bl);
    if (lane == 0) {
      acc_sh[g][0] = rms_a > 1.0f ? a.burst_abs_ref / rms_a : 0.0f;
      acc_sh[g][1] = rms_b > 1.0f ? a.burst_abs_ref / rms_b : 0.0f;
    }
  }
  if (!write_output) return;  // uniform over the pair: no barrier follows
  pair_sync<TP>();
  const float acc_a = acc_sh[g][0], acc_b = acc_sh[g][1];
  uint16_t* oa = a.chroma + (size_t)(line0 + la) * a.out_w;
  uint16_t* ob = a.chroma + (size_t)(line0 + lb) * a.out_w;
  for (int c = tid; c < a.out_w; c += TP) {
    const float2 v = sm[pidx(c)];
    const float xa = fminf(fmaxf(v.x * acc_a + 32768.0f, 0.0f), 65535.0f);
    oa[c] = (uint16_t)(xa + 0.5f);
    if (has_b) {
      const float xb = fminf(fmaxf(v.y * acc_b + 32768.0f, 0.0f), 65535.0f);
      ob[c] = (uint16_t)(xb + 0.5f);
    }
  }
}

// One CTA per field: mean over line pairs (16+2p, 17+2p), p < (out_h - 33)/2,
// of the mean |a + b| over the burst window.  Each thread sums one pair's
// window in sample order (its loads all issued first), and the first warp
// adds the pair means exactly as a warp-per-field loop would: lane l takes
// pairs l, l + 32, ... in order, then a butterfly over the lanes.
// BL: the burst window length when known at compile time (NTSC 36, PAL 40), 0 = a.burst_len.
constexpr int kMetricThreads = 256;
// nfields < 0: every field of the capture (a batched round).
template <int BL, class Src>
__global__ void __launch_bounds__(kMetricThreads) metric_kernel(const __grid_constant__ Src src, int field0,
                                                                int nfields) {
  const ChromaArgs& a = src.get();
  if (nfields < 0) nfields = a.fields;
  chain_wait();
  __shared__ double pair_mean[kMetricThreads];
  const int bl = BL > 0 ? BL : a.burst_len;
  const int f = field0 + blockIdx.x;
  if (blockIdx.x >= nfields) return;  // whole CTA
  const int skip = 16;
  const int npairs = min((a.out_h - 2 * skip - 1) / 2, kMetricThreads);
  for (int p = threadIdx.x; p < npairs; p += kMetricThreads) {
    const int line = f * a.out_h + skip + 2 * p;
    const float* x = a.burst + (size_t)line * bl;
    const float* y = x + bl;
    double s = 0.0;
    if constexpr (BL > 0 && BL % 4 == 0) {
      // rows start on 16-byte boundaries (BL floats per row)
      float4 xv[BL / 4], yv[BL / 4];
#pragma unroll
      for (int q = 0; q < BL / 4; q++) {
        xv[q] = __ldg(reinterpret_cast<const float4*>(x) + q);
        yv[q] = __ldg(reinterpret_cast<const float4*>(y) + q);
      }
#pragma unroll
      for (int q = 0; q < BL / 4; q++) {
        s += fabs((double)xv[q].x + (double)yv[q].x);
        s += fabs((double)xv[q].y + (double)yv[q].y);
        s += fabs((double)xv[q].z + (double)yv[q].z);
        s += fabs((double)xv[q].w + (double)yv[q].w);
      }
    } else {
      for (int i = 0; i < bl; i++) s += fabs((double)x[i] + (double)y[i]);
    }
    pair_mean[p] = s / bl;
  }
  __syncthreads();
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  double acc = 0.0;
  for (int p = lane; p < npairs; p += 32) acc += pair_mean[p];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) a.metric[f] = npairs > 0 ? acc / npairs : 1e9;
}

// The trial passes' burst metrics: per trial, pair means (one thread each,
// the window summed in sample order) added in line order by one thread, the
// host restatement's operations in its order, so the pick is the host's.
constexpr int kPickThreads = 256;
__global__ void __launch_bounds__(kPickThreads) track_pick_kernel(const TrackPickArgs a) {
  chain_wait();
  __shared__ double pair_mean[2][kPickThreads];
  __shared__ int det;
  const int skip = 16, bl = a.burst_len;
  int npairs = 0;
  for (int line = skip; line < a.out_h - skip - 1; line += 2) npairs++;
  npairs = min(npairs, kPickThreads);
  for (int k = threadIdx.x; k < 2 * npairs; k += kPickThreads) {
    const int t = k / npairs, p = k % npairs;
    const float* x = (t ? a.burst1 : a.burst0) + (size_t)(skip + 2 * p) * bl;
    const float* y = x + bl;
    double s = 0.0;
    for (int i = 0; i < bl; i++) s += fabs((double)x[i] + (double)y[i]);
    pair_mean[t][p] = s / bl;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m[2];
    for (int t = 0; t < 2; t++) {
      double total = 0.0;
      for (int p = 0; p < npairs; p++) total += pair_mean[t][p];
      m[t] = npairs > 0 ? total / npairs : 1e9;
    }
    det = (m[1] < m[0]) ? 1 : 0;
    *a.pick = det;
  }
  __syncthreads();
  for (int f = threadIdx.x; f < a.fields; f += kPickThreads) a.track[f] = (f & 1) ? (1 - det) : det;
}

}  // namespace

void launch_track_pick(const TrackPickArgs& a, cudaStream_t st) {
  launch_chained(track_pick_kernel, dim3(1), dim3(kPickThreads), 0, st, a);
}

namespace {
template <class S>
void prefilter_launch(const S& src, const ChromaArgs& a, int portions, int max_tiles, cudaStream_t st) {
  const size_t smem = sizeof(float2) * fft_pad(Design::kNc);
  dim3 grid((a.spp + 2 * a.c_out - 1) / (2 * a.c_out), max_tiles, portions);
  auto go = [&](auto kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    launch_chained(kernel, grid, dim3(kThreadsC), smem, st, src);
  };
  if (a.in_fmt == kInS16) go(prefilter_kernel<kInS16, S>);
  else if (a.in_fmt == kInU16) go(prefilter_kernel<kInU16, S>);
  else go(prefilter_kernel<kInU8, S>);
}

template <class S>
void lines_launch(const S& src, const ChromaArgs& a, int portions, int line0, int nlines, int max_lines,
                  bool write_output, cudaStream_t st) {
  if (max_lines <= 0) return;
  const int pairs = (max_lines + 1) / 2;
  auto go = [&](auto kernel, int per_cta, int threads) {
    // the largest shared-memory carveout, so that the register limit sets the CTAs per SM
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    launch_chained(kernel, dim3((pairs + per_cta - 1) / per_cta, 1, portions), dim3(threads), 0, st, src, line0,
                   nlines, write_output ? 1 : 0);
  };
  if (a.line_fft == 2048) go(lines_kernel<2048, S>, line_pairs<2048>(), line_threads<2048>());
  else go(lines_kernel<1024, S>, line_pairs<1024>(), line_threads<1024>());
}

template <class S>
void metric_launch(const S& src, const ChromaArgs& a, int portions, int field0, int nfields, int max_fields,
                   cudaStream_t st) {
  if (max_fields <= 0) return;
  auto go = [&](auto kernel) {
    launch_chained(kernel, dim3(max_fields, 1, portions), dim3(kMetricThreads), 0, st, src, field0, nfields);
  };
  if (a.burst_len == 36) go(metric_kernel<36, S>);
  else if (a.burst_len == 40) go(metric_kernel<40, S>);
  else go(metric_kernel<0, S>);
}
}  // namespace

void launch_chroma_prefilter(const ChromaArgs& a, cudaStream_t st) {
  prefilter_launch(ArgsOne<ChromaArgs>{a}, a, 1, a.fields, st);
}

void launch_chroma_lines(const ChromaArgs& a, int field0, int nfields, bool write_output, cudaStream_t st) {
  const int nlines = nfields * a.out_h;
  lines_launch(ArgsOne<ChromaArgs>{a}, a, 1, field0 * a.out_h, nlines, nlines, write_output, st);
}

void launch_burst_metric(const ChromaArgs& a, int field0, int nfields, cudaStream_t st) {
  metric_launch(ArgsOne<ChromaArgs>{a}, a, 1, field0, nfields, nfields, st);
}

void launch_chroma_prefilter_many(const ArgsMany<ChromaArgs>& p, int portions, int max_tiles, cudaStream_t st) {
  if (portions > 0) prefilter_launch(p, p.a[0], portions, max_tiles, st);
}

void launch_chroma_lines_many(const ArgsMany<ChromaArgs>& p, int portions, int nfields, int max_fields,
                              bool write_output, cudaStream_t st) {
  if (portions <= 0) return;
  const ChromaArgs& a = p.a[0];
  if (nfields < 0) lines_launch(p, a, portions, 0, -1, max_fields * a.out_h, write_output, st);
  else lines_launch(p, a, portions, 0, nfields * a.out_h, nfields * a.out_h, write_output, st);
}

void launch_burst_metric_many(const ArgsMany<ChromaArgs>& p, int portions, int max_fields, cudaStream_t st) {
  if (portions > 0) metric_launch(p, p.a[0], portions, 0, -1, max_fields, st);
}

}  // namespace cuvhs
