// Forward and adjoint kernels of the calibration decode model (adjoint.h).
//
// Backward passes recompute what they need from the fixed inputs instead of
// reading stored intermediates: the video is refiltered from the demod, the
// resampling coordinates and carriers are re-evaluated per pixel, and the
// de-emphasis gradient transforms the demod block again next to the video
// gradient.  Per-row and per-block partial sums are written to fixed slots
// and summed on the host in a fixed order; only the video-gradient scatter of
// the luma resampler uses atomics.
#include <cuda_runtime.h>

#include "adjoint.h"
#include "reg_fft.cuh"

namespace cuvhs {
namespace {

constexpr int kN = Design::kNb;
constexpr int kT = kN / 16;
constexpr int kRowThreads = 128;
constexpr int kLineWarps = 4;
// The calibration model is NTSC: 910-sample lines in a 1024-point line
// transform, a 36-sample burst window.
constexpr int kLineFFT = 1024;
constexpr int kBurstLen = 36;

template <int THREADS, int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* sh /* [THREADS/32][K] */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++)
    for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; k++) sh[warp * K + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s = 0.0;
      for (int w = 0; w < THREADS / 32; w++) s += sh[w * K + k];
      v[k] = s;
    }
}

// Catmull-Rom of s at x (the decoder's resampler), its x-derivative and taps.
struct Resample {
  bool ok;
  int ci;
  float v, dv, w[4];
};
__device__ __forceinline__ Resample catmull_rom(const float* __restrict__ s, double x, long long total) {
  Resample r;
  r.ci = (int)x;
  r.ok = r.ci >= 1 && (long long)r.ci + 2 < total;
  if (!r.ok) {
    r.v = r.dv = 0.0f;
    r.w[0] = r.w[1] = r.w[2] = r.w[3] = 0.0f;
    return r;
  }
  const float fr = (float)(x - (double)r.ci);
  const float p0 = __ldg(&s[r.ci - 1]), p1 = __ldg(&s[r.ci]);
  const float p2 = __ldg(&s[r.ci + 1]), p3 = __ldg(&s[r.ci + 2]);
  const float c1 = p2 - p0;
  const float c2 = 2.0f * p0 - 5.0f * p1 + 4.0f * p2 - p3;
  const float c3 = 3.0f * (p1 - p2) + p3 - p0;
  r.v = p1 + 0.5f * fr * (c1 + fr * (c2 + fr * c3));
  r.dv = 0.5f * (c1 + fr * (2.0f * c2 + 3.0f * fr * c3));
  const float f2 = fr * fr, f3 = f2 * fr;
  r.w[0] = 0.5f * (-fr + 2.0f * f2 - f3);
  r.w[1] = 1.0f + 0.5f * (-5.0f * f2 + 3.0f * f3);
  r.w[2] = 0.5f * (fr + 4.0f * f2 - 3.0f * f3);
  r.w[3] = 0.5f * (f3 - f2);
  return r;
}

// Start of row r of field f with its offset.
__device__ __forceinline__ double row_start(const AdjArgs& a, int f, int r) {
  return a.ll[(size_t)f * a.lpf + r] + a.line_off[(size_t)f * (a.out_h + 1) + r];
}

// ------------------------------------------------------------------ video
// Overlap-save over [0, total) with zero padding; the kernel is real, so two
// blocks ride in the real and imaginary parts of one transform.
__global__ void __launch_bounds__(kT, 1) adj_video_kernel(AdjArgs a) {
  extern __shared__ float2 sm[];
  const int t = threadIdx.x;
  const long long j0 = (long long)(2 * blockIdx.x) * a.b_out;
  float2 v[16];
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const long long p0 = j0 - a.b_pos + t + kT * q, p1 = p0 + a.b_out;
    v[q] = make_float2(p0 >= 0 && p0 < a.total ? __ldg(&a.dem[p0]) : 0.0f,
                       p1 >= 0 && p1 < a.total ? __ldg(&a.dem[p1]) : 0.0f);
  }
  RegFFT<kN>::run<false>(v, sm, a.tw_b, t);
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const float2 g = __ldg(&a.gv[t + kT * q]);
    v[q] = make_float2(v[q].x * g.x - v[q].y * g.y, v[q].x * g.y + v[q].y * g.x);
  }
  RegFFT<kN>::run<true>(v, sm, a.tw_b_inv, t);
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int i = t + kT * q - a.b_pos;
    if (i >= 0 && i < a.b_out) {
      const long long p = j0 + i;
      if (p < a.total) a.video[p] = v[q].x;
      if (p + a.b_out < a.total) a.video[p + a.b_out] = v[q].y;
    }
  }
}

// ------------------------------------------------------------------- luma
template <int MODE>
__global__ void __launch_bounds__(kRowThreads) adj_luma_kernel(AdjArgs a) {
  __shared__ double sh[kRowThreads / 32 * 5];
  const int grow = blockIdx.x;
  const int f = grow / a.out_h, r = grow % a.out_h;
  const int W = a.out_w;
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // loss, carrier, deviation, x0, x1
  const bool has_line = r + 1 < a.lpf;
  const bool in_loss = has_line && r >= a.row0 && r < a.row1;
  const double a0 = has_line ? row_start(a, f, r) : 0.0;
  const double span = has_line ? row_start(a, f, r + 1) - a0 : 0.0;
  const double kA = a.luma_gain / a.deviation;
  for (int c = threadIdx.x; c < W; c += kRowThreads) {
    const size_t pix = (size_t)grow * W + c;
    const double fc = __ldg(&a.col_frac[c]);
    Resample s;
    s.ok = false;
    if (has_line) s = catmull_rom(a.video, a0 + fc * span, a.total);
    const double Y = s.ok ? ((double)s.v - a.carrier) * kA + a.luma_offset : 1024.0;
    if (a.y_out) a.y_out[pix] = (float)Y;
    if (!in_loss || !s.ok || c < a.col0 || c >= a.col1) continue;
    const double e = Y - (double)__ldg(&a.tgt_y[pix]);
    acc[0] += e * e;
    if (MODE == 1) {
      const double k = 2.0 * e * a.inv_ny * kA;  // dL/dv
      acc[1] -= k;
      acc[2] -= k * ((double)s.v - a.carrier) / a.deviation;
      const double gx = k * (double)s.dv;
      acc[3] += gx * (1.0 - fc);
      acc[4] += gx * fc;
#pragma unroll
      for (int j = 0; j < 4; j++) atomicAdd(&a.gvideo[s.ci - 1 + j], (float)(k * (double)s.w[j]));
    }
  }
  block_sum<kRowThreads, 5>(acc, sh);
  if (threadIdx.x == 0) {
    double* rp = a.row + (size_t)grow * kAdjRowVals;
    rp[kRowLossY] = acc[0];
    rp[kRowCarrier] = acc[1];
    rp[kRowDeviation] = acc[2];
    rp[kRowLumaX0] = acc[3];
    rp[kRowLumaX1] = acc[4];
  }
}

// ----------------------------------------------------------------- chroma
struct ChromaSample {
  Resample s;
  float het, sn;  // -cos(theta), sin(theta) = d het / d phase
  double fc;
};

__device__ __forceinline__ ChromaSample chroma_sample(const AdjArgs& a, int gl, int c) {
  ChromaSample o;
  const int f = gl / a.out_h, r = gl % a.out_h;
  o.fc = __ldg(&a.col_frac[c]);
  o.s.ok = false;
  o.s.v = o.s.dv = 0.0f;
  o.het = o.sn = 0.0f;
  if (r + 1 >= a.lpf) return o;
  const double a0 = row_start(a, f, r), a1 = row_start(a, f, r + 1);
  o.s = catmull_rom(a.pre, a0 + o.fc * (a1 - a0), a.total);
  const int rot = a.track[f] ? 1 : 3;
  const int lp = (r * rot) & 3;
  const double u = a.het_scale * (double)(r * a.out_w + c);
  const float fr = (float)(u - floor(u));
  const float ph = (float)(a.phase[(size_t)f * a.out_h + r] * (1.0 / 3.14159265358979323846));
  const float arg = 2.0f * fr + 0.5f * (float)lp + ph;
  float sn, cs;
  sincospif(arg, &sn, &cs);
  o.het = -cs;
  o.sn = sn;
  return o;
}

// 1024-point band-pass of the two lines held in sm (real and imaginary parts).
__device__ __forceinline__ void line_bandpass(float2* sm, const AdjArgs& a, int lane) {
  __syncwarp();
  smem_fft<kLineFFT, 32, false>(sm, a.tw_l, lane);
  const int lo = a.fsc_bin - a.bw_bins, hi = a.fsc_bin + a.bw_bins;
  const float scale = 1.0f / (float)kLineFFT;
  for (int k = lane; k < kLineFFT; k += 32) {
    const int kk = k <= kLineFFT / 2 ? k : kLineFFT - k;
    const float m = (kk >= lo && kk <= hi) ? scale : 0.0f;
    const float2 x = sm[pidx(k)];
    sm[pidx(k)] = make_float2(x.x * m, x.y * m);
  }
  __syncwarp();
  smem_fft<kLineFFT, 32, true>(sm, a.tw_l_inv, opaque_index(lane));
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// One warp per pair of chroma lines.  MODE 0: forward; 1: forward + backward.
// Each line's gain is the decoder's ACC, recomputed from the band-passed
// burst at the current parameters (g = ref / rms over the burst window), so
// the backward pass also carries dL/dg back into the burst samples.
template <int MODE>
__global__ void __launch_bounds__(32 * kLineWarps) adj_chroma_kernel(AdjArgs a) {
  __shared__ float2 sm_all[kLineWarps][fft_pad(kLineFFT)];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* sm = sm_all[warp];
  const int nlines = a.fields * a.out_h;
  const int la = 2 * (blockIdx.x * kLineWarps + warp), lb = la + 1;
  if (la >= nlines) return;  // whole warp
  const bool has_b = lb < nlines;
  const int W = a.out_w;
  for (int c = lane; c < kLineFFT; c += 32) {
    float xa = 0.0f, xb = 0.0f;
    if (c < W) {
      const ChromaSample sa = chroma_sample(a, la, c);
      xa = sa.s.v * sa.het;
      if (has_b) {
        const ChromaSample sb = chroma_sample(a, lb, c);
        xb = sb.s.v * sb.het;
      }
    }
    sm[pidx(c)] = make_float2(xa, xb);
  }
  line_bandpass(sm, a, lane);
  // ACC gains from the burst window
  double ssa = 0.0, ssb = 0.0;
  for (int i = lane; i < kBurstLen; i += 32) {
    const float2 v = sm[pidx(a.burst_start + i)];
    ssa += (double)v.x * v.x;
    ssb += (double)v.y * v.y;
  }
  ssa = warp_sum(ssa);
  ssb = warp_sum(ssb);
  const double rms_a = sqrt(ssa / kBurstLen), rms_b = sqrt(ssb / kBurstLen);
  const double ga = rms_a > 1.0 ? (double)a.burst_abs_ref / rms_a : 0.0;
  const double gb = (has_b && rms_b > 1.0) ? (double)a.burst_abs_ref / rms_b : 0.0;
  if (lane == 0) {
    a.gain_out[la] = (float)ga;
    if (has_b) a.gain_out[lb] = (float)gb;
  }
  const int ra = la % a.out_h, rb = lb % a.out_h;
  const bool loss_a = ra >= a.row0 && ra < a.row1 && ra + 1 < a.lpf;
  const bool loss_b = has_b && rb >= a.row0 && rb < a.row1 && rb + 1 < a.lpf;
  double la_loss = 0.0, lb_loss = 0.0, dga = 0.0, dgb = 0.0;
  // dL/dC per column, kept per lane
  constexpr int kPerLane = (kLineFFT + 31) / 32;  // columns per lane (out_w <= kLineFFT)
  float ea[kPerLane], eb[kPerLane];
  int n = 0;
  for (int c = lane; c < W; c += 32, n++) {
    const float2 v = sm[pidx(c)];
    const size_t pa = (size_t)la * W + c, pb = (size_t)lb * W + c;
    const double Ca = ga * (double)v.x + 32768.0, Cb = gb * (double)v.y + 32768.0;
    if (a.c_out) {
      a.c_out[pa] = (float)Ca;
      if (has_b) a.c_out[pb] = (float)Cb;
    }
    const bool col = c >= a.col0 && c < a.col1;
    const double da = loss_a && col ? Ca - (double)__ldg(&a.tgt_c[pa]) : 0.0;
    const double db = loss_b && col ? Cb - (double)__ldg(&a.tgt_c[pb]) : 0.0;
    la_loss += da * da;
    lb_loss += db * db;
    const double gca = 2.0 * da * a.inv_nc, gcb = 2.0 * db * a.inv_nc;
    ea[n] = (float)gca;
    eb[n] = (float)gcb;
    dga += gca * (double)v.x;  // dL/dgain
    dgb += gcb * (double)v.y;
  }
  la_loss = warp_sum(la_loss);
  lb_loss = warp_sum(lb_loss);
  double* rpa = a.row + (size_t)la * kAdjRowVals;
  double* rpb = a.row + (size_t)lb * kAdjRowVals;
  if (lane == 0) {
    rpa[kRowLossC] = la_loss;
    if (has_b) rpb[kRowLossC] = lb_loss;
  }
  if (MODE == 0) return;
  dga = warp_sum(dga);
  dgb = warp_sum(dgb);
  // dL/d(band-passed line) = g dL/dC + dL/dg dg/dbp, with dg/dbp_i = -g bp_i / ss
  // on the burst window
  const double ka = ssa > 0.0 && ga > 0.0 ? -dga * ga / ssa : 0.0;
  const double kb = ssb > 0.0 && gb > 0.0 ? -dgb * gb / ssb : 0.0;
  __syncwarp();
  n = 0;
  for (int c = lane; c < kLineFFT; c += 32) {
    const float2 bp = sm[pidx(c)];
    double ha = 0.0, hb = 0.0;
    if (c < W) {
      ha = ga * (double)ea[n];
      hb = gb * (double)eb[n];
      n++;
    }
    if (c >= a.burst_start && c < a.burst_start + kBurstLen) {
      ha += ka * (double)bp.x;
      hb += kb * (double)bp.y;
    }
    sm[pidx(c)] = make_float2((float)ha, (float)hb);
  }
  line_bandpass(sm, a, lane);  // BP is symmetric: its own adjoint
  double ph_a = 0.0, ph_b = 0.0, x0a = 0.0, x1a = 0.0, x0b = 0.0, x1b = 0.0;
  for (int c = lane; c < W; c += 32) {
    const float2 h = sm[pidx(c)];
    const ChromaSample sa = chroma_sample(a, la, c);
    if (sa.s.ok) {
      ph_a += (double)h.x * (double)sa.s.v * (double)sa.sn;
      const double gx = (double)h.x * (double)sa.het * (double)sa.s.dv;
      x0a += gx * (1.0 - sa.fc);
      x1a += gx * sa.fc;
    }
    if (has_b) {
      const ChromaSample sb = chroma_sample(a, lb, c);
      if (sb.s.ok) {
        ph_b += (double)h.y * (double)sb.s.v * (double)sb.sn;
        const double gx = (double)h.y * (double)sb.het * (double)sb.s.dv;
        x0b += gx * (1.0 - sb.fc);
        x1b += gx * sb.fc;
      }
    }
  }
  ph_a = warp_sum(ph_a);
  x0a = warp_sum(x0a);
  x1a = warp_sum(x1a);
  ph_b = warp_sum(ph_b);
  x0b = warp_sum(x0b);
  x1b = warp_sum(x1b);
  if (lane == 0) {
    rpa[kRowPhase] = ph_a;
    rpa[kRowChromaX0] = x0a;
    rpa[kRowChromaX1] = x1a;
    if (has_b) {
      rpb[kRowPhase] = ph_b;
      rpb[kRowChromaX0] = x0b;
      rpb[kRowChromaX1] = x1b;
    }
  }
}

// ------------------------------------------------------------- de-emphasis
// One CTA per video block: X = FFT(demod window), W = FFT(video gradient on
// the block's outputs, zero elsewhere); dL/dtheta_j = sum_k Re(X[k] dG_j[k]
// conj(W[k])).  The two transforms are separate: the demod (~1e5 Hz with a
// large DC term) and the gradient differ by many orders of magnitude, so
// packing them into one FP32 transform would bury W in X's rounding.
__global__ void __launch_bounds__(kT, 1) adj_deemph_kernel(AdjArgs a) {
  extern __shared__ float2 sm[];
  float2* sx = sm + fft_pad(kN);  // X in natural order
  __shared__ double sh[kT / 32 * 4];
  const int t = threadIdx.x;
  const long long j0 = (long long)blockIdx.x * a.b_out;
  float2 v[16];
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const long long p = j0 - a.b_pos + t + kT * q;
    v[q] = make_float2(p >= 0 && p < a.total ? __ldg(&a.dem[p]) : 0.0f, 0.0f);
  }
  RegFFT<kN>::run<false>(v, sm, a.tw_b, t);
#pragma unroll
  for (int q = 0; q < 16; q++) sx[pidx(t + kT * q)] = v[q];
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int i = t + kT * q - a.b_pos;
    v[q] = make_float2((i >= 0 && i < a.b_out && j0 + i < a.total) ? __ldg(&a.gvideo[j0 + i]) : 0.0f, 0.0f);
  }
  RegFFT<kN>::run<false>(v, sm, a.tw_b, t);  // each thread reads back only its own X slots
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int k = t + kT * q;
    const float2 x = sx[pidx(k)], w = v[q];
    const double pr = (double)x.x * w.x + (double)x.y * w.y;  // X conj(W)
    const double pi = (double)x.y * w.x - (double)x.x * w.y;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float2 d = __ldg(&a.dg[(size_t)j * kN + k]);
      acc[j] += pr * (double)d.x - pi * (double)d.y;
    }
  }
  block_sum<kT, 4>(acc, sh);
  if (t == 0)
#pragma unroll
    for (int j = 0; j < 4; j++) a.blk[(size_t)blockIdx.x * 4 + j] = acc[j];
}

}  // namespace

void launch_adj_video(const AdjArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(float2) * fft_pad(kN);
  cudaFuncSetAttribute(adj_video_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  adj_video_kernel<<<(a.blocks + 1) / 2, kT, smem, st>>>(a);
}

void launch_adj_luma(const AdjArgs& a, int mode, cudaStream_t st) {
  const int rows = a.fields * a.out_h;
  if (mode == 1) adj_luma_kernel<1><<<rows, kRowThreads, 0, st>>>(a);
  else adj_luma_kernel<0><<<rows, kRowThreads, 0, st>>>(a);
}

void launch_adj_chroma(const AdjArgs& a, int mode, cudaStream_t st) {
  const int pairs = (a.fields * a.out_h + 1) / 2;
  const int grid = (pairs + kLineWarps - 1) / kLineWarps;
  if (mode == 1) adj_chroma_kernel<1><<<grid, 32 * kLineWarps, 0, st>>>(a);
  else adj_chroma_kernel<0><<<grid, 32 * kLineWarps, 0, st>>>(a);
}

void launch_adj_deemph(const AdjArgs& a, cudaStream_t st) {
  const size_t smem = 2 * sizeof(float2) * fft_pad(kN);
  cudaFuncSetAttribute(adj_deemph_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  adj_deemph_kernel<<<a.blocks, kT, smem, st>>>(a);
}

}  // namespace cuvhs
