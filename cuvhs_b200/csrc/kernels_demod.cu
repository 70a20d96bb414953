// FM demodulation kernels (reference stage K1, src/pipeline/fm_demod.cu:396-485)
// and the sync-threshold edge finder (replaces the per-field serial scans of
// src/pipeline/vsync_discover.cu:5-45 and src/pipeline/sync_pulses.cu:10-58).
//
// Each tile f of the reference covers chunk samples [f*spp - 2048, f*spp - 2048 + tile)
// (clamped to the chunk) and is filtered circularly.  A CTA here computes a
// contiguous run of one tile's outputs with one shared-memory FFT pair: gather
// the tile window (mod tile, clamped) into shared memory, forward FFT, multiply
// by the block spectrum of the truncated kernel, inverse FFT, emit the valid
// middle.  HBM traffic is the stage interface only: K1a reads u8 and writes the
// FP32 demod and envelope; K1b reads the demod and writes video and sync.
#include <cuda_runtime.h>

#include "cuvhs_internal.h"
#include "smem_fft.cuh"

namespace cuvhs {
namespace {

constexpr int kThreadsA = 256;
constexpr int kThreadsB = 512;

__device__ __forceinline__ int wrap_tile(int q, int tile) {
  return q < 0 ? q + tile : (q >= tile ? q - tile : q);
}
__device__ __forceinline__ long long clamp_ll(long long p, long long total) {
  return p < 0 ? 0 : (p >= total ? total - 1 : p);
}

// K1a: u8 -> analytic signal -> phase step (FP32 Hz, relative to ire0) + envelope.
__global__ void __launch_bounds__(kThreadsA) k1a_kernel(DemodArgs a) {
  constexpr int N = Design::kNa;
  extern __shared__ float2 sm[];
  __shared__ double red[kThreadsA / 32];
  const int f = blockIdx.y;
  const int j0 = kOverlap + blockIdx.x * a.a_out;       // first demod output (tile position)
  const long long tile0 = (long long)f * a.spp - kOverlap;  // chunk position of tile position 0
  const int base = j0 - 1 - a.a_pos;                    // tile position of block sample 0
  for (int t = threadIdx.x; t < N; t += kThreadsA) {
    const int q = wrap_tile(base + t, a.tile);
    const long long p = clamp_ll(tile0 + q, a.total);
    const float v = ((float)a.raw[p] - 128.0f) * 256.0f;
    sm[pidx(t)] = make_float2(v, 0.0f);
  }
  __syncthreads();
  smem_fft<N, kThreadsA, false>(sm, a.tw_a);
  for (int k = threadIdx.x; k < N; k += kThreadsA) {
    const float2 x = sm[pidx(k)], g = __ldg(&a.ga[k]);
    sm[pidx(k)] = make_float2(x.x * g.x - x.y * g.y, x.x * g.y + x.y * g.x);
  }
  __syncthreads();
  smem_fft<N, kThreadsA, true>(sm, a.tw_a);
  const int nout = min(a.a_out, kOverlap + a.spp - j0);
  const size_t o0 = (size_t)f * a.spp + (size_t)(j0 - kOverlap);
  double esum = 0.0;
  for (int i = threadIdx.x; i < nout; i += kThreadsA) {
    const int t = a.a_pos + 1 + i;
    const float2 z = sm[pidx(t)], zp = sm[pidx(t - 1)];
    // z * conj(zp) rotated by the nominal step, so atan2 sees a small angle
    const float re0 = z.x * zp.x + z.y * zp.y;
    const float im0 = z.y * zp.x - z.x * zp.y;
    const float re = re0 * a.rot_re - im0 * a.rot_im;
    const float im = re0 * a.rot_im + im0 * a.rot_re;
    float r = atan2f(im, re);
    // keep the un-rotated step in (-pi, pi] as the reference's wrap does
    if (r + a.d0 > 3.14159265358979f) r -= 6.28318530717959f;
    a.dem[o0 + i] = r * a.demod_scale + a.demod_offset;
    const float e = sqrtf(z.x * z.x + z.y * z.y);
    a.env[o0 + i] = e;
    esum += (double)e;
  }
  // Deterministic per-CTA envelope partial sums (the dropout stage needs the
  // tile mean).
  for (int off = 16; off > 0; off >>= 1) esum += __shfl_down_sync(0xffffffffu, esum, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = esum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kThreadsA / 32; w++) s += red[w];
    a.env_part[(size_t)f * a.env_blocks + blockIdx.x] = s;
  }
}

// K1b: demod -> video (real part) and sync (imag part) in one complex transform.
__global__ void __launch_bounds__(kThreadsB) k1b_kernel(DemodArgs a) {
  constexpr int N = Design::kNb;
  extern __shared__ float2 sm[];
  const int f = blockIdx.y;
  const int j0 = kOverlap + blockIdx.x * a.b_out;
  const long long tile0 = (long long)f * a.spp - kOverlap;
  const int base = j0 - a.b_pos;
  for (int t = threadIdx.x; t < N; t += kThreadsB) {
    const int q = wrap_tile(base + t, a.tile);
    const long long p = clamp_ll(tile0 + q, a.total);
    sm[pidx(t)] = make_float2(__ldg(&a.dem[p]), 0.0f);
  }
  __syncthreads();
  smem_fft<N, kThreadsB, false>(sm, a.tw_b);
  for (int k = threadIdx.x; k < N; k += kThreadsB) {
    const float2 x = sm[pidx(k)], g = __ldg(&a.gb[k]);
    sm[pidx(k)] = make_float2(x.x * g.x - x.y * g.y, x.x * g.y + x.y * g.x);
  }
  __syncthreads();
  smem_fft<N, kThreadsB, true>(sm, a.tw_b);
  const int nout = min(a.b_out, kOverlap + a.spp - j0);
  const size_t o0 = (size_t)f * a.spp + (size_t)(j0 - kOverlap);
  for (int i = threadIdx.x; i < nout; i += kThreadsB) {
    const float2 v = sm[pidx(a.b_pos + i)];
    a.video[o0 + i] = v.x + a.corr_video;
    a.sync[o0 + i] = v.y + a.corr_sync;
  }
}

// Threshold edges.  Positions are chunk-relative sample indices.
__global__ void edges_kernel(const float* __restrict__ x, long long total, float thr, unsigned* __restrict__ fall,
                             unsigned* __restrict__ rise, int* __restrict__ counts, int cap) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool f_edge = false, r_edge = false;
  if (i < total) {
    const float v = __ldg(&x[i]);
    const bool in = v <= thr;
    const bool prev_in = i > 0 ? (__ldg(&x[i - 1]) <= thr) : false;
    f_edge = in && (i == 0 || !prev_in);
    r_edge = !in && i > 0 && prev_in;
  }
  // warp-aggregated appends
  const unsigned mf = __ballot_sync(0xffffffffu, f_edge);
  const unsigned mr = __ballot_sync(0xffffffffu, r_edge);
  const int lane = threadIdx.x & 31;
  int bf = 0, br = 0;
  if (lane == 0) {
    if (mf) bf = atomicAdd(&counts[0], __popc(mf));
    if (mr) br = atomicAdd(&counts[1], __popc(mr));
  }
  bf = __shfl_sync(0xffffffffu, bf, 0);
  br = __shfl_sync(0xffffffffu, br, 0);
  const unsigned below = (1u << lane) - 1u;
  if (f_edge) {
    const int k = bf + __popc(mf & below);
    if (k < cap) fall[k] = (unsigned)i;
  }
  if (r_edge) {
    const int k = br + __popc(mr & below);
    if (k < cap) rise[k] = (unsigned)i;
  }
}

}  // namespace

void launch_k1a(const DemodArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(float2) * fft_pad(Design::kNa);
  dim3 grid((a.spp + a.a_out - 1) / a.a_out, a.tiles);
  k1a_kernel<<<grid, kThreadsA, smem, st>>>(a);
}

void launch_k1b(const DemodArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(float2) * fft_pad(Design::kNb);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k1b_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  dim3 grid((a.spp + a.b_out - 1) / a.b_out, a.tiles);
  k1b_kernel<<<grid, kThreadsB, smem, st>>>(a);
}

void launch_edges(const float* sync, long long total, float thr_rel, unsigned* fall, unsigned* rise, int* counts,
                  int cap, cudaStream_t st) {
  const int threads = 256;
  const long long blocks = (total + threads - 1) / threads;
  edges_kernel<<<(unsigned)blocks, threads, 0, st>>>(sync, total, thr_rel, fall, rise, counts, cap);
}

}  // namespace cuvhs
