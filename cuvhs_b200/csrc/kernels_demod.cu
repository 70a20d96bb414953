// FM demodulation kernels (reference stage K1, src/pipeline/fm_demod.cu:396-485)
// and the sync-threshold edge finder (replaces the per-field serial scans of
// src/pipeline/vsync_discover.cu:5-45 and src/pipeline/sync_pulses.cu:10-58).
//
// Each tile f of the reference covers chunk samples [f*spp - 2048, f*spp - 2048 + tile)
// (clamped to the chunk) and is filtered circularly.  A CTA here computes two
// adjacent runs of one tile's outputs: gather both block windows (mod tile,
// clamped) as the real and imaginary parts of one input, forward FFT,
// separate and multiply by the block spectrum of the truncated kernel,
// inverse FFT per block, emit the valid middles.  HBM traffic is the stage interface only: K1a reads u8 and writes the
// FP32 demod and envelope; K1b reads the demod and writes video and sync.
#include <cuda_runtime.h>

#include "chain.cuh"
#include "cuvhs_internal.h"
#include "raw_input.cuh"
#include "reg_fft.cuh"

namespace cuvhs {
namespace {

constexpr int kThreadsA = Design::kNa / 16;
constexpr int kThreadsB = Design::kNb / 16;

__device__ __forceinline__ int wrap_tile(int q, int tile) {
  return q < 0 ? q + tile : (q >= tile ? q - tile : q);
}

// Both demod stages filter a real signal with a complex kernel g, so one CTA
// takes two adjacent blocks x1, x2 of a tile in one forward transform of
// u = x1 + i*x2.  With m = -k mod N, X1[k] = (U[k] + conj(U[m]))/2 and
// X2[k] = (U[k] - conj(U[m]))/2i, so Z1 = X1*g and Z2 = X2*g follow from U and
// its mirror (g is stored halved); each is inverted on its own.  Three
// transforms serve two blocks instead of four.  ONE_SIDED (the analytic-signal
// kernel of K1a, whose tile response is zero at negative frequencies) skips
// bins k >= N/2: they are not formed and enter the inverse as zeros, which
// also prunes the inverse's first pass.
//
// On return v holds Z1 (RegFFT layout) and sA holds Z2 in natural order; sB
// is free once the caller's next barrier has passed.
template <int N, bool ONE_SIDED>
__device__ __forceinline__ void pair_spectra(float2 (&v)[16], float2* sA, float2* sB, const float2* __restrict__ g,
                                             const float2* __restrict__ tw, int t) {
  constexpr int T = N / 16;
  RegFFT<N>::template run<false>(v, sA, tw, t);
#pragma unroll
  for (int q = 0; q < 16; q++) sB[pidx(t + T * q)] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 16; q++) {
    if (ONE_SIDED && q >= 8) {
      v[q] = make_float2(0.0f, 0.0f);  // k >= N/2: the kernel passes no negative frequencies
      continue;
    }
    const int k = t + T * q;
    const float2 um = sB[pidx((N - k) & (N - 1))];
    const float2 u = v[q];
    const float2 gg = __ldg(&g[k]);
    const float2 x1 = make_float2(u.x + um.x, u.y - um.y);
    const float2 x2 = make_float2(u.y + um.y, um.x - u.x);
    v[q] = make_float2(x1.x * gg.x - x1.y * gg.y, x1.x * gg.y + x1.y * gg.x);
    sA[pidx(k)] = make_float2(x2.x * gg.x - x2.y * gg.y, x2.x * gg.y + x2.y * gg.x);
  }
}

// Z2 back from sA into the RegFFT layout (slots q >= 8 are zero when ONE_SIDED).
template <int N, bool ONE_SIDED>
__device__ __forceinline__ void load_second(float2 (&v)[16], const float2* sA, int t) {
  constexpr int T = N / 16;
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = (ONE_SIDED && q >= 8) ? make_float2(0.0f, 0.0f) : sA[pidx(t + T * q)];
}

// Angle of (x, y) in [-pi, pi], the phase step of K1a: octant reduction to
// t = min(|x|, |y|) / max(|x|, |y|) in [0, 1], then atan(t) = t + t^3 Q(t^2)
// with Q a degree-7 polynomial fitted for this kernel (least squares
// reweighted to minimax on [0, 1]; within 1.7 ulp of atan in FP32), and the
// octant restored.  About half the instructions of a library atan2 and within
// a few FP32 ulp of the angle: a few hundredths of a hertz of demodulated
// frequency, below the FP32 rounding of the stage.
__device__ __forceinline__ float phase_angle(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  const float t = mx > 0.0f ? __fdividef(mn, mx) : 0.0f;
  const float s = t * t;
  float q = 0.00262222f;
  q = fmaf(q, s, -0.01513242f);
  q = fmaf(q, s, 0.04112168f);
  q = fmaf(q, s, -0.07366692f);
  q = fmaf(q, s, 0.10573926f);
  q = fmaf(q, s, -0.14185974f);
  q = fmaf(q, s, 0.19990396f);
  q = fmaf(q, s, -0.33332986f);
  float r = fmaf(t * s, q, t);
  if (ay > ax) r = 1.57079632679489662f - r;
  if (x < 0.0f) r = 3.14159265358979324f - r;
  return copysignf(r, y);
}

// K1a output stage for one block: phase step (FP32 Hz, relative to ire0) and
// envelope of outputs [j0, j0 + nout) of tile f, and the block's envelope sum.
// z (thread t, slot q) is block sample t + T*q; its predecessor is held by
// thread t-1 (same q), or for t = 0 by thread T-1 at q-1.
template <int T>
__device__ __forceinline__ void k1a_emit(const DemodArgs& a, const float2 (&z)[16], int f, int j0, int block,
                                         float2 (*warp_last)[16], double* red, int t) {
  const int lane = t & 31, warp = t >> 5;
  if (lane == 31) {
#pragma unroll
    for (int q = 0; q < 16; q++) warp_last[warp][q] = z[q];
  }
  __syncthreads();
  const int nout = min(a.a_out, kOverlap + a.spp - j0);
  float* dem_out = a.dem + (f * a.spp + (j0 - kOverlap));
  float* env_out = a.env + (f * a.spp + (j0 - kOverlap));
  double esum = 0.0;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    float2 zp;
    zp.x = __shfl_up_sync(0xffffffffu, z[q].x, 1);
    zp.y = __shfl_up_sync(0xffffffffu, z[q].y, 1);
    if (lane == 0) zp = warp > 0 ? warp_last[warp - 1][q] : (q > 0 ? warp_last[T / 32 - 1][q - 1] : z[q]);
    const int i = t + T * q - (a.a_pos + 1);
    if (i >= 0 && i < nout) {
      const float2 zz = z[q];
      // z * conj(zp) rotated by the nominal step, so atan2 sees a small angle
      const float re0 = zz.x * zp.x + zz.y * zp.y;
      const float im0 = zz.y * zp.x - zz.x * zp.y;
      const float re = re0 * a.rot_re - im0 * a.rot_im;
      const float im = re0 * a.rot_im + im0 * a.rot_re;
      float r = phase_angle(im, re);
      // keep the un-rotated step in (-pi, pi] as the reference's wrap does
      if (r + a.d0 > 3.14159265358979f) r -= 6.28318530717959f;
      dem_out[i] = r * a.demod_scale + a.demod_offset;
      const float e = sqrtf(zz.x * zz.x + zz.y * zz.y);
      env_out[i] = e;
      esum += (double)e;
    }
  }
  // Deterministic per-block envelope partial sums (the dropout stage needs
  // the tile mean).
  for (int off = 16; off > 0; off >>= 1) esum += __shfl_down_sync(0xffffffffu, esum, off);
  if (lane == 0) red[warp] = esum;
  __syncthreads();
  if (t == 0) {
    double sacc = 0.0;
    for (int w = 0; w < T / 32; w++) sacc += red[w];
    a.env_part[(size_t)f * a.env_blocks + block] = sacc;
  }
}

// K1a: u8 -> analytic signal -> phase step + envelope, blocks 2x and 2x+1 of
// the tile (the second may lie past the tile's end).
template <int FMT, class Src>
__global__ void __launch_bounds__(kThreadsA, 3) k1a_kernel(const __grid_constant__ Src src, int f_begin) {
  constexpr int N = Design::kNa, T = kThreadsA;
  const DemodArgs& a = src.get();
  if (f_begin + (int)blockIdx.y >= a.tiles) return;  // whole CTA: a batched capture with fewer tiles
  chain_wait();
  extern __shared__ float2 sm[];
  float2* sA = sm;
  float2* sB = sm + fft_pad(N);
  __shared__ float2 warp_last[T / 32][16];
  __shared__ double red[T / 32];
  const int t = threadIdx.x;
  const int f = f_begin + blockIdx.y;
  const int blk0 = 2 * blockIdx.x;
  const int j0 = kOverlap + blk0 * a.a_out;  // first demod output of block 0 (tile position)
  // chunk positions fit in 32 bits (the batch is capped so T * spp < 2^31)
  const int tile0 = f * a.spp - kOverlap;    // chunk position of tile position 0
  const int last = (int)a.total - 1;
  const int base = j0 - 1 - a.a_pos;         // tile position of block-0 sample 0
  float2 v[16];
  // Interior windows (no wrap inside the tile, no clamp at the chunk ends)
  // take the direct addresses; the CTA-uniform test keeps the loop branch-free.
  const int span = a.a_out + N;  // tile positions [base, base + span) are read
  const float dc = a.dc ? *a.dc : 0.0f;
  if (base >= 0 && base + span <= a.tile && tile0 + base >= 0 && tile0 + base + span - 1 <= last &&
      tile0 + base + span <= a.n_read) {
    const int p = tile0 + base + t;
#pragma unroll
    for (int q = 0; q < 16; q++)
      v[q] = make_float2(raw_convert<FMT>(a.raw, p + T * q) - dc, raw_convert<FMT>(a.raw, p + T * q + a.a_out) - dc);
  } else {
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int q0 = base + t + T * q;
      const int p0 = min(max(tile0 + wrap_tile(q0, a.tile), 0), last);
      const int p1 = min(max(tile0 + wrap_tile(q0 + a.a_out, a.tile), 0), last);
      v[q] = make_float2(raw_sample<FMT>(a.raw, p0, a.n_read, dc), raw_sample<FMT>(a.raw, p1, a.n_read, dc));
    }
  }
  pair_spectra<N, true>(v, sA, sB, a.ga, a.tw_a, t);
  // one copy of the inverse transform and output stage serves both blocks
  // (a rolled loop keeps the kernel body small for the instruction cache)
#pragma unroll 1
  for (int b = 0; b < 2; b++) {
    if (b == 1) {
      if (blk0 + 1 >= a.env_blocks) return;  // whole CTA
      load_second<N, true>(v, sA, t);
    }
    RegFFT<N>::run<true>(v, b == 0 ? sB : sA, a.tw_a_inv, t);
    k1a_emit<T>(a, v, f, j0 + b * a.a_out, blk0 + b, warp_last, red, t);
  }
}

// K1b output stage: video (real part) and sync (imaginary part) of one block.
// Sync samples within guard_hz of the pulse threshold are listed for the FP64
// re-evaluation (kernels_guard.cu); a handful per field.
template <int T>
__device__ __forceinline__ void k1b_emit(const DemodArgs& a, const float2 (&z)[16], int f, int j0, int t) {
  const int nout = min(a.b_out, kOverlap + a.spp - j0);
  const int out0 = f * a.spp + (j0 - kOverlap);
  float* video_out = a.video + out0;
  float* sync_out = a.sync + out0;
  const int lane = t & 31;
  // slot q's 32 consecutive positions (one per lane) as an in-pulse word:
  // lane q keeps slot q's ballot, and after the loop lanes 0..15 OR their
  // words into the (at most two) bit words each straddles, in parallel
  unsigned mine = 0;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int i = t + T * q - a.b_pos;
    bool in = false;
    if (i >= 0 && i < nout) {
      video_out[i] = z[q].x + a.corr_video;
      const float sv = z[q].y + a.corr_sync;
      sync_out[i] = sv;
      in = sv <= a.thr_rel;
      if (fabsf(sv - a.thr_rel) < a.guard_hz && a.guard_list) {
        const int slot = atomicAdd(a.guard_count, 1);
        if (slot < a.guard_cap) {
          a.guard_list[slot] = (unsigned)(out0 + i);
        }
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, in);
    mine = lane == q ? m : mine;
  }
  if (a.pulse_bits && mine) {  // only lanes 0..15 hold a word
    long long p0 = (long long)out0 + (t - lane) + (long long)T * lane - a.b_pos;
    if (p0 < 0) {  // positions before the chunk start hold no bits
      mine >>= (int)(-p0);
      p0 = 0;
    }
    const long long w = p0 >> 5;
    const int sh = (int)(p0 & 31);
    atomicOr(&a.pulse_bits[w], mine << sh);
    if (sh && (mine >> (32 - sh))) atomicOr(&a.pulse_bits[w + 1], mine >> (32 - sh));
  }
}

// K1b: demod -> video + sync, blocks 2x and 2x+1 of the tile.
template <class Src>
__global__ void __launch_bounds__(kThreadsB, 1) k1b_kernel(const __grid_constant__ Src src, int f_begin) {
  constexpr int N = Design::kNb, T = kThreadsB;
  const DemodArgs& a = src.get();
  if (f_begin + (int)blockIdx.y >= a.tiles) return;  // whole CTA
  chain_wait();
  extern __shared__ float2 sm[];
  float2* sA = sm;
  float2* sB = sm + fft_pad(N);
  const int t = threadIdx.x;
  const int f = f_begin + blockIdx.y;
  const int blk0 = 2 * blockIdx.x;
  const int j0 = kOverlap + blk0 * a.b_out;
  const int tile0 = f * a.spp - kOverlap;
  const int last = (int)a.total - 1;
  const int base = j0 - a.b_pos;
  float2 v[16];
  const int span = a.b_out + N;  // tile positions [base, base + span) are read
  if (base >= 0 && base + span <= a.tile && tile0 + base >= 0 && tile0 + base + span - 1 <= last) {
    // interior: no wrap inside the tile, no clamp at the chunk ends
    const float* p = a.dem + (tile0 + base + t);
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = make_float2(__ldg(p + T * q), __ldg(p + T * q + a.b_out));
  } else {
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int q0 = base + t + T * q;
      const int p0 = min(max(tile0 + wrap_tile(q0, a.tile), 0), last);
      const int p1 = min(max(tile0 + wrap_tile(q0 + a.b_out, a.tile), 0), last);
      v[q] = make_float2(__ldg(&a.dem[p0]), __ldg(&a.dem[p1]));
    }
  }
  pair_spectra<N, false>(v, sA, sB, a.gb, a.tw_b, t);
  // both blocks' inverses in lockstep (sB and sA as their buffers)
  float2 v2[16];
  __syncthreads();  // Z2 complete in sA
  load_second<N, false>(v2, sA, t);
  RegFFT<N>::run2<true>(v, sB, v2, sA, a.tw_b_inv, opaque_index(t));
  k1b_emit<T>(a, v, f, j0, t);
  if (kOverlap + (blk0 + 1) * a.b_out >= kOverlap + a.spp) return;  // the second block lies past the tile
  k1b_emit<T>(a, v2, f, j0 + a.b_out, t);
}

// Threshold edges in sample order.  Each thread owns 16 consecutive samples
// (one 64-byte line), a CTA 4096.  The count pass reads the signal once and
// keeps each thread's 16-bit falling / rising masks; one scan turns the
// per-CTA counts into offsets; the write pass reads only the masks and writes
// the positions in order, so the host receives sorted edge lists.
constexpr int kEdgeThreads = 256;
constexpr int kEdgePer = 16;
constexpr int kEdgeSeg = kEdgeThreads * kEdgePer;

__device__ __forceinline__ void edge_masks(const float* __restrict__ x, long long total, float thr, long long i0,
                                           unsigned& fm, unsigned& rm) {
  fm = 0;
  rm = 0;
  if (i0 >= total) return;
  float v[kEdgePer];
  // 16-byte loads where the signal is 16-byte aligned (a batched capture's
  // sync may start at any sample)
  if (i0 + kEdgePer <= total && (reinterpret_cast<uintptr_t>(x) & 15) == 0) {
    const float4* p = reinterpret_cast<const float4*>(x + i0);
#pragma unroll
    for (int q = 0; q < kEdgePer / 4; q++) {
      const float4 t = __ldg(p + q);
      v[4 * q] = t.x;
      v[4 * q + 1] = t.y;
      v[4 * q + 2] = t.z;
      v[4 * q + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < kEdgePer; j++) v[j] = (i0 + j < total) ? __ldg(&x[i0 + j]) : 0.0f;
  }
  bool prev_in = i0 > 0 ? (__ldg(&x[i0 - 1]) <= thr) : false;
#pragma unroll
  for (int j = 0; j < kEdgePer; j++) {
    if (i0 + j >= total) break;
    const bool in = v[j] <= thr;
    if (in && (i0 + j == 0 || !prev_in)) fm |= 1u << j;
    if (!in && i0 + j > 0 && prev_in) rm |= 1u << j;
    prev_in = in;
  }
}

// Block-wide exclusive scan of two counters; returns the block totals.
__device__ __forceinline__ int2 block_scan2(int a, int b, int& pa, int& pb) {
  __shared__ int2 warp_tot[kEdgeThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int sa = a, sb = b;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int ta = __shfl_up_sync(0xffffffffu, sa, off), tb = __shfl_up_sync(0xffffffffu, sb, off);
    if (lane >= off) {
      sa += ta;
      sb += tb;
    }
  }
  if (lane == 31) warp_tot[warp] = make_int2(sa, sb);
  __syncthreads();
  int ba = 0, bb = 0, ta = 0, tb = 0;
  for (int w = 0; w < kEdgeThreads / 32; w++) {
    if (w < warp) {
      ba += warp_tot[w].x;
      bb += warp_tot[w].y;
    }
    ta += warp_tot[w].x;
    tb += warp_tot[w].y;
  }
  pa = ba + sa - a;
  pb = bb + sb - b;
  return make_int2(ta, tb);
}

__global__ void __launch_bounds__(kEdgeThreads) edge_count_kernel(const float* __restrict__ x, long long total,
                                                                  float thr, int2* __restrict__ blk,
                                                                  unsigned* __restrict__ masks) {
  chain_wait();
  const long long i0 = (long long)blockIdx.x * kEdgeSeg + (long long)threadIdx.x * kEdgePer;
  unsigned fm, rm;
  edge_masks(x, total, thr, i0, fm, rm);
  masks[(size_t)blockIdx.x * kEdgeThreads + threadIdx.x] = fm | (rm << 16);
  int pa, pb;
  const int2 t = block_scan2(__popc(fm), __popc(rm), pa, pb);
  if (threadIdx.x == 0) blk[blockIdx.x] = t;
}

// One CTA: exclusive scan of the per-CTA counts in place, totals to
// counts[0..1].  Thread t sums a contiguous run of ceil(nblk / 1024) counts,
// the runs' totals are scanned with warp shuffles, then each thread writes its
// run's offsets.
constexpr int kScanThreads = 1024;
__device__ __forceinline__ void scan_blocks(int2* __restrict__ blk, int nblk, int* __restrict__ counts) {
  __shared__ int2 warp_tot[kScanThreads / 32];
  chain_wait();
  const int per = (nblk + kScanThreads - 1) / kScanThreads;
  const int b0 = min(nblk, (int)threadIdx.x * per), b1 = min(nblk, b0 + per);
  int sa = 0, sb = 0;
  for (int b = b0; b < b1; b++) {
    const int2 v = blk[b];
    sa += v.x;
    sb += v.y;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int ia = sa, ib = sb;  // inclusive within the warp
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int ta = __shfl_up_sync(0xffffffffu, ia, off), tb = __shfl_up_sync(0xffffffffu, ib, off);
    if (lane >= off) {
      ia += ta;
      ib += tb;
    }
  }
  if (lane == 31) warp_tot[warp] = make_int2(ia, ib);
  __syncthreads();
  if (warp == 0) {
    int wa = warp_tot[lane].x, wb = warp_tot[lane].y;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int ta = __shfl_up_sync(0xffffffffu, wa, off), tb = __shfl_up_sync(0xffffffffu, wb, off);
      if (lane >= off) {
        wa += ta;
        wb += tb;
      }
    }
    warp_tot[lane] = make_int2(wa, wb);  // inclusive over warps
  }
  __syncthreads();
  int ca = ia - sa, cb = ib - sb;  // exclusive start of this thread's run
  if (warp > 0) {
    ca += warp_tot[warp - 1].x;
    cb += warp_tot[warp - 1].y;
  }
  for (int b = b0; b < b1; b++) {
    const int2 v = blk[b];
    blk[b] = make_int2(ca, cb);
    ca += v.x;
    cb += v.y;
  }
  if (threadIdx.x == 0) {
    counts[0] = warp_tot[kScanThreads / 32 - 1].x;
    counts[1] = warp_tot[kScanThreads / 32 - 1].y;
  }
}


__global__ void __launch_bounds__(kScanThreads) edge_scan_kernel(int2* __restrict__ blk, int nblk,
                                                                 int* __restrict__ counts) {
  scan_blocks(blk, nblk, counts);
}

__global__ void __launch_bounds__(kEdgeThreads) edge_write_kernel(long long total, const unsigned* __restrict__ masks,
                                                                  const int2* __restrict__ blk,
                                                                  unsigned* __restrict__ fall,
                                                                  unsigned* __restrict__ rise, int cap) {
  chain_wait();
  const long long i0 = (long long)blockIdx.x * kEdgeSeg + (long long)threadIdx.x * kEdgePer;
  const unsigned m = __ldg(&masks[(size_t)blockIdx.x * kEdgeThreads + threadIdx.x]);
  unsigned fm = m & 0xFFFFu, rm = m >> 16;
  (void)total;
  int pa, pb;
  block_scan2(__popc(fm), __popc(rm), pa, pb);
  int kf = blk[blockIdx.x].x + pa, kr = blk[blockIdx.x].y + pb;
  while (fm) {
    const int j = __ffs(fm) - 1;
    fm &= fm - 1;
    if (kf < cap) fall[kf] = (unsigned)(i0 + j);
    kf++;
  }
  while (rm) {
    const int j = __ffs(rm) - 1;
    rm &= rm - 1;
    if (kr < cap) rise[kr] = (unsigned)(i0 + j);
    kr++;
  }
}

// Threshold edges from in-pulse bits: one thread per 32-position word (a CTA
// 8192 positions).  falling = in now and not before, rising = out now and in
// before; position 0 counts as preceded by "out" (a pulse open there falls
// there), positions at or past total hold no bits.
constexpr int kBitEdgeSeg = kEdgeThreads * 32;

__device__ __forceinline__ void bit_edges(const unsigned* __restrict__ bits, long long total, long long w,
                                          unsigned& fm, unsigned& rm) {
  const long long p0 = w * 32;
  fm = rm = 0;
  if (p0 >= total) return;
  const unsigned valid = total - p0 >= 32 ? 0xffffffffu : ((1u << (unsigned)(total - p0)) - 1u);
  const unsigned in = __ldg(&bits[w]) & valid;
  const unsigned prev = w > 0 ? (__ldg(&bits[w - 1]) >> 31) : 0u;
  const unsigned before = (in << 1) | prev;  // bit j: in at position j - 1
  fm = in & ~before;
  rm = ~in & before & valid;
}

template <class Src>
__global__ void __launch_bounds__(kEdgeThreads) edge_bits_count_kernel(const __grid_constant__ Src src) {
  const EdgeArgs& e = src.get();
  if ((long long)blockIdx.x * kBitEdgeSeg >= e.total) return;  // whole CTA
  chain_wait();
  const long long w = (long long)blockIdx.x * kEdgeThreads + threadIdx.x;
  unsigned fm, rm;
  bit_edges(e.bits, e.total, w, fm, rm);
  int pa, pb;
  const int2 tot = block_scan2(__popc(fm), __popc(rm), pa, pb);
  if (threadIdx.x == 0) e.blk[blockIdx.x] = tot;
}

template <class Src>
__global__ void __launch_bounds__(kScanThreads) edge_bits_scan_kernel(const __grid_constant__ Src src) {
  const EdgeArgs& e = src.get();
  scan_blocks(e.blk, (int)((e.total + kBitEdgeSeg - 1) / kBitEdgeSeg), e.counts);
}

template <class Src>
__global__ void __launch_bounds__(kEdgeThreads) edge_bits_write_kernel(const __grid_constant__ Src src) {
  const EdgeArgs& e = src.get();
  if ((long long)blockIdx.x * kBitEdgeSeg >= e.total) return;  // whole CTA
  chain_wait();
  const long long w = (long long)blockIdx.x * kEdgeThreads + threadIdx.x;
  unsigned fm, rm;
  bit_edges(e.bits, e.total, w, fm, rm);
  int pa, pb;
  block_scan2(__popc(fm), __popc(rm), pa, pb);
  int kf = e.blk[blockIdx.x].x + pa, kr = e.blk[blockIdx.x].y + pb;
  const long long p0 = w * 32;
  while (fm) {
    const int j = __ffs(fm) - 1;
    fm &= fm - 1;
    if (kf < e.cap) e.fall[kf] = (unsigned)(p0 + j);
    kf++;
  }
  while (rm) {
    const int j = __ffs(rm) - 1;
    rm &= rm - 1;
    if (kr < e.cap) e.rise[kr] = (unsigned)(p0 + j);
    kr++;
  }
}

}  // namespace

size_t pulse_bit_words(long long total) { return (size_t)((total + 31) / 32) + 1; }

void launch_edges_bits(const unsigned* bits, long long total, unsigned* fall, unsigned* rise, int* counts, int cap,
                       int2* blk, cudaStream_t st) {
  const int nblk = (int)((total + kBitEdgeSeg - 1) / kBitEdgeSeg);
  if (nblk <= 0) return;
  ArgsOne<EdgeArgs> e;
  e.a[0].bits = bits;
  e.a[0].total = total;
  e.a[0].blk = blk;
  e.a[0].counts = counts;
  e.a[0].fall = fall;
  e.a[0].rise = rise;
  e.a[0].cap = cap;
  using S = ArgsOne<EdgeArgs>;
  launch_chained(edge_bits_count_kernel<S>, dim3(nblk), dim3(kEdgeThreads), 0, st, e);
  launch_chained(edge_bits_scan_kernel<S>, dim3(1), dim3(kScanThreads), 0, st, e);
  launch_chained(edge_bits_write_kernel<S>, dim3(nblk), dim3(kEdgeThreads), 0, st, e);
}

void launch_edges_bits_many(const ArgsMany<EdgeArgs>& e, int portions, long long max_total, cudaStream_t st) {
  const int nblk = (int)((max_total + kBitEdgeSeg - 1) / kBitEdgeSeg);
  if (nblk <= 0 || portions <= 0) return;
  using S = ArgsMany<EdgeArgs>;
  launch_chained(edge_bits_count_kernel<S>, dim3(nblk, 1, portions), dim3(kEdgeThreads), 0, st, e);
  launch_chained(edge_bits_scan_kernel<S>, dim3(1, 1, portions), dim3(kScanThreads), 0, st, e);
  launch_chained(edge_bits_write_kernel<S>, dim3(nblk, 1, portions), dim3(kEdgeThreads), 0, st, e);
}

void launch_k1a(const DemodArgs& a, int f0, int nf, cudaStream_t st) {
  if (nf <= 0) return;
  const size_t smem = 2 * sizeof(float2) * fft_pad(Design::kNa);
  const int blocks = (a.spp + a.a_out - 1) / a.a_out;  // = env_blocks
  dim3 grid((blocks + 1) / 2, nf);
  const ArgsOne<DemodArgs> src{a};
  auto go = [&](auto kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    launch_chained(kernel, grid, dim3(kThreadsA), smem, st, src, f0);
  };
  using S = ArgsOne<DemodArgs>;
  if (a.in_fmt == kInS16) go(k1a_kernel<kInS16, S>);
  else if (a.in_fmt == kInU16) go(k1a_kernel<kInU16, S>);
  else go(k1a_kernel<kInU8, S>);
}

void launch_k1a_many(const ArgsMany<DemodArgs>& p, int portions, int max_tiles, cudaStream_t st) {
  if (portions <= 0 || max_tiles <= 0) return;
  const DemodArgs& a = p.a[0];  // the design constants every capture of a round shares
  const size_t smem = 2 * sizeof(float2) * fft_pad(Design::kNa);
  const int blocks = (a.spp + a.a_out - 1) / a.a_out;
  dim3 grid((blocks + 1) / 2, max_tiles, portions);
  auto go = [&](auto kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    launch_chained(kernel, grid, dim3(kThreadsA), smem, st, p, 0);
  };
  using S = ArgsMany<DemodArgs>;
  if (a.in_fmt == kInS16) go(k1a_kernel<kInS16, S>);
  else if (a.in_fmt == kInU16) go(k1a_kernel<kInU16, S>);
  else go(k1a_kernel<kInU8, S>);
}

namespace {

// Sum of the converted samples as a 64-bit integer (every converted value is
// an integer, so the sum is exact and order-free).
template <int FMT>
__global__ void dc_sum_kernel(const uint8_t* raw, int n, unsigned long long* sum) {
  __shared__ long long part[8];
  long long acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc += (long long)raw_convert<FMT>(raw, i);
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += part[w];
    atomicAdd(sum, (unsigned long long)s);
  }
}

__global__ void dc_mean_kernel(const unsigned long long* sum, int n, float* dc) {
  *dc = (float)((double)(long long)*sum / (double)n);
}

}  // namespace

void launch_dc_mean(const uint8_t* raw, int n, int in_fmt, unsigned long long* sum, float* dc, cudaStream_t st) {
  cudaMemsetAsync(sum, 0, sizeof(unsigned long long), st);
  const int threads = 256, blocks = 148 * 8;
  if (n > 0) {
    if (in_fmt == kInS16) dc_sum_kernel<kInS16><<<blocks, threads, 0, st>>>(raw, n, sum);
    else if (in_fmt == kInU16) dc_sum_kernel<kInU16><<<blocks, threads, 0, st>>>(raw, n, sum);
    else dc_sum_kernel<kInU8><<<blocks, threads, 0, st>>>(raw, n, sum);
  }
  dc_mean_kernel<<<1, 1, 0, st>>>(sum, n > 0 ? n : 1, dc);
}

void launch_k1b(const DemodArgs& a, int f0, int nf, cudaStream_t st) {
  if (nf <= 0) return;
  const size_t smem = 2 * sizeof(float2) * fft_pad(Design::kNb);
  using S = ArgsOne<DemodArgs>;
  cudaFuncSetAttribute(k1b_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int blocks = (a.spp + a.b_out - 1) / a.b_out;
  dim3 grid((blocks + 1) / 2, nf);
  const S src{a};
  launch_chained(k1b_kernel<S>, grid, dim3(kThreadsB), smem, st, src, f0);
}

void launch_k1b_many(const ArgsMany<DemodArgs>& p, int portions, int max_tiles, cudaStream_t st) {
  if (portions <= 0 || max_tiles <= 0) return;
  const DemodArgs& a = p.a[0];
  const size_t smem = 2 * sizeof(float2) * fft_pad(Design::kNb);
  using S = ArgsMany<DemodArgs>;
  cudaFuncSetAttribute(k1b_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int blocks = (a.spp + a.b_out - 1) / a.b_out;
  dim3 grid((blocks + 1) / 2, max_tiles, portions);
  launch_chained(k1b_kernel<S>, grid, dim3(kThreadsB), smem, st, p, 0);
}

int edge_blocks(long long total) { return (int)((total + kEdgeSeg - 1) / kEdgeSeg); }

size_t edge_mask_words(long long total) { return (size_t)edge_blocks(total) * kEdgeThreads; }

void launch_edges(const float* sync, long long total, float thr_rel, unsigned* fall, unsigned* rise, int* counts,
                  int cap, int2* blk, unsigned* masks, cudaStream_t st) {
  const int nblk = edge_blocks(total);
  if (nblk <= 0) return;
  launch_chained(edge_count_kernel, dim3(nblk), dim3(kEdgeThreads), 0, st, sync, total, thr_rel, blk, masks);
  launch_chained(edge_scan_kernel, dim3(1), dim3(kScanThreads), 0, st, blk, nblk, counts);
  launch_chained(edge_write_kernel, dim3(nblk), dim3(kEdgeThreads), 0, st, total, (const unsigned*)masks,
                 (const int2*)blk, fall, rise, cap);
}

}  // namespace cuvhs
