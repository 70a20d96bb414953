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
// Work: one CTA per listed sample.  The 2*hb + 1 demod positions the sample's
// sync sum reads split into a few runs -- consecutive chunk positions of one
// owning tile, or one clamped position repeated -- and each run's analytic
// signal is one FP64 overlap-save convolution: its raw window (tile wrap and
// chunk clamp applied per sample) goes through a 4096-point FP64 FFT in shared
// memory, is multiplied by the FFT of the truncated taps and transformed back,
// giving every z of up to 4095 - 2*ha consecutive positions at once.  The
// phase differences fill a demod array indexed like the sync taps, and the
// sync sum is taken in a fixed order, so the result is deterministic.
#include <cuda_runtime.h>

#include <algorithm>

#include "chain.cuh"
#include "cuvhs_internal.h"
#include "raw_input.cuh"

namespace cuvhs {
namespace {

constexpr int kGT = 512;                  // threads per CTA (two CTAs per SM)
constexpr int kN = Design::kGuardN;       // FFT length
constexpr int kBfly = kN / 4 / kGT;       // radix-4 butterflies per thread per pass
constexpr int kTwQ = kN / 4;              // twiddles held in shared memory: exp(-2 pi i k / kN), k < kN / 4
constexpr double kPi64 = 3.14159265358979323846;
constexpr double kTau64 = 2.0 * kPi64;
static_assert(kN == 4096 && kBfly >= 1 && kN / 4 % kGT == 0, "the FFT passes assume 4096 points");

__device__ __forceinline__ long long wrap_pos(long long q, long long tile) {
  return q < 0 ? q + tile : (q >= tile ? q - tile : q);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(-2 pi i j / kN) for j < 3 kN / 4 from the quarter table: the quadrant
// q = j / (kN / 4) multiplies by (-i)^q.
__device__ __forceinline__ double2 twiddle(const double2* tq, int j) {
  const double2 w = tq[j & (kTwQ - 1)];
  switch (j / kTwQ) {
    case 0: return w;
    case 1: return make_double2(w.y, -w.x);
    default: return make_double2(-w.x, -w.y);
  }
}

// In-place radix-4 Stockham FFT of kN points in shared memory (every thread
// holds its butterflies' inputs in registers across a barrier, so one buffer
// serves as source and destination).  tq: the quarter twiddle table; the
// inverse conjugates the twiddles and is unnormalised.
template <bool kInverse>
__device__ void fft_n(double2* buf, const double2* tq) {
  const int t = threadIdx.x;
  for (int ns = 1; ns < kN; ns *= 4) {
    double2 v[kBfly][4];
#pragma unroll
    for (int b = 0; b < kBfly; b++) {
      const int j = t + b * kGT;
#pragma unroll
      for (int r = 0; r < 4; r++) v[b][r] = buf[j + r * (kN / 4)];
    }
    __syncthreads();
    const int stride = kN / (4 * ns);
#pragma unroll
    for (int b = 0; b < kBfly; b++) {
      const int j = t + b * kGT;
      const int k = j & (ns - 1);
#pragma unroll
      for (int r = 1; r < 4; r++) {
        double2 w = twiddle(tq, r * k * stride);
        if (kInverse) w.y = -w.y;
        v[b][r] = cmul(v[b][r], w);
      }
      const double2 a0 = v[b][0], a1 = v[b][1], a2 = v[b][2], a3 = v[b][3];
      const double2 s02 = make_double2(a0.x + a2.x, a0.y + a2.y), d02 = make_double2(a0.x - a2.x, a0.y - a2.y);
      const double2 s13 = make_double2(a1.x + a3.x, a1.y + a3.y), d13 = make_double2(a1.x - a3.x, a1.y - a3.y);
      // forward: X1 = d02 - i d13, X3 = d02 + i d13; the inverse swaps them
      const double2 m = kInverse ? make_double2(-d13.y, d13.x) : make_double2(d13.y, -d13.x);  // -/+ i d13
      const int base = (j / ns) * ns * 4 + k;
      buf[base] = make_double2(s02.x + s13.x, s02.y + s13.y);
      buf[base + ns] = make_double2(d02.x + m.x, d02.y + m.y);
      buf[base + 2 * ns] = make_double2(s02.x - s13.x, s02.y - s13.y);
      buf[base + 3 * ns] = make_double2(d02.x - m.x, d02.y - m.y);
    }
    __syncthreads();
  }
}

// A run of the sample's demod positions: taps kk0..kk1 read chunk position
// c0 + step * (kk - kk0), step -1 (consecutive positions of one owning tile)
// or 0 (one clamped position).
struct Run {
  int kk0, kk1, step;
  long long c0;
};
constexpr int kMaxRuns = 8;

// Phase clocks for inspection (thread 0, first block of a sample only).
__device__ __forceinline__ void phase_clock(const GuardArgs& g, int y, int k) {
  if (g.dbg_clk && threadIdx.x == 0 && y < kGuardClockSamples) g.dbg_clk[(size_t)y * kPhaseSlots + k] = clock64();
}

template <int FMT, class Src>
__global__ void __launch_bounds__(kGT, 2) guard_kernel(const __grid_constant__ Src src) {
  const GuardArgs& g = src.get();
  chain_wait();
  extern __shared__ double2 gsm[];
  double2* buf = gsm;                                        // [kN]
  double2* tq = gsm + kN;                                    // [kTwQ]
  double* dem = reinterpret_cast<double*>(gsm + kN + kTwQ);  // [2 * hb + 1], indexed like the sync taps
  __shared__ Run runs[kMaxRuns];
  __shared__ int nruns, skip;
  __shared__ double red[kGT / 32];
  const int n_listed = min(*g.count, g.cap);
  const int t = threadIdx.x;
  const double dc = g.dc ? (double)*g.dc : 0.0;
  const long long last = g.total - 1;
  const int W = 2 * g.hb + 1;
  const int V = kN - 1 - 2 * g.ha;  // demod positions one FFT block yields
  if ((int)blockIdx.x >= n_listed) return;  // whole CTA
  for (int k = t; k < kTwQ; k += kGT) tq[k] = __ldg(&g.tw[k]);
  __syncthreads();
  for (int y = blockIdx.x; y < n_listed; y += gridDim.x) {
    const long long s = g.list[y];
    const long long f = s / g.spp;
    const long long J = kOverlap + (s - f * g.spp);
    phase_clock(g, y, 0);
    if (t == 0) {
      // tap kk reads tile position q = wrap(J + hb - kk), chunk position
      // clamp(f * spp - kOverlap + q): one or two runs of q (the tile wrap),
      // each cut where the clamp starts or the owning tile changes
      int n = 0;
      auto add_q_run = [&](int kk0, int kk1, long long q0) {
        const long long c0 = f * g.spp - kOverlap + q0;  // unclamped, falls by one per tap
        int kk = kk0;
        while (kk <= kk1 && n < kMaxRuns) {
          const long long c = c0 - (kk - kk0);
          int kend;
          if (c > last) {
            kend = (int)min((long long)kk1, kk0 + (c0 - last) - 1);
            runs[n++] = {kk, kend, 0, last};
          } else if (c < 0) {
            kend = kk1;
            runs[n++] = {kk, kend, 0, 0};
          } else {
            const long long stop = (c / g.spp) * g.spp;  // the owning tile's first position
            kend = (int)min((long long)kk1, kk + (c - stop));
            runs[n++] = {kk, kend, -1, c};
          }
          kk = kend + 1;
        }
      };
      const long long top = J + g.hb;  // q of tap 0 before the wrap
      if (top >= g.tile) {
        const int kw = (int)(top - g.tile);  // last tap whose q wraps
        add_q_run(0, kw, top - g.tile);
        add_q_run(kw + 1, W - 1, g.tile - 1);
      } else {
        add_q_run(0, W - 1, top);
      }
      nruns = n;
      // A window that reaches the zero fill past the samples read (the
      // capture's end) has analytic-signal values built from the taps' tails
      // alone, whose phase no FP64 evaluation fixes (the FFT's rounding, the
      // reference's included, exceeds them): such a sample keeps its FP32
      // value.
      int sk = 0;
      if (g.n_read < g.total) {
        for (int r = 0; r < n; r++) {
          const long long owner = runs[r].c0 / g.spp;
          const long long tile0 = owner * g.spp - kOverlap;
          const long long vmax = (kOverlap + runs[r].c0 - owner * g.spp) + g.ha;  // highest tile position read
          const long long pmax = min(tile0 + min(vmax, (long long)g.tile - 1), last);
          if (pmax >= g.n_read) sk = 1;
        }
      }
      skip = sk;
    }
    __syncthreads();
    if (skip) {
      if (t == 0 && g.values) g.values[y] = __longlong_as_double(0x7ff8000000000000LL);
      __syncthreads();  // runs and skip are rewritten for the next sample
      continue;
    }
    for (int r = 0; r < nruns; r++) {
      const Run run = runs[r];
      const long long c_hi = run.c0, c_lo = run.c0 + (long long)run.step * (run.kk1 - run.kk0);
      const long long owner = c_lo / g.spp;
      const long long tile0 = owner * g.spp - kOverlap;  // chunk position of the owner's tile position 0
      for (long long cb = c_lo; cb <= c_hi; cb += V) {
        const long long ce = min(cb + V - 1, c_hi);
        const int nz = (int)(ce - cb) + 2;             // z at tile positions J2(cb) - 1 .. J2(ce)
        const long long v0 = (kOverlap + cb - owner * g.spp) - 1 - g.ha;  // tile position of buf[0]
        const int L = nz + 2 * g.ha;
        for (int u = t; u < kN; u += kGT) {
          double x = 0.0;
          if (u < L) {
            const long long p = min(max(tile0 + wrap_pos(v0 + u, g.tile), 0LL), last);
            x = p < g.n_read ? (double)raw_convert<FMT>(g.raw, (int)p) - dc : 0.0;
          }
          buf[u] = make_double2(x, 0.0);
        }
        __syncthreads();
        const bool first_block = r == 0 && cb == c_lo;
        if (first_block) phase_clock(g, y, 1);
        fft_n<false>(buf, tq);
        if (first_block) phase_clock(g, y, 2);
#pragma unroll
        for (int k = t; k < kN; k += kGT) buf[k] = cmul(buf[k], __ldg(&g.gfft[k]));
        __syncthreads();
        fft_n<true>(buf, tq);
        if (first_block) phase_clock(g, y, 3);
        // phases of the block's z, in place
        for (int i = t; i < nz; i += kGT) {
          const double2 z = buf[g.ha + i];
          buf[g.ha + i].x = atan2(z.y, z.x);
        }
        __syncthreads();
        // k_unwrap_to_hz (fm_demod.cu:222-244) for chunk positions cb .. ce
        for (int i = t; i + 1 < nz; i += kGT) {
          double d = buf[g.ha + i + 1].x - buf[g.ha + i].x;
          if (d > kPi64) d -= kTau64;
          if (d < -kPi64) d += kTau64;
          const double hz = d * g.scale;
          if (run.step == 0) {
            for (int kk = run.kk0; kk <= run.kk1; kk++) dem[kk] = hz;  // one position, many taps
          } else {
            dem[run.kk0 + (int)(run.c0 - (cb + i))] = hz;
          }
        }
        __syncthreads();  // buf is refilled by the next block
        if (first_block) phase_clock(g, y, 4);
      }
    }
    phase_clock(g, y, 5);
    // sync sum in a fixed order: strided partials, warp tree, warps in order
    double acc = 0.0;
    for (int kk = t; kk < W; kk += kGT) acc += __ldg(&g.hs64[kk]) * dem[kk];
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((t & 31) == 0) red[t >> 5] = acc;
    __syncthreads();
    if (t == 0) {
      double x64 = 0.0;
      for (int w = 0; w < kGT / 32; w++) x64 += red[w];
      const bool in_pulse = x64 <= g.thr_hz;  // the reference's FP64 decision
      if (g.flips && in_pulse != (g.sync[s] <= g.thr_rel)) atomicAdd(g.flips, 1);
      float r = (float)(x64 - g.ire0);
      if (in_pulse && !(r <= g.thr_rel)) r = g.thr_rel;
      if (!in_pulse && r <= g.thr_rel) r = nextafterf(g.thr_rel, 3.0e38f);
      g.sync[s] = r;
      if (g.values) g.values[y] = x64;
      if (g.dbg_clk && y < kGuardClockSamples) g.dbg_clk[(size_t)y * kPhaseSlots + 7] = nruns;
    }
    phase_clock(g, y, 6);
    __syncthreads();  // runs, dem and red are reused by the next sample
  }
}

}  // namespace

size_t guard_smem_bytes(int hb) {
  return (size_t)(kN + kTwQ) * sizeof(double2) + (size_t)(2 * hb + 1) * sizeof(double);
}

bool guard_supported(int ha, int hb) {
  // one FFT block must yield at least one position, and the sync window must
  // not wrap below the tile start (J - hb >= 0 for every J >= kOverlap)
  return 2 * ha + 2 <= kN && hb < kOverlap && guard_smem_bytes(hb) <= (size_t)kMaxClassBytes;
}

namespace {
template <class S>
cudaError_t launch_guard(const S& src, const GuardArgs& g, int portions, int ctas, cudaStream_t st) {
  const size_t smem = guard_smem_bytes(g.hb);
  auto go = [&](auto kernel) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return launch_chained(kernel, dim3(ctas, 1, portions), dim3(kGT), smem, st, src);
  };
  if (g.in_fmt == kInS16) return go(guard_kernel<kInS16, S>);
  if (g.in_fmt == kInU16) return go(guard_kernel<kInU16, S>);
  return go(guard_kernel<kInU8, S>);
}
}  // namespace

cudaError_t launch_sync_guard(const GuardArgs& g, cudaStream_t st) {
  if (!guard_supported(g.ha, g.hb) || g.cap <= 0) return cudaErrorInvalidValue;
  // a typical chunk lists a few dozen samples, each on its own SM; two CTAs fit an SM
  const int ctas = std::max(1, std::min(g.cap, 148 * 2));
  return launch_guard(ArgsOne<GuardArgs>{g}, g, 1, ctas, st);
}

cudaError_t launch_sync_guard_many(const ArgsMany<GuardArgs>& p, int portions, cudaStream_t st) {
  if (portions <= 0) return cudaSuccess;
  const GuardArgs& g = p.a[0];  // the design every capture of a round shares
  if (!guard_supported(g.ha, g.hb) || g.cap <= 0) return cudaErrorInvalidValue;
  const int ctas = std::max(1, std::min(g.cap, (148 * 2 + portions - 1) / portions));
  return launch_guard(p, g, portions, ctas, st);
}

}  // namespace cuvhs
