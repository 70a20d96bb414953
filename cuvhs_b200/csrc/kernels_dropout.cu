// Dropout detection, TBC mapping and concealment (reference K7,
// src/pipeline/dropout_detect.cu:17-339).
//
// The tile mean of the envelope comes from the per-CTA partial sums K1a
// already wrote.  Block means (16 samples) over the active range are
// classified into below-down / above-up / between; the two-state hysteresis
// over those classes is a "last decisive class" scan, so each segment's
// incoming state comes from one prefix pass instead of the reference's
// one-thread-per-field walk.  The short list of state changes is then merged,
// filtered and mapped to TBC lines in order by one thread, and one warp
// conceals the entries column step by column step (all loads of a step before
// its stores), which is how the reference's copy loop behaves.
//
// Two forms share those steps:
//  * two-pass (the decoder): a wide class kernel (one thread per block, every
//    field at once, the envelope staged through shared memory with coalesced
//    loads) writes one class byte per block, and a per-field kernel reads the
//    bytes back from L2, scans, maps and conceals the luma.  The envelope read
//    -- the stage's HBM traffic -- runs on every SM.  Luma is final once the
//    luma resampler has run, so it is concealed (and can leave the device)
//    while chroma is still being decoded; chroma is concealed afterwards.
//  * fused (cuvhs_dropouts_noalloc): one CTA per field does everything, with
//    the classes in shared memory, so it needs no scratch beyond the partials.
#include <cuda_runtime.h>

#include "chain.cuh"
#include "cuvhs_internal.h"

namespace cuvhs {
namespace {

constexpr int kThreadsD = 256;       // fused kernel and class kernel
constexpr int kThreadsScan = 512;    // two-pass scan kernel
constexpr int kMaxEvents = 2048;
constexpr int kStage = kThreadsD * 16;  // envelope samples one class CTA stages
constexpr int kMaxEnvBlocks = 1024;     // envelope partials a class CTA holds in shared memory

__device__ int find_line(const double* ll, int als, int n, double pos) {
  if (pos < ll[als] || pos >= ll[als + n]) return -1;
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (ll[als + mid] <= pos) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Active sample range [s0, s1) of field f (chunk sample indices).
__device__ __forceinline__ void active_range(const DropoutArgs& a, int f, int& s0, int& s1) {
  const double* ll = a.ll + (size_t)f * a.lines_per_frame;
  const int fstart = f * a.spp;
  s0 = max((int)ll[a.active_line_start], fstart);
  s1 = min((int)ll[a.active_line_start + a.out_h], fstart + a.spp);
}

// Lower threshold: 0.18 x the tile mean of the envelope, summed in partial order.
__device__ __forceinline__ double down_threshold(const DropoutArgs& a, int f) {
  double tot = 0.0;
  for (int b = 0; b < a.env_blocks; b++) tot += a.env_part[(size_t)f * a.env_blocks + b];
  return tot / (double)a.spp * 0.18;
}

__device__ __forceinline__ unsigned char block_class(double sum, int n, double down, double up) {
  const double m = sum / (double)n;
  return m <= down ? 0 : (m >= up ? 1 : 2);  // 0 = at/below down, 1 = at/above up, 2 = between
}

// Step 4 (thread 0): merge start/end events (<= 30 samples apart), keep <= 128
// spans, drop spans < 10 samples, map to TBC lines.  Returns the entry count.
__device__ int map_events(const DropoutArgs& a, int f, const int* events, int ne, int s0, int s1, int* rf_s,
                          int* rf_e) {
  const double* ll = a.ll + (size_t)f * a.lines_per_frame;
  const int als = a.active_line_start, H = a.out_h, W = a.out_w;
  int* ol = a.do_lines + (size_t)f * kMaxDropouts;
  int* os = a.do_starts + (size_t)f * kMaxDropouts;
  int* oe = a.do_ends + (size_t)f * kMaxDropouts;
  int nrf = 0, open = -1;
  for (int e = 0; e < ne; e++) {
    const int pos = s0 + (events[e] >> 1) * 16;
    if (events[e] & 1) {
      open = pos;
    } else if (open >= 0) {
      if (nrf > 0 && open - rf_e[nrf - 1] <= 30) rf_e[nrf - 1] = pos;
      else if (nrf < kMaxRfDropouts) { rf_s[nrf] = open; rf_e[nrf] = pos; nrf++; }
      open = -1;
    }
  }
  if (open >= 0) {
    if (nrf > 0 && open - rf_e[nrf - 1] <= 30) rf_e[nrf - 1] = s1;
    else if (nrf < kMaxRfDropouts) { rf_s[nrf] = open; rf_e[nrf] = s1; nrf++; }
  }
  int n = 0;
  for (int i = 0; i < nrf && n < kMaxDropouts; i++) {
    if (rf_e[i] - rf_s[i] < 10) continue;
    const double sa = (double)rf_s[i], ea = (double)rf_e[i];
    const int sl = find_line(ll, als, H, sa);
    if (sl < 0) continue;
    int el = find_line(ll, als, H, ea - 1.0);
    if (el < 0) el = H - 1;
    for (int l = sl; l <= el && n < kMaxDropouts; l++) {
      const double l0 = ll[als + l], l1 = ll[als + l + 1], len = l1 - l0;
      if (len <= 0.0) continue;
      const int sx = (l == sl) ? max(0, (int)((sa - l0) / len * (double)W)) : 0;
      const int ex = (l == el) ? min(W, (int)((ea - l0) / len * (double)W + 0.999)) : W;
      if (ex > sx) { ol[n] = l; os[n] = sx; oe[n] = ex; n++; }
    }
  }
  a.do_count[f] = n;
  return n;
}

// Step 5 (one warp): conceal from the line above (below for line 0), groups of
// 32 entries, every load of a column step before its stores.  Planes are
// independent, so luma and chroma may be concealed in separate passes.
__device__ void conceal(const DropoutArgs& a, int f, int n, int lane, bool luma, bool chroma) {
  const int H = a.out_h, W = a.out_w;
  const int* ol = a.do_lines + (size_t)f * kMaxDropouts;
  const int* os = a.do_starts + (size_t)f * kMaxDropouts;
  const int* oe = a.do_ends + (size_t)f * kMaxDropouts;
  uint16_t* lf = a.luma + (size_t)f * H * W;
  uint16_t* cf = a.chroma + (size_t)f * H * W;
  for (int g = 0; g < n; g += 32) {
    const int d = g + lane;
    int line = 0, sx = 0, ex = 0, src = H;
    if (d < n) {
      line = ol[d]; sx = os[d]; ex = oe[d];
      src = line > 0 ? line - 1 : line + 1;
    }
    const int span = (d < n && src < H) ? ex - sx : 0;
    int maxspan = span;
    for (int off = 16; off > 0; off >>= 1) maxspan = max(maxspan, __shfl_xor_sync(0xffffffffu, maxspan, off));
    for (int it = 0; it < maxspan; it++) {
      const bool act = it < span;
      uint16_t vl = 0, vc = 0;
      if (act && luma) vl = lf[src * W + sx + it];
      if (act && chroma) vc = cf[src * W + sx + it];
      __syncwarp();
      if (act && luma) lf[line * W + sx + it] = vl;
      if (act && chroma) cf[line * W + sx + it] = vc;
      __syncwarp();
    }
  }
}

// ------------------------------------------------------------------ fused form

__global__ void __launch_bounds__(kThreadsD) dropout_kernel(DropoutArgs a) {
  chain_wait();
  extern __shared__ unsigned char cls[];  // [a.max_blocks]
  __shared__ int last_cls[kThreadsD];
  __shared__ int state_in[kThreadsD];
  __shared__ int ev_count[kThreadsD];
  __shared__ int ev_off[kThreadsD];
  __shared__ int events[kMaxEvents];  // block index * 2 + (1 = start, 0 = end)
  __shared__ int n_events;
  __shared__ int rf_s[kMaxRfDropouts], rf_e[kMaxRfDropouts];
  __shared__ int n_entries;
  __shared__ double down_s;
  const int f = blockIdx.x;
  const int tid = threadIdx.x;
  if (tid == 0) down_s = down_threshold(a, f);
  int s0, s1;
  active_range(a, f, s0, s1);
  __syncthreads();
  if (s1 <= s0) {
    if (tid == 0) a.do_count[f] = 0;
    return;
  }
  const int nb = min((s1 - s0 + 15) / 16, a.max_blocks);
  const double down = down_s, up = down * 1.25;
  // 1. classify blocks
  for (int b = tid; b < nb; b += kThreadsD) {
    const int b0 = s0 + b * 16, b1 = min(b0 + 16, s1);
    double sum = 0.0;
    for (int i = b0; i < b1; i++) sum += (double)__ldg(&a.env[i]);
    cls[b] = block_class(sum, b1 - b0, down, up);
  }
  __syncthreads();
  // 2. per-segment last decisive class
  const int per = (nb + kThreadsD - 1) / kThreadsD;
  const int b_lo = min(nb, tid * per), b_hi = min(nb, b_lo + per);
  int lc = -1;
  for (int b = b_lo; b < b_hi; b++)
    if (cls[b] != 2) lc = cls[b];
  last_cls[tid] = lc;
  __syncthreads();
  if (tid == 0) {
    int st = 0;  // 0 = no dropout open
    for (int t = 0; t < kThreadsD; t++) {
      state_in[t] = st;
      if (last_cls[t] == 0) st = 1;
      else if (last_cls[t] == 1) st = 0;
    }
  }
  __syncthreads();
  // 3. state changes, counted then written in order
  int st = state_in[tid], cnt = 0;
  for (int b = b_lo; b < b_hi; b++) {
    if (cls[b] == 0 && !st) { st = 1; cnt++; }
    else if (cls[b] == 1 && st) { st = 0; cnt++; }
  }
  ev_count[tid] = cnt;
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int t = 0; t < kThreadsD; t++) { ev_off[t] = acc; acc += ev_count[t]; }
    n_events = acc;
  }
  __syncthreads();
  st = state_in[tid];
  int k = ev_off[tid];
  for (int b = b_lo; b < b_hi; b++) {
    if (cls[b] == 0 && !st) { st = 1; if (k < kMaxEvents) events[k] = b * 2 + 1; k++; }
    else if (cls[b] == 1 && st) { st = 0; if (k < kMaxEvents) events[k] = b * 2; k++; }
  }
  __syncthreads();
  if (tid == 0) n_entries = map_events(a, f, events, min(n_events, kMaxEvents), s0, s1, rf_s, rf_e);
  __syncthreads();
  if (tid < 32) conceal(a, f, n_entries, tid, true, true);
}

// --------------------------------------------------------------- two-pass form

// grid (ceil(max_blocks / kThreadsD), fields): CTA x classifies blocks
// [x*256, x*256 + 256) of field y.  The 4096 envelope samples behind them are
// staged with coalesced loads into rows of 17 floats (conflict-free column
// reads), then each thread sums its row in sample order.
template <class Src>
__global__ void __launch_bounds__(kThreadsD) dropout_class_kernel(const __grid_constant__ Src src) {
  const DropoutArgs& a = src.get();
  if ((int)blockIdx.y >= a.fields) return;  // whole CTA: a batched capture with fewer fields
  chain_wait();
  __shared__ float stage[kThreadsD * 17];
  __shared__ double part[kMaxEnvBlocks];
  __shared__ double down_s;
  const int f = blockIdx.y, tid = threadIdx.x;
  int s0, s1;
  active_range(a, f, s0, s1);
  const int nb = min((s1 - s0 + 15) / 16, a.max_blocks);
  const int b_first = blockIdx.x * kThreadsD;
  if (s1 <= s0 || b_first >= nb) return;  // whole CTA leaves together
  // the field's envelope partial sums, loaded in parallel with the stage
  const bool part_in_smem = a.env_blocks <= kMaxEnvBlocks;
  if (part_in_smem)
    for (int b = tid; b < a.env_blocks; b += kThreadsD) part[b] = a.env_part[(size_t)f * a.env_blocks + b];
  const int x0 = s0 + b_first * 16;
  const int nx = min(kStage, s1 - x0);
  // loads at a clamped index, so that all of a thread's loads are in flight
  // at once; samples past the range are zeroed afterwards
#pragma unroll
  for (int i = tid; i < kStage; i += kThreadsD) {
    const float e = __ldg(&a.env[x0 + min(i, nx - 1)]);
    stage[(i >> 4) * 17 + (i & 15)] = i < nx ? e : 0.0f;
  }
  __syncthreads();
  if (tid == 0) {
    // summed in partial order, as down_threshold
    double tot = 0.0;
    if (part_in_smem)
      for (int b = 0; b < a.env_blocks; b++) tot += part[b];
    else
      for (int b = 0; b < a.env_blocks; b++) tot += a.env_part[(size_t)f * a.env_blocks + b];
    down_s = tot / (double)a.spp * 0.18;
  }
  __syncthreads();
  const int b = b_first + tid;
  if (b >= nb) return;
  const int n = min(16, s1 - (s0 + b * 16));
  double sum = 0.0;
  for (int i = 0; i < n; i++) sum += (double)stage[tid * 17 + i];
  const double down = down_s;
  a.cls[(size_t)f * a.max_blocks + b] = block_class(sum, n, down, down * 1.25);
}

// Block-wide exclusive scans over kThreadsScan threads (warp shuffles, then
// the warp totals).  wsh holds 32 ints; every thread must call.
__device__ __forceinline__ int block_excl_sum(int v, int* wsh, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = kThreadsScan / 32;
  int x = v;
  for (int off = 1; off < 32; off <<= 1) {
    const int o = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += o;
  }
  if (lane == 31) wsh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < NW ? wsh[lane] : 0;
    for (int off = 1; off < 32; off <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += o;
    }
    if (lane < NW) wsh[lane] = w;  // inclusive warp prefix
  }
  __syncthreads();
  const int res = x - v + (warp > 0 ? wsh[warp - 1] : 0);
  *total = wsh[NW - 1];
  __syncthreads();  // wsh free for the next scan
  return res;
}

// "Last decisive class" prefix: combine(left, right) = right != -1 ? right : left.
__device__ __forceinline__ int block_excl_last(int v, int* wsh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = kThreadsScan / 32;
  int x = v;
  for (int off = 1; off < 32; off <<= 1) {
    const int o = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off && x == -1) x = o;
  }
  if (lane == 31) wsh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < NW ? wsh[lane] : -1;
    for (int off = 1; off < 32; off <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off && w == -1) w = o;
    }
    if (lane < NW) wsh[lane] = w;
  }
  __syncthreads();
  int ex = __shfl_up_sync(0xffffffffu, x, 1);
  if (lane == 0) ex = -1;
  if (ex == -1 && warp > 0) ex = wsh[warp - 1];
  __syncthreads();
  return ex;
}

// One CTA per field: class bytes back from L2 into shared memory, then the
// hysteresis scan, event list, mapping and luma concealment (chroma is
// concealed by dropout_chroma_kernel once the chroma planes are final).
template <class Src>
__global__ void __launch_bounds__(kThreadsScan) dropout_scan_kernel(const __grid_constant__ Src src) {
  const DropoutArgs& a = src.get();
  if ((int)blockIdx.x >= a.fields) return;  // whole CTA
  chain_wait();
  extern __shared__ uint4 cls4[];  // [a.max_blocks / 16]
  __shared__ int wsh[32];
  __shared__ int events[kMaxEvents];
  __shared__ int rf_s[kMaxRfDropouts], rf_e[kMaxRfDropouts];
  __shared__ int n_entries;
  const unsigned char* cls = reinterpret_cast<const unsigned char*>(cls4);
  const int f = blockIdx.x, tid = threadIdx.x;
  int s0, s1;
  active_range(a, f, s0, s1);
  if (s1 <= s0) {
    if (tid == 0) a.do_count[f] = 0;
    return;  // whole CTA leaves together
  }
  const int nb = min((s1 - s0 + 15) / 16, a.max_blocks);
  const uint4* cls_in = reinterpret_cast<const uint4*>(a.cls + (size_t)f * a.max_blocks);
  for (int i = tid; i < (nb + 15) / 16; i += kThreadsScan) cls4[i] = cls_in[i];
  __syncthreads();
  const int per = (nb + kThreadsScan - 1) / kThreadsScan;
  const int b_lo = min(nb, tid * per), b_hi = min(nb, b_lo + per);
  int lc = -1;
  for (int b = b_lo; b < b_hi; b++)
    if (cls[b] != 2) lc = cls[b];
  const int lc_in = block_excl_last(lc, wsh);
  const int st_in = lc_in == 0 ? 1 : 0;  // 1 = dropout open
  int st = st_in, cnt = 0;
  for (int b = b_lo; b < b_hi; b++) {
    if (cls[b] == 0 && !st) { st = 1; cnt++; }
    else if (cls[b] == 1 && st) { st = 0; cnt++; }
  }
  int n_events;
  int k = block_excl_sum(cnt, wsh, &n_events);
  st = st_in;
  for (int b = b_lo; b < b_hi; b++) {
    if (cls[b] == 0 && !st) { st = 1; if (k < kMaxEvents) events[k] = b * 2 + 1; k++; }
    else if (cls[b] == 1 && st) { st = 0; if (k < kMaxEvents) events[k] = b * 2; k++; }
  }
  __syncthreads();
  if (tid == 0) n_entries = map_events(a, f, events, min(n_events, kMaxEvents), s0, s1, rf_s, rf_e);
  __syncthreads();
  if (tid < 32) conceal(a, f, n_entries, tid, true, false);
}

// One warp per field: chroma concealment from the entries the scan kernel wrote.
template <class Src>
__global__ void dropout_chroma_kernel(const __grid_constant__ Src src, int f0, int nf) {
  const DropoutArgs& a = src.get();
  chain_wait();
  const int f = f0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (f >= f0 + nf || f >= a.fields) return;  // whole warp
  const int n = min(max(a.do_count[f], 0), kMaxDropouts);
  conceal(a, f, n, threadIdx.x & 31, false, true);
}

}  // namespace

// The per-field class bytes live in dynamic shared memory.  Both kernels that
// hold them are given the same fixed cap (kMaxClassBytes, not the size one
// call needs), so contexts of different rates on different host threads never
// lower the cap between another thread's set and its launch.
cudaError_t launch_dropouts(const DropoutArgs& a, cudaStream_t st) {
  if (a.fields <= 0) return cudaSuccess;
  const size_t smem = (size_t)a.max_blocks;
  if (smem > (size_t)kMaxClassBytes) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(dropout_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxClassBytes);
  if (e != cudaSuccess) return e;
  return launch_chained(dropout_kernel, dim3(a.fields), dim3(kThreadsD), smem, st, a);
}

size_t dropout_class_bytes_per_field(int spp) { return (size_t)(((spp + 15) / 16 + 15) / 16 * 16); }

namespace {
template <class S>
void two_pass_launch(const S& src, const DropoutArgs& a, int portions, int max_fields, cudaStream_t st) {
  dim3 grid((a.max_blocks + kThreadsD - 1) / kThreadsD, max_fields, portions);
  launch_chained(dropout_class_kernel<S>, grid, dim3(kThreadsD), 0, st, src);
  const size_t smem = (size_t)a.max_blocks;
  cudaFuncSetAttribute(dropout_scan_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxClassBytes);
  launch_chained(dropout_scan_kernel<S>, dim3(max_fields, 1, portions), dim3(kThreadsScan), smem, st, src);
}

template <class S>
void conceal_launch(const S& src, int portions, int f0, int nf, cudaStream_t st) {
  const int threads = 128;
  launch_chained(dropout_chroma_kernel<S>, dim3((nf * 32 + threads - 1) / threads, 1, portions), dim3(threads), 0, st,
                 src, f0, nf);
}
}  // namespace

void launch_dropouts_two_pass(const DropoutArgs& a, cudaStream_t st) {
  if (a.fields <= 0) return;
  two_pass_launch(ArgsOne<DropoutArgs>{a}, a, 1, a.fields, st);
}

void launch_dropout_conceal_chroma(const DropoutArgs& a, int f0, int nf, cudaStream_t st) {
  if (nf <= 0 || f0 < 0 || f0 >= a.fields) return;
  conceal_launch(ArgsOne<DropoutArgs>{a}, 1, f0, nf, st);
}

void launch_dropouts_two_pass_many(const ArgsMany<DropoutArgs>& p, int portions, int max_fields, cudaStream_t st) {
  if (portions > 0 && max_fields > 0) two_pass_launch(p, p.a[0], portions, max_fields, st);
}

void launch_dropout_conceal_chroma_many(const ArgsMany<DropoutArgs>& p, int portions, int max_fields,
                                        cudaStream_t st) {
  if (portions > 0 && max_fields > 0) conceal_launch(p, portions, 0, max_fields, st);
}

}  // namespace cuvhs
