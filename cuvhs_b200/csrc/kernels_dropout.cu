// Dropout detection, TBC mapping and concealment (reference K7,
// src/pipeline/dropout_detect.cu:17-339).
//
// One CTA per field.  The tile mean of the envelope comes from the per-CTA
// partial sums K1a already wrote.  Block means (16 samples) over the active
// range are classified in parallel into below-down / above-up / between; the
// two-state hysteresis over those classes is a "last decisive class" scan, so
// the CTA finds each segment's incoming state with one prefix pass instead of
// the reference's one-thread-per-field walk.  The short list of state changes
// is then merged, filtered and mapped to TBC lines in order by one thread, and
// one warp conceals the entries column step by column step (all loads of a
// step before its stores), which is how the reference's copy loop behaves.
#include <cuda_runtime.h>

#include "cuvhs_internal.h"

namespace cuvhs {
namespace {

constexpr int kThreadsD = 256;
constexpr int kMaxBlocks = 49152;   // 16-sample blocks per field held in shared memory
constexpr int kMaxEvents = 2048;

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

__global__ void __launch_bounds__(kThreadsD) dropout_kernel(DropoutArgs a) {
  extern __shared__ unsigned char cls[];  // [kMaxBlocks]
  __shared__ int last_cls[kThreadsD];
  __shared__ int state_in[kThreadsD];
  __shared__ int ev_count[kThreadsD];
  __shared__ int ev_off[kThreadsD];
  __shared__ int events[kMaxEvents];  // block index * 2 + (1 = start, 0 = end)
  __shared__ int n_events;
  __shared__ int rf_s[kMaxRfDropouts], rf_e[kMaxRfDropouts];
  __shared__ int n_entries;
  __shared__ double down_s, up_s;
  const int f = blockIdx.x;
  const int tid = threadIdx.x;
  const double* ll = a.ll + (size_t)f * a.lines_per_frame;
  const int als = a.active_line_start, H = a.out_h, W = a.out_w;
  if (tid == 0) {
    double tot = 0.0;
    for (int b = 0; b < a.env_blocks; b++) tot += a.env_part[(size_t)f * a.env_blocks + b];
    const double mean = tot / (double)a.spp;
    down_s = mean * 0.18;
    up_s = down_s * 1.25;
    n_entries = 0;
  }
  const int fstart = f * a.spp;
  const int s0 = max((int)ll[als], fstart);
  const int s1 = min((int)ll[als + H], fstart + a.spp);
  int* ol = a.do_lines + (size_t)f * kMaxDropouts;
  int* os = a.do_starts + (size_t)f * kMaxDropouts;
  int* oe = a.do_ends + (size_t)f * kMaxDropouts;
  __syncthreads();
  if (s1 <= s0) {
    if (tid == 0) a.do_count[f] = 0;
    return;
  }
  const int nb = min((s1 - s0 + 15) / 16, kMaxBlocks);
  const double down = down_s, up = up_s;
  // 1. classify blocks: 0 = at/below down, 1 = at/above up, 2 = between
  for (int b = tid; b < nb; b += kThreadsD) {
    const int b0 = s0 + b * 16, b1 = min(b0 + 16, s1);
    double sum = 0.0;
    for (int i = b0; i < b1; i++) sum += (double)__ldg(&a.env[i]);
    const double m = sum / (double)(b1 - b0);
    cls[b] = m <= down ? 0 : (m >= up ? 1 : 2);
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
  // 4. merge (<= 30 samples apart), keep <= 128, drop < 10, map to TBC lines
  if (tid == 0) {
    const int ne = min(n_events, kMaxEvents);
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
    n_entries = n;
    a.do_count[f] = n;
  }
  __syncthreads();
  // 5. conceal from the line above (below for line 0), warp 0, groups of 32 entries
  if (tid < 32) {
    const int n = n_entries;
    uint16_t* lf = a.luma + (size_t)f * H * W;
    uint16_t* cf = a.chroma + (size_t)f * H * W;
    for (int g = 0; g < n; g += 32) {
      const int d = g + tid;
      int line = 0, sx = 0, ex = 0, src = H;
      if (d < n) {
        line = ol[d]; sx = os[d]; ex = oe[d];
        src = line > 0 ? line - 1 : line + 1;
      }
      int span = (d < n && src < H) ? ex - sx : 0;
      int maxspan = span;
      for (int off = 16; off > 0; off >>= 1) maxspan = max(maxspan, __shfl_xor_sync(0xffffffffu, maxspan, off));
      for (int it = 0; it < maxspan; it++) {
        const bool act = it < span;
        uint16_t vl = 0, vc = 0;
        if (act) { vl = lf[src * W + sx + it]; vc = cf[src * W + sx + it]; }
        __syncwarp();
        if (act) { lf[line * W + sx + it] = vl; cf[line * W + sx + it] = vc; }
        __syncwarp();
      }
    }
  }
}

}  // namespace

void launch_dropouts(const DropoutArgs& a, cudaStream_t st) {
  if (a.fields <= 0) return;
  const size_t smem = kMaxBlocks;
  cudaFuncSetAttribute(dropout_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dropout_kernel<<<a.fields, kThreadsD, smem, st>>>(a);
}

}  // namespace cuvhs
