// Field windows and line locations on the GPU: the reference's VSYNC
// clustering (src/pipeline/pipeline.cu:1567-1651), pulse windows
// (src/pipeline/sync_pulses.cu:10-58), its validated host line location "K2b"
// (pipeline.cu:410-893, driven from :1717-1778) and its single-pass line
// locator (src/pipeline/line_locs.cu:62-543).
//
// The reference runs K2b on the host, one field after another, because each
// field's anchor may use the previous field's.  Most of the work needs no
// carried state, so here it runs one CTA per field, in parallel:
//  * pulse validation: the reference walks the raw pulses once, appending
//    hsync-width pulses and, at an EQ-width pulse after an hsync, the output
//    of a vertical-blanking recogniser started two pulses back (kept if the
//    sequence closes).  The walk advances one pulse per step whatever happens,
//    and a recogniser attempt depends only on the raw pulses, so every
//    attempt is evaluated in parallel; one thread then resolves, pulse by
//    pulse, which attempts fire (an O(1) step each), a scan places every
//    pulse's output, and the "good" cadence flags follow from neighbouring
//    entries;
//  * mean line length (longest hsync run), blanking scan (last match per
//    slot), and -- when the field's own half-line pattern fixes its order --
//    the anchor fit and the 525-line snap, exactly as the in-order pass would
//    compute them for any previous field.
// A single CTA then walks the fields in order with the carried state
// (pipeline.h:92-97, kept on the device), reusing the speculative grid or
// fitting and snapping again.  FP64 throughout; sums whose order matters
// (anchor offsets) are taken in the reference's order by one thread, sums of
// integers in parallel.  This file is compiled with -fmad=false so that every
// a * b + c rounds as two operations, as the reference's host code does; the
// single-pass locator, whose reference is device code, writes its fused
// multiply-adds out with fma().
#include <cuda_runtime.h>

#include <cstdint>

#include "chain.cuh"
#include "cuvhs_internal.h"

namespace cuvhs {
namespace {

constexpr int kLT = 256;           // threads per line-location CTA
constexpr int kSortMax = 4096;     // validated pulses sorted in shared memory
constexpr int kSmemValid = 2048;   // validated pulses held in shared memory

__device__ __forceinline__ bool within(double v, double lo, double hi) { return v >= lo && v <= hi; }

// Phase clocks for inspection: thread 0 records the SM clock at phase k of
// field f's CTA when the caller asked for them.
__device__ __forceinline__ void phase_clock(const LineLocArgs& a, int f, int k) {
  if (a.dbg_clk && threadIdx.x == 0) a.dbg_clk[(size_t)f * kPhaseSlots + k] = clock64();
}

// ------------------------------------------------------------ field windows

// First index in sorted a[0, n) whose value is > v.
__device__ __forceinline__ int upper_idx(const unsigned* a, int n, unsigned v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// End of the threshold run that starts at falling edge i: the first rising
// edge after it, or the range end.  Every sample is in or out of a pulse, so
// in sample order the edges alternate, falling first (a pulse open at the
// chunk's first sample falls there): rising edge i closes run i.
__device__ __forceinline__ long long run_end(const LineLocArgs& a, int nrise, int i) {
  return i < nrise ? (long long)a.rise[i] : a.total;
}

// One CTA: VSYNC candidates (runs of 20-35 us, vsync_discover.cu:58-72) in
// sample order, clustered into field windows (pipeline.cu:1567-1651).
//
// Candidates: the falling edges are taken 1024 at a time, one per thread
// (coalesced), and a block scan appends the candidates in order.  Clustering:
// the reference opens a window at the first candidate and at every later
// candidate more than half a field past the open window's start (the
// candidate less five lines), so the window that follows candidate j opens at
// the first candidate past off(j) + spf / 2 -- found for every candidate at
// once by binary search -- and one thread follows that chain from the first
// candidate, one step per field.
constexpr int kWinThreads = 1024;
constexpr int kWinSmemCand = 12288;  // candidates clustered in shared memory; more: the serial path
size_t fieldwin_smem_bytes() { return (size_t)kWinSmemCand * 2 * sizeof(int); }

template <class Src>
__global__ void __launch_bounds__(kWinThreads) fieldwin_kernel(const __grid_constant__ Src src) {
  const LineLocArgs& a = src.get();
  chain_wait();
  extern __shared__ int wsm[];
  int* scand = wsm;                  // [kWinSmemCand] candidate positions
  int* snext = wsm + kWinSmemCand;   // [kWinSmemCand] index of the next window's first candidate
  __shared__ int warp_tot[kWinThreads / 32];
  __shared__ int base_s;
  const int nfall = min(a.counts[0], a.edge_cap), nrise = min(a.counts[1], a.edge_cap);
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) {
    a.win->err = (a.counts[0] > a.edge_cap || a.counts[1] > a.edge_cap) ? 1 : 0;
    base_s = 0;
  }
  __syncthreads();
  // candidates in order, one tile of falling edges per step (the next tile's
  // edges are loaded before the current tile's scan)
  int nf = 0, nr = 0;
  if (t < nfall) {
    nf = (int)a.fall[t];
    nr = t < nrise ? (int)a.rise[t] : 0;
  }
  for (int i0 = 0; i0 < nfall; i0 += kWinThreads) {
    const int i = i0 + t;
    const long long fpos = (unsigned)nf;
    const long long end = i < nrise ? (long long)(unsigned)nr : a.total;  // run_end
    const bool cand = i < nfall && end - fpos >= a.minw && end - fpos <= a.maxw;
    const int j = i + kWinThreads;
    if (j < nfall) {
      nf = (int)a.fall[j];
      nr = j < nrise ? (int)a.rise[j] : 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, cand);
    if (lane == 0) warp_tot[warp] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < kWinThreads / 32; w++) {
      if (w < warp) before += warp_tot[w];
      total += warp_tot[w];
    }
    const int k = base_s + before + __popc(m & ((1u << lane) - 1u));
    if (cand) {
      if (k < a.cand_cap) a.cand[k] = (int)fpos;
      if (k < kWinSmemCand) scand[k] = (int)fpos;
    }
    __syncthreads();
    if (t == 0) base_s += total;
    __syncthreads();
  }
  const int base = base_s;
  const int ncand = min(base, a.cand_cap);
  const long long spf = a.fmt.samples_per_field, spl = a.fmt.samples_per_line;
  auto off_of = [&](long long pos) { return pos > 5 * spl ? pos - 5 * spl : 0LL; };
  const bool in_smem = ncand <= kWinSmemCand;
  if (in_smem) {
    for (int j = t; j < ncand; j += kWinThreads) {
      const long long lim = off_of(scand[j]) + spf / 2;  // the next window: first candidate past lim
      int lo = j + 1, hi = ncand;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((long long)scand[mid] > lim) hi = mid;
        else lo = mid + 1;
      }
      snext[j] = lo;
    }
  }
  __syncthreads();
  if (t != 0) return;
  int n = 0;
  if (in_smem) {
    for (int j = 0; j < ncand && n < a.num_fields; j = snext[j]) a.offs[n++] = off_of(scand[j]);
  } else {
    long long open = 0;
    for (int j = 0; j < ncand; j++) {
      const long long pos = a.cand[j];
      if (n == 0 || pos - open > spf / 2) {
        if (n >= a.num_fields) break;  // later windows are cut off anyway
        open = off_of(pos);
        a.offs[n++] = open;
      }
    }
  }
  if (n == 0)
    for (int i = 0; i < a.tiles && i < a.num_fields; i++) a.offs[n++] = (long long)i * spf;
  long long actual = spf;
  if (n >= 2) actual = (a.offs[n - 1] - a.offs[0]) / (n - 1);
  const long long predicted = a.offs[n - 1] + actual, margin = 10 * spl;
  a.win->fields = n;
  a.win->ncand = base;
  a.win->next_rel = predicted > margin ? predicted - margin : predicted;
}

// Grid (num_fields): the pulses of field f's window (sync_pulses.cu:10-58):
// threshold runs that start after the window start and end within the
// spp-sample scan, at most kMaxPulses.
template <class Src>
__global__ void __launch_bounds__(kLT) pulses_kernel(const __grid_constant__ Src src) {
  const LineLocArgs& a = src.get();
  chain_wait();
  __shared__ int brk;
  const int f = blockIdx.x;
  if (f >= a.win->fields) return;
  const int nfall = min(a.counts[0], a.edge_cap), nrise = min(a.counts[1], a.edge_cap);
  const long long off = a.offs[f], lim = off + a.fmt.spp - 1;
  const int i0 = upper_idx(a.fall, nfall, (unsigned)min(off, (long long)UINT32_MAX));  // first start > off
  const int i1 = upper_idx(a.fall, nfall, (unsigned)min(lim, (long long)UINT32_MAX));  // first start > lim
  if (threadIdx.x == 0) brk = i1;
  __syncthreads();
  for (int b = i0; b < i1 && b < brk; b += kLT) {
    const int i = b + threadIdx.x;
    if (i < i1 && run_end(a, nrise, i) > lim) atomicMin(&brk, i);
    __syncthreads();
  }
  const int n = min(brk - i0, kMaxPulses);
  int* ps = a.ps + (size_t)f * kMaxPulses;
  int* pl = a.pl + (size_t)f * kMaxPulses;
  for (int k = threadIdx.x; k < n; k += kLT) {
    const unsigned s = a.fall[i0 + k];
    ps[k] = (int)s;
    pl[k] = (int)(run_end(a, nrise, i0 + k) - (long long)s);
  }
  if (threadIdx.x == 0) a.pn[f] = max(n, 0);
}

// ------------------------------------------------------------ K2b per field

struct Windows {  // adaptive pulse-width classes (pipeline.cu:450-477)
  double h_lo, h_hi, e_lo, e_hi, v_lo, v_hi;
};

__device__ bool spacing_ok(int prev_type, int type, int delta, int line_len) {
  double lo, hi;
  if (prev_type > 0 && type > 0) {
    lo = 0.4;
    hi = 0.6;
  } else if (prev_type == 0 && type == 0) {
    lo = 0.9;
    hi = 1.1;
  } else {
    lo = 0.4;
    hi = 1.1;
  }
  const double span = (double)delta / (double)line_len;
  return span >= lo && span <= hi;
}

__device__ const double* field_pattern(int system, bool first) {
  // Spacings (lines) of the last hsync -> first EQ and last EQ -> first hsync
  // around this field's blanking interval, then around the next one
  // (pipeline.cu:704-716).
  static __device__ const double ntsc_first[4] = {1, 0.5, 0.5, 1}, ntsc_second[4] = {0.5, 1, 1, 0.5};
  static __device__ const double pal_first[4] = {0.5, 0.5, 1, 1}, pal_second[4] = {1, 1, 0.5, 0.5};
  if (system == kPal) return first ? pal_first : pal_second;
  return first ? ntsc_first : ntsc_second;
}

__device__ double predicted_field_lines(const Format& fmt, bool first) {
  const int cur = first ? fmt.field_lines_first : fmt.field_lines_second;
  const int prev = first ? fmt.field_lines_second : fmt.field_lines_first;
  return fmt.system == kPal ? cur : prev;
}

__device__ double half_line_round(double lines) { return round(0.5 * round(lines / 0.5) * 10.0) / 10.0; }

// Width classes as integer bounds: a pulse length (an integer) lies in
// [lo, hi] exactly when it lies in [ceil(lo), floor(hi)].
struct IWindows {
  int h_lo, h_hi, e_lo, e_hi, v_lo, v_hi;
};
__device__ __forceinline__ int ceil_int(double x) { return (int)fmin(fmax(ceil(x), -2147483647.0), 2147483647.0); }
__device__ __forceinline__ int floor_int(double x) { return (int)fmin(fmax(floor(x), -2147483647.0), 2147483647.0); }
__device__ IWindows int_windows(const Windows& w) {
  IWindows r;
  r.h_lo = ceil_int(w.h_lo);
  r.h_hi = floor_int(w.h_hi);
  r.e_lo = ceil_int(w.e_lo);
  r.e_hi = floor_int(w.e_hi);
  r.v_lo = ceil_int(w.v_lo);
  r.v_hi = floor_int(w.v_hi);
  return r;
}
__device__ __forceinline__ bool in_class(int len, int lo, int hi) { return len >= lo && len <= hi; }

// The vertical-blanking recogniser (pipeline.cu:519-609) from pulse `first`,
// over at most 26 pulses, entered with an hsync as the list's last entry.
// Returns whether the sequence closed, with the number appended and the type
// of the last one.  With out_s given, the appended entries (start, length,
// type) are written there.  Widths and the hold-off position are compared as
// integers: a start x (an integer) is past the FP64 hold-off h exactly when
// x > floor(h), and before it exactly when x < ceil(h).
__device__ bool attempt(const int* ps, const int* pl, int n, int first, const IWindows& w, int eq_pulses, int line_len,
                        int* appended, int* last_type, int* out_s = nullptr, int* out_l = nullptr,
                        unsigned char* out_t = nullptr) {
  bool done = false;
  const double half = eq_pulses / 2.0;
  bool vsync_seen = false;
  long long hold_floor = 0, hold_ceil = 0;  // of the FP64 hold-off position (0.0 at first)
  double pending = -1.0;
  int cur = kHsync, cnt = 0;
  const int end = min(n, first + 26);
  for (int i = first; i < end; i++) {
    const int len = pl[i];
    const int start = ps[i];
    int type = -1;
    switch (cur) {
      case kHsync:
        if (in_class(len, w.h_lo, w.h_hi)) {
          type = kHsync;
        } else if (in_class(len, w.e_lo, w.e_hi)) {
          type = kEq1;
          pending = half;
        } else if (in_class(len, w.v_lo, w.v_hi)) {
          vsync_seen = true;
          type = kVsync;
        }
        break;
      case kEq1:
        if (in_class(len, w.e_lo, w.e_hi)) {
          type = kEq1;
        } else if (in_class(len, w.v_lo, w.v_hi)) {
          vsync_seen = true;
          type = kVsync;
          pending = half;
        } else if (in_class(len, w.h_lo, w.h_hi)) {
          type = kHsync;
        }
        break;
      case kVsync:
        if (in_class(len, w.e_lo, w.e_hi)) {
          type = kEq2;
          pending = half;
        } else if (in_class(len, w.v_lo, w.v_hi)) {
          type = kVsync;
        } else if ((long long)start > hold_floor && in_class(len, w.h_lo, w.h_hi)) {
          type = kHsync;
        }
        break;
      case kEq2:
        if (in_class(len, w.e_lo, w.e_hi)) {
          type = kEq2;
        } else if (in_class(len, w.h_lo, w.h_hi)) {
          type = kHsync;
          done = true;
        }
        break;
    }
    bool keep = type >= 0;
    if (keep && type != cur) {
      if ((long long)start < hold_ceil) {
        keep = false;
      } else if (pending > 0.0) {
        const double hold = (double)start + ((pending - 0.1) * (double)line_len);
        hold_floor = (long long)floor(hold);
        hold_ceil = (long long)ceil(hold);
        pending = -1.0;
      }
    }
    if (keep) {
      if (out_s) {
        out_s[cnt] = start;
        out_l[cnt] = len;
        out_t[cnt] = (unsigned char)type;
      }
      cnt++;
      cur = type;
    }
    if (done && vsync_seen) break;
  }
  *appended = cnt;
  *last_type = cur;
  return done && cnt > 0;
}

// The same recogniser run by a whole warp on one attempt: lane k holds pulse
// first + k, and every lane steps the state machine over the lanes' pulses
// (broadcast by shuffles), so no lane diverges and no step waits on shared
// memory.  Returns the closing flag, the count and last type, and the kept
// steps (bit k) with their types (2 bits at 2k).
struct WarpAttempt {
  bool ok;
  int cnt, last;
  unsigned keep;
  unsigned long long types;
};
__device__ WarpAttempt attempt_warp(const int* ps, const int* pl, int n, int first, const IWindows& w, int eq_pulses,
                                    int line_len) {
  const int lane = threadIdx.x & 31;
  const int end = min(n, first + 26);
  const int mine = first + lane;
  const int my_len = mine < end ? pl[mine] : 0, my_start = mine < end ? ps[mine] : 0;
  bool done = false, vsync_seen = false;
  const double half = eq_pulses / 2.0;
  long long hold_floor = 0, hold_ceil = 0;
  double pending = -1.0;
  int cur = kHsync, cnt = 0;
  unsigned keep_mask = 0;
  unsigned long long types = 0;
  const int steps = end - first;
  for (int k = 0; k < steps; k++) {
    const int len = __shfl_sync(0xffffffffu, my_len, k);
    const int start = __shfl_sync(0xffffffffu, my_start, k);
    int type = -1;
    const bool h = in_class(len, w.h_lo, w.h_hi), e = in_class(len, w.e_lo, w.e_hi),
               v = in_class(len, w.v_lo, w.v_hi);
    switch (cur) {
      case kHsync:
        if (h) type = kHsync;
        else if (e) {
          type = kEq1;
          pending = half;
        } else if (v) {
          vsync_seen = true;
          type = kVsync;
        }
        break;
      case kEq1:
        if (e) type = kEq1;
        else if (v) {
          vsync_seen = true;
          type = kVsync;
          pending = half;
        } else if (h) type = kHsync;
        break;
      case kVsync:
        if (e) {
          type = kEq2;
          pending = half;
        } else if (v) type = kVsync;
        else if ((long long)start > hold_floor && h) type = kHsync;
        break;
      case kEq2:
        if (e) type = kEq2;
        else if (h) {
          type = kHsync;
          done = true;
        }
        break;
    }
    bool kept = type >= 0;
    if (kept && type != cur) {
      if ((long long)start < hold_ceil) {
        kept = false;
      } else if (pending > 0.0) {
        const double hold = (double)start + ((pending - 0.1) * (double)line_len);
        hold_floor = (long long)floor(hold);
        hold_ceil = (long long)ceil(hold);
        pending = -1.0;
      }
    }
    if (kept) {
      keep_mask |= 1u << k;
      types |= (unsigned long long)type << (2 * k);
      cnt++;
      cur = type;
    }
    if (done && vsync_seen) break;
  }
  return WarpAttempt{done && cnt > 0, cnt, cur, keep_mask, types};
}

// Block-wide sum of a long long (kLT threads); every thread gets the total.
__device__ long long block_sum_ll(long long v, long long* sh) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  long long t = 0;
  for (int w = 0; w < kLT / 32; w++) t += sh[w];
  __syncthreads();
  return t;
}

// The validated pulses of one field, in global scratch (start, length,
// type | good << 2).
struct VList {
  int* s;
  int* l;
  unsigned char* tg;
  double* d;  // scratch doubles, one per entry
  int n;
};
__device__ __forceinline__ int vtype(const VList& v, int k) { return v.tg[k] & 3; }
__device__ __forceinline__ bool vgood(const VList& v, int k) { return (v.tg[k] >> 2) & 1; }

// Shared memory of a per-field CTA.
struct FieldSmem {
  int ps[kMaxPulses], pl[kMaxPulses];
  unsigned char cls[kMaxPulses];  // bit 0: hsync width, bit 1: attempt start
  int att_len[kMaxPulses];
  unsigned char att_ok[kMaxPulses], att_last[kMaxPulses];
  int pos[kMaxPulses + 1];
  long long red[kLT / 32];
  int imin, imax[12];
  double dsh[8];
  int ish[8];
  double sort[kSortMax];
  // the validated list when it has at most kSmemValid entries (nearly always)
  int vs[kSmemValid];
  unsigned char vt[kSmemValid];
  int nexth[kSmemValid];  // first non-hsync entry at or after each entry
};

// Pulse validation (pipeline.cu:611-648) into v; returns the entry count.
__device__ int validate(const LineLocArgs& a, FieldSmem& sm, int n, VList& v) {
  const Format& fmt = a.fmt;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  // width classes adapted to the field's mean hsync width (pipeline.cu:450-477)
  const double tol = fmt.fs_hz * 0.5e-6;
  const double loose_lo = fmt.hsync_width - 3.5 * tol, loose_hi = fmt.hsync_width + 4.0 * tol;
  long long lsum = 0, lcnt = 0;
  for (int i = t; i < n; i += kLT) {
    const double l = (double)sm.pl[i];
    if (l >= loose_lo && l <= loose_hi) {
      lsum += sm.pl[i];
      lcnt++;
    }
  }
  lsum = block_sum_ll(lsum, sm.red);
  lcnt = block_sum_ll(lcnt, sm.red);
  phase_clock(a, blockIdx.x, 21);
  const double est = lcnt > 0 ? ((double)lsum / (double)lcnt) : fmt.hsync_width;
  const double shift = est - fmt.hsync_width;
  Windows wd;
  const double hnom = fmt.hsync_width + shift;
  wd.h_lo = hnom - tol;
  wd.h_hi = hnom + tol;
  wd.e_lo = fmt.eq_pulse_width + shift - tol;
  wd.e_hi = fmt.eq_pulse_width + shift + tol;
  wd.v_lo = (fmt.vsync_width + shift) * 0.5;
  wd.v_hi = fmt.vsync_width + shift + 2.0 * tol;
  const IWindows w = int_windows(wd);
  // classes, then every recogniser attempt (one per EQ-width pulse), a warp
  // per attempt over a compacted list of them
  __shared__ int n_att;
  int* att_list = sm.pos;  // free until the placement scan
  if (t == 0) n_att = 0;
  __syncthreads();
  for (int i0 = 0; i0 < n; i0 += kLT) {
    const int i = i0 + t;
    bool e = false;
    if (i < n) {
      const int len = sm.pl[i];
      const bool h = in_class(len, w.h_lo, w.h_hi);
      e = !h && i > 2 && in_class(len, w.e_lo, w.e_hi);
      sm.cls[i] = (h ? 1 : 0) | (e ? 2 : 0);
      sm.att_ok[i] = 0;
      sm.att_len[i] = 0;
      sm.att_last[i] = (unsigned char)kHsync;
    }
    const unsigned m = __ballot_sync(0xffffffffu, e);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(&n_att, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (e) att_list[base + __popc(m & ((1u << lane) - 1u))] = i;
  }
  __syncthreads();
  for (int q = warp; q < n_att; q += kLT / 32) {
    const int i = att_list[q];
    const WarpAttempt r = attempt_warp(sm.ps, sm.pl, n, i - 2, w, fmt.num_eq_pulses, fmt.samples_per_line);
    if (lane == 0) {
      sm.att_ok[i] = r.ok ? 1 : 0;
      sm.att_len[i] = r.cnt;
      sm.att_last[i] = (unsigned char)r.last;
    }
  }
  __syncthreads();
  phase_clock(a, blockIdx.x, 22);
  // Which attempts fire: at an EQ-width pulse while the list's last entry is
  // an hsync.  The list's state before pulse i -- empty, last entry an hsync,
  // or last entry something else -- follows from pulse i-1's state by a map
  // of the three states (an hsync pulse sets "hsync"; a firing attempt sets
  // its last type; other pulses change nothing).  Composition is associative,
  // so the whole CTA scans the maps (each thread over a run of pulses), and
  // every pulse's output length and position follow from a second scan.
  auto pulse_map = [&](int i) -> unsigned {  // 2 bits per incoming state (0 empty, 1 hsync, 2 other)
    if (sm.cls[i] & 1) return 1u | (1u << 2) | (1u << 4);  // every state -> hsync
    if ((sm.cls[i] & 2) && sm.att_ok[i]) {
      const unsigned after = sm.att_last[i] == kHsync ? 1u : 2u;
      return 0u | (after << 2) | (2u << 4);  // fires only after an hsync
    }
    return 0u | (1u << 2) | (2u << 4);  // identity
  };
  auto apply = [](unsigned m, unsigned st) { return (m >> (2 * st)) & 3u; };
  auto compose = [&](unsigned first, unsigned then) {  // then(first(s))
    return apply(then, apply(first, 0)) | (apply(then, apply(first, 1)) << 2) | (apply(then, apply(first, 2)) << 4);
  };
  constexpr unsigned kIdentity = 0u | (1u << 2) | (2u << 4);
  __shared__ unsigned warp_map[kLT / 32];
  __shared__ int warp_len[kLT / 32];
  const int per = (n + kLT - 1) / kLT;
  const int i0 = min(n, t * per), i1 = min(n, i0 + per);
  unsigned m = kIdentity;
  for (int i = i0; i < i1; i++) m = compose(m, pulse_map(i));
  unsigned incl = m;
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned o = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl = compose(o, incl);
  }
  if (lane == 31) warp_map[warp] = incl;
  __syncthreads();
  unsigned before = kIdentity;  // the maps of every earlier warp
  for (int w2 = 0; w2 < warp; w2++) before = compose(before, warp_map[w2]);
  unsigned excl = __shfl_up_sync(0xffffffffu, incl, 1);
  if (lane == 0) excl = kIdentity;
  unsigned st = apply(compose(before, excl), 0);  // the list starts empty
  int len_sum = 0;
  for (int i = i0; i < i1; i++) {
    int len = 0;
    if (sm.cls[i] & 1) len = 1;
    else if ((sm.cls[i] & 2) && sm.att_ok[i] && st == 1) len = sm.att_len[i];
    sm.pos[i] = len;
    len_sum += len;
    st = apply(pulse_map(i), st);
  }
  int lincl = len_sum;
  for (int off = 1; off < 32; off <<= 1) {
    const int o = __shfl_up_sync(0xffffffffu, lincl, off);
    if (lane >= off) lincl += o;
  }
  if (lane == 31) warp_len[warp] = lincl;
  __syncthreads();
  int run = lincl - len_sum;
  for (int w2 = 0; w2 < warp; w2++) run += warp_len[w2];
  for (int i = i0; i < i1; i++) {
    const int len = sm.pos[i];
    sm.pos[i] = run;
    run += len;
  }
  if (t == kLT - 1) sm.pos[n] = run;  // the last thread ends at the total
  __syncthreads();
  phase_clock(a, blockIdx.x, 23);
  const int nv = sm.pos[n];
  // place every pulse's output: hsyncs one per thread, the attempts that
  // fire (a few per field) by a warp each, their kept steps written in order
  __shared__ int n_fire;
  __shared__ int fire_list[64];
  if (t == 0) n_fire = 0;
  __syncthreads();
  for (int i = t; i < n; i += kLT) {
    const int p = sm.pos[i], len = sm.pos[i + 1] - p;
    if (len <= 0) continue;
    if (sm.cls[i] & 1) {
      v.s[p] = sm.ps[i];
      v.l[p] = sm.pl[i];
      v.tg[p] = kHsync;
    } else {
      const int q = atomicAdd(&n_fire, 1);
      if (q < 64) {
        fire_list[q] = i;
      } else {  // more firing attempts than the list holds: this thread writes its own
        int cnt = 0, last = 0;
        attempt(sm.ps, sm.pl, n, i - 2, w, fmt.num_eq_pulses, fmt.samples_per_line, &cnt, &last, v.s + p, v.l + p,
                v.tg + p);
      }
    }
  }
  __syncthreads();
  for (int q = warp; q < min(n_fire, 64); q += kLT / 32) {
    const int i = fire_list[q];
    const int p = sm.pos[i];
    const WarpAttempt r = attempt_warp(sm.ps, sm.pl, n, i - 2, w, fmt.num_eq_pulses, fmt.samples_per_line);
    if ((r.keep >> lane) & 1u) {
      const int o = p + __popc(r.keep & ((1u << lane) - 1u));
      v.s[o] = sm.ps[i - 2 + lane];
      v.l[o] = sm.pl[i - 2 + lane];
      v.tg[o] = (unsigned char)((r.types >> (2 * lane)) & 3u);
    }
  }
  __syncthreads();
  phase_clock(a, blockIdx.x, 24);
  // cadence flags from each entry's predecessor (pipeline.cu:133-148)
  for (int k = t; k < nv; k += kLT) {
    const bool good = k > 0 && spacing_ok(vtype(v, k - 1), vtype(v, k), v.s[k] - v.s[k - 1], fmt.samples_per_line);
    v.tg[k] = (unsigned char)(vtype(v, k) | (good ? 4 : 0));
  }
  __syncthreads();
  phase_clock(a, blockIdx.x, 25);
  return nv;
}

// Mean line length from the longest hsync run (pipeline.cu:479-517): the
// first longest run; spacings within 5% of nominal, its last one excluded.
__device__ double mean_line(FieldSmem& sm, const VList& v, double nominal) {
  const int t = threadIdx.x;
  const bool in_smem = v.tg == sm.vt;
  if (in_smem) {
    // first non-hsync entry at or after each entry: a backward pass per
    // contiguous strip, then the strips' minima carried from the right
    __shared__ int strip_min[kLT];
    const int per = (v.n + kLT - 1) / kLT;
    const int k0 = min(v.n, t * per), k1 = min(v.n, k0 + per);
    int cur = INT_MAX;
    for (int k = k1 - 1; k >= k0; k--) {
      if (vtype(v, k) != kHsync) cur = k;
      sm.nexth[k] = cur;
    }
    strip_min[t] = cur;
    __syncthreads();
    if (t < 32) {  // suffix minimum over the strips, one warp
      const int q = (kLT + 31) / 32, a0 = t * q;
      int m = INT_MAX;
      for (int j = a0 + q - 1; j >= a0; j--) m = min(m, strip_min[j]);
      int suf = m;  // inclusive suffix minimum over lanes >= t
      for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_down_sync(0xffffffffu, suf, off);
        if (t + off < 32) suf = min(suf, o);
      }
      int carry = __shfl_down_sync(0xffffffffu, suf, 1);
      if (t == 31) carry = INT_MAX;
      for (int j = a0 + q - 1; j >= a0; j--) {
        const int own = strip_min[j];
        strip_min[j] = carry;  // minimum over the strips after j
        carry = min(carry, own);
      }
    }
    __syncthreads();
    for (int k = k0; k < k1; k++)
      if (sm.nexth[k] == INT_MAX) sm.nexth[k] = strip_min[t];
    __syncthreads();
  }
  // best run as (run_len << 32 | ~start): the largest run_len, then the first
  unsigned long long best = 0;
  bool any = false;
  for (int k = t; k < v.n; k += kLT) {
    if (vtype(v, k) != kHsync || (k > 0 && vtype(v, k - 1) == kHsync)) continue;
    int e;
    if (in_smem) {
      e = sm.nexth[k] == INT_MAX ? v.n : sm.nexth[k];
    } else {
      e = k + 1;
      while (e < v.n && vtype(v, e) == kHsync) e++;
    }
    const unsigned long long key = ((unsigned long long)(unsigned)(e - k - 1) << 32) | (0xFFFFFFFFu - (unsigned)k);
    if (!any || key > best) best = key;
    any = true;
  }
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_down_sync(0xffffffffu, best, off);
    best = o > best ? o : best;
  }
  __shared__ unsigned long long wbest[kLT / 32];
  if ((t & 31) == 0) wbest[t >> 5] = best;
  __syncthreads();
  unsigned long long b = 0;
  for (int w = 0; w < kLT / 32; w++) b = wbest[w] > b ? wbest[w] : b;
  __syncthreads();
  // a run exists iff the list holds an hsync; key 0 is only possible for a
  // single-entry run at index 0xFFFFFFFF, so test the list instead
  bool has_run = false;
  for (int k = t; k < v.n && !has_run; k += kLT) has_run = vtype(v, k) == kHsync;
  has_run = __syncthreads_or(has_run);
  const int best_len = has_run ? (int)(b >> 32) : -1;
  const int best_start = has_run ? (int)(0xFFFFFFFFu - (unsigned)(b & 0xFFFFFFFFu)) : -1;
  long long sum = 0, cnt = 0;
  if (best_start >= 1 && best_len >= 1) {
    for (int i = best_start + 1 + t; i < best_start + best_len; i += kLT) {
      const double l = (double)(v.s[i] - v.s[i - 1]);
      const double r = l / nominal;
      if (r >= 0.95 && r <= 1.05) {
        sum += v.s[i] - v.s[i - 1];
        cnt++;
      }
    }
  }
  sum = block_sum_ll(sum, sm.red);
  cnt = block_sum_ll(cnt, sm.red);
  return cnt == 0 ? nominal : (double)sum / (double)cnt;
}

// Vertical-blanking pulses and pattern agreement (pipeline.cu:650-716): each
// slot keeps its last match.
__device__ BlankingScan scan_blanking(FieldSmem& sm, const VList& v, double mll, const Format& fmt) {
  const int t = threadIdx.x;
  BlankingScan s;
  for (int i = 0; i < 8; i++) s.vb_pulse[i] = -1;
  for (int i = 0; i < 4; i++) s.order_len[i] = -1;
  s.agree = s.seen = 0.0;
  if (v.n == 0 || mll <= 0.0) return s;
  if (t == 0) sm.imin = INT_MAX;
  if (t < 12) sm.imax[t] = -1;
  __syncthreads();
  const double second = (double)v.s[0] + fmt.field_lines_first * mll;
  for (int i = 1 + t; i < v.n; i += kLT)
    if (vgood(v, i) && (double)v.s[i] > second) atomicMin(&sm.imin, i);
  __syncthreads();
  const int g0 = sm.imin;
  for (int i = 1 + t; i < v.n; i += kLT) {
    if (!vgood(v, i)) continue;
    const int grp = i >= g0 ? 4 : 0, fgrp = i >= g0 ? 2 : 0;
    const int pt = vtype(v, i - 1), ty = vtype(v, i);
    // slots 0..7 vb_pulse, 8..11 order_len
    if (pt == kHsync && ty > kHsync) {
      atomicMax(&sm.imax[0 + grp], i);
      atomicMax(&sm.imax[8 + 0 + fgrp], i);
    } else if (pt == kEq1 && ty == kVsync) {
      atomicMax(&sm.imax[1 + grp], i);
    } else if (pt == kVsync && ty == kEq2) {
      atomicMax(&sm.imax[2 + grp], i);
    } else if (pt > kHsync && ty == kHsync) {
      atomicMax(&sm.imax[3 + grp], i);
      atomicMax(&sm.imax[8 + 1 + fgrp], i);
    }
  }
  __syncthreads();
  for (int k = 0; k < 8; k++) {
    const int i = sm.imax[k];
    if (i < 0) continue;
    s.vb_pulse[k] = (k & 3) == 3 ? v.s[i - 1] : v.s[i];
  }
  for (int k = 0; k < 4; k++) {
    const int i = sm.imax[8 + k];
    if (i >= 0) s.order_len[k] = half_line_round((v.s[i] - v.s[i - 1]) / mll);
  }
  const double* first_pat = field_pattern(fmt.system, true);
  const double* second_pat = field_pattern(fmt.system, false);
  for (int i = 0; i < 4; i++) {
    if (s.order_len[i] == first_pat[i]) {
      s.agree += 1.0;
      s.seen += 1.0;
    }
    if (s.order_len[i] == second_pat[i]) s.seen += 1.0;
  }
  __syncthreads();
  return s;
}

// The blanking pattern's vote on the field order (pipeline.cu:729-745): the
// parts of the decision that need no carried state.
__device__ void pattern_vote(const BlankingScan& s, FieldPrep& p) {
  p.pat_default = (s.seen == 0.0 || round(s.agree / fmax(1.0, s.seen)) == 1.0) ? 1 : 0;
  p.c_first = p.c_second = 0;
  if (s.seen > 0.0) {
    const double weight = s.seen / 4.0;
    p.c_first = (int)llround((s.agree / s.seen) * weight * 100.0);
    p.c_second = (int)llround(((s.seen - s.agree) / s.seen) * weight * 100.0);
  }
}

// Field order from the previous field's and the vote (pipeline.cu:729-745).
__device__ bool decide_first(const FieldPrep& p, int prev_first, double prev_loc, int confidence) {
  bool first = prev_first == -1 ? p.pat_default != 0 : !prev_first;
  if (p.scan.seen > 0.0) {
    if (prev_loc < 0.0) confidence = min(confidence, 50);
    if (p.c_first >= confidence && p.c_first > p.c_second) first = true;
    else if (p.c_second >= confidence && p.c_second > p.c_first) first = false;
  }
  return first;
}

// The order the vote alone fixes, whatever the previous field: 1 first, 0
// second, -1 none.
__device__ int pattern_first(const FieldPrep& p, int confidence) {
  if (p.scan.seen <= 0.0) return -1;
  if (p.c_first >= confidence && p.c_first > p.c_second) return 1;
  if (p.c_second >= confidence && p.c_second > p.c_first) return 0;
  return -1;
}

// First-hsync anchor for field order `first` (pipeline.cu:650-855).  The
// pairwise estimates are formed one per thread and combined by thread 0 in the
// reference's order; the hsync-offset correction's terms are formed in
// parallel and added in list order by thread 0.  Every thread gets the result.
__device__ AnchorFit fit_anchor(FieldSmem& sm, const BlankingScan& s, const VList& v, double mll, const Format& fmt,
                                bool first, double prev_off_lines, double prev_loc, double prev_diff,
                                long long* clk = nullptr) {
  const int t = threadIdx.x;
  auto stamp = [&](int k) {
    if (clk && t == 0) clk[k] = clock64();
  };
  __shared__ AnchorFit res;
  __shared__ double loc_s;
  __shared__ int go_s;
  // pair estimates: 6 within each blanking interval, then 16 across them
  constexpr int kPairs = 28;
  __shared__ double pair_off[kPairs], pair_loc[kPairs];
  __shared__ unsigned char pair_ok[kPairs];
  const double cur_lines = first ? fmt.field_lines_first : fmt.field_lines_second;
  const double tol_lines = 0.5;
  const double section = fmt.num_eq_pulses / 2.0;
  const double* pat = field_pattern(fmt.system, first);
  double vb_line[8];
  vb_line[0] = 0.0 + pat[0];
  vb_line[1] = vb_line[0] + section;
  vb_line[2] = vb_line[1] + section;
  vb_line[3] = vb_line[2] + section - 0.5;
  const double hsync_line = vb_line[3] + pat[1];
  vb_line[4] = cur_lines + pat[2];
  vb_line[5] = vb_line[4] + section;
  vb_line[6] = vb_line[5] + section;
  vb_line[7] = vb_line[6] + section - 0.5;
  const bool any = v.n > 0 && mll > 0.0;
  if (any && t < kPairs) {
    // pair t in the reference's loop order: (x < y) over slots 0..3, the same
    // over slots 4..7, then (x, 4 + y) for x, y in 0..3
    int i1, i2;
    if (t < 12) {
      const int q = t % 6;
      const int x = q < 3 ? 0 : (q < 5 ? 1 : 2);
      const int y = q < 3 ? q + 1 : (q < 5 ? q - 1 : 3);
      i1 = x + (t < 6 ? 0 : 4);
      i2 = y + (t < 6 ? 0 : 4);
    } else {
      i1 = (t - 12) >> 2;
      i2 = 4 + ((t - 12) & 3);
    }
    const int p1 = s.vb_pulse[i1], p2 = s.vb_pulse[i2];
    bool ok = false;
    if (p1 != -1 && p2 != -1 && mll != 0.0) {
      const double actual = ((double)p1 - (double)p2) / mll;
      const double expect = vb_line[i1] - vb_line[i2];
      if (actual < expect + tol_lines && actual > expect - tol_lines) {
        ok = true;
        pair_off[t] = actual - expect;
        pair_loc[t] = (double)p2 + mll * (hsync_line - vb_line[i2]);
      }
    }
    pair_ok[t] = ok ? 1 : 0;
  }
  __syncthreads();
  stamp(26);
  if (t == 0) {
    AnchorFit out;
    go_s = 0;
    if (any) {
      const double pred_lines = predicted_field_lines(fmt, first);
      auto add = [&](int k, double& loc, int& cnt, double& off) {
        if (!pair_ok[k]) return;
        off += pair_off[k];
        loc += pair_loc[k];
        cnt += 1;
      };
      double a_loc = 0.0, a_off = 0.0, b_loc = 0.0, b_off = 0.0;
      int a_cnt = 0, b_cnt = 0;
      for (int k = 0; k < 6; k++) add(k, a_loc, a_cnt, a_off);
      for (int k = 6; k < 12; k++) add(k, b_loc, b_cnt, b_off);
      double loc = 0.0, off = 0.0;
      int cnt = 0;
      const double a_est = a_cnt ? a_loc / a_cnt : 0.0, b_est = b_cnt ? b_loc / b_cnt : 0.0;
      if (a_cnt && b_cnt && a_est < b_est + tol_lines * mll && a_est > b_est - tol_lines * mll) {
        loc = a_loc + b_loc;
        cnt = a_cnt + b_cnt;
        off = a_off + b_off;
        for (int k = 12; k < kPairs; k++) add(k, loc, cnt, off);
      } else if (a_cnt == 6 || (prev_loc <= 0.0 && a_cnt > b_cnt)) {
        loc = a_loc;
        cnt = a_cnt;
        off = a_off;
      } else if (b_cnt == 6 || (prev_loc <= 0.0 && b_cnt > a_cnt)) {
        loc = b_loc;
        cnt = b_cnt;
        off = b_off;
      }
      const int predicted = (int)llround((prev_off_lines + pred_lines + prev_loc / mll) * mll);
      if (cnt == 0 && prev_loc > 0.0) {
        double p = (prev_diff <= 0.5 && prev_diff >= -0.5) ? predicted + mll * prev_diff : (double)predicted;
        if (p <= 0.0) p = (double)v.s[0];
        loc += p;
        cnt += 1;
        out.used_prediction = true;
      }
      out.cnt = cnt;
      if (cnt > 0) {
        off /= cnt;
        loc = round((loc + off) / cnt);
        out.loc_round = loc;
        out.hsync_line = hsync_line;
        loc_s = loc;
        go_s = 1;
      }
    }
    res = out;
    sm.imin = INT_MAX;
  }
  __syncthreads();
  stamp(27);
  if (!go_s) {
    const AnchorFit r = res;
    __syncthreads();
    return r;
  }
  // hsync-offset correction: terms of the hsync entries before the first one
  // past the field's last line
  const double loc = loc_s;
  for (int k = t; k < v.n; k += kLT) {
    double term = __longlong_as_double(0x7ff8000000000000LL);  // NaN: not counted
    if (vtype(v, k) == kHsync && vgood(v, k)) {
      const double line = ((double)v.s[k] - loc) / mll + hsync_line;
      const int rl = (int)llround(line);
      if (rl > cur_lines) atomicMin(&sm.imin, k);
      else if (rl >= hsync_line) term = loc + mll * ((double)rl - hsync_line) - (double)v.s[k];
    }
    v.d[k] = term;
  }
  __syncthreads();
  stamp(28);
  // the counted terms packed in list order (a block scan over contiguous
  // strips), so the one thread that adds them in the reference's order reads
  // only counted terms
  const int end = min(sm.imin, v.n);
  double* packed = reinterpret_cast<double*>(sm.nexth);  // free once the mean line is known
  constexpr int kPackMax = kSmemValid / 2;
  int packed_n;
  {
    __shared__ int wsum[kLT / 32];
    const int per = (end + kLT - 1) / kLT;
    const int k0 = min(end, t * per), k1 = min(end, k0 + per);
    int cnt = 0;
    for (int k = k0; k < k1; k++) cnt += v.d[k] == v.d[k] ? 1 : 0;
    int incl = cnt;
    for (int off = 1; off < 32; off <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, incl, off);
      if ((t & 31) >= off) incl += o;
    }
    if ((t & 31) == 31) wsum[t >> 5] = incl;
    __syncthreads();
    int pre = incl - cnt;
    packed_n = 0;
    for (int w2 = 0; w2 < kLT / 32; w2++) {
      if (w2 < (t >> 5)) pre += wsum[w2];
      packed_n += wsum[w2];
    }
    if (packed_n <= kPackMax)
      for (int k = k0; k < k1; k++) {
        const double x = v.d[k];
        if (x == x) packed[pre++] = x;
      }
    __syncthreads();
  }
  if (t == 0) {
    double hoff = 0.0;
    int hcnt = 0;
    if (packed_n <= kPackMax) {
#pragma unroll 8
      for (int k = 0; k < packed_n; k++) hoff += packed[k];
      hcnt = packed_n;
    } else {
      for (int k = 0; k < end; k++) {
        const double x = v.d[k];
        if (x == x) {
          hoff += x;
          hcnt++;
        }
      }
    }
    double l = loc;
    if (hcnt > 0) {
      hoff /= hcnt;
      l -= hoff;
    }
    res.loc = l;
  }
  __syncthreads();
  stamp(29);
  const AnchorFit r = res;
  __syncthreads();
  return r;
}

// The carried hsync_diff after a fit that used no prediction.
__device__ double hsync_diff_after(const AnchorFit& f, const Format& fmt, bool first, double mll, double prev_off_lines,
                                   double prev_loc) {
  const int predicted = (int)llround((prev_off_lines + predicted_field_lines(fmt, first) + prev_loc / mll) * mll);
  return (f.loc_round - predicted) / mll;
}

// Sorted validated starts in sm.sort (bitonic, padded with +inf) or, past
// kSortMax entries, in v.d (insertion sort by thread 0).  Returns the array.
__device__ const double* sorted_starts(FieldSmem& sm, const VList& v) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (v.n <= kSortMax) {
    // The list is a few ascending runs (the recogniser re-emits the pulses
    // just before a blanking interval, and the walk then goes on from the
    // pulse after it): each entry's place is its index in its run plus, per
    // other run, the entries below it (an earlier run's equal entries first),
    // found by binary search -- a stable merge in one parallel pass.
    constexpr int kMaxRuns = 32;
    __shared__ int runs[kMaxRuns + 1];
    __shared__ int wcnt[kLT / 32];
    int nruns = 0;
    for (int k0 = 0; k0 < v.n; k0 += kLT) {
      const int k = k0 + t;
      const bool start = k < v.n && (k == 0 || v.s[k] < v.s[k - 1]);
      const unsigned m = __ballot_sync(0xffffffffu, start);
      if (lane == 0) wcnt[warp] = __popc(m);
      __syncthreads();
      int before = 0, total = 0;
      for (int w = 0; w < kLT / 32; w++) {
        if (w < warp) before += wcnt[w];
        total += wcnt[w];
      }
      if (start) {
        const int r = nruns + before + __popc(m & ((1u << lane) - 1u));
        if (r < kMaxRuns) runs[r] = k;
      }
      nruns += total;
      __syncthreads();
    }
    if (nruns <= kMaxRuns) {
      if (t == 0) runs[nruns] = v.n;
      __syncthreads();
      for (int k = t; k < v.n; k += kLT) {
        const int x = v.s[k];
        int lo = 0, hi = nruns;  // the run holding k: last start <= k
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (runs[mid] <= k) lo = mid;
          else hi = mid;
        }
        const int r = lo;
        int rank = k - runs[r];
        for (int q = 0; q < nruns; q++) {
          if (q == r) continue;
          int b = runs[q], e = runs[q + 1];  // entries of run q below x (at most x for an earlier run)
          while (b < e) {
            const int mid = (b + e) >> 1;
            const bool below = q < r ? v.s[mid] <= x : v.s[mid] < x;
            if (below) b = mid + 1;
            else e = mid;
          }
          rank += b - runs[q];
        }
        sm.sort[rank] = (double)x;
      }
      __syncthreads();
      return sm.sort;
    }
    int m = 1;
    while (m < v.n) m <<= 1;
    for (int k = t; k < m; k += kLT) sm.sort[k] = k < v.n ? (double)v.s[k] : __longlong_as_double(0x7ff0000000000000LL);
    __syncthreads();
    for (int size = 2; size <= m; size <<= 1)
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int k = t; k < m; k += kLT) {
          const int j = k ^ stride;
          if (j > k) {
            const bool up = (k & size) == 0;
            const double x = sm.sort[k], y = sm.sort[j];
            if ((x > y) == up) {
              sm.sort[k] = y;
              sm.sort[j] = x;
            }
          }
        }
        __syncthreads();
      }
    return sm.sort;
  }
  if (t == 0) {
    for (int k = 0; k < v.n; k++) v.d[k] = (double)v.s[k];
    for (int a = 1; a < v.n; a++) {  // nearly sorted already
      const double x = v.d[a];
      int b = a;
      while (b > 0 && v.d[b - 1] > x) {
        v.d[b] = v.d[b - 1];
        b--;
      }
      v.d[b] = x;
    }
  }
  __syncthreads();
  return v.d;
}

// Nominal line grid snapped to the nearest pulse (pipeline.cu:857-893).
//
// The reference walks the lines with a cursor into the sorted starts: from
// the cursor it steps right while the distance to the line's nominal position
// does not grow, takes the last position checked (the walk checks no position
// past the second-to-last) if it is within mll / 1.5, and moves the cursor
// past it.  The distances to sorted starts fall to a minimum and then grow, so
// from any cursor at or before S -- the first index whose successor is
// strictly farther -- the walk stops at S.  Each thread therefore finds S of
// its lines by binary search; one warp then carries the cursor over the lines,
// 32 at a time: while every line meets a cursor at or before its S, the cursor
// is a running maximum (a warp scan), and a line whose S lies behind the
// cursor (its pulse taken by an earlier line) is walked from the cursor by one
// lane, as the reference does.
__device__ void snap_lines(FieldSmem& sm, const VList& v, double ref_pos, double ref_line, double mll, int nlines,
                           double* locs, long long* clk = nullptr) {
  const double* ps = sorted_starts(sm, v);
  const int t = threadIdx.x, np = v.n;
  if (clk && t == 0) clk[30] = clock64();
  const double max_dist = mll / 1.5;
  int* stop = sm.pos;      // per line: S capped at np - 2, << 1 | within max_dist
  int* taken = sm.att_len; // per line: the pulse it snaps to, or -1
  auto expect_of = [&](int line) { return ref_pos + mll * ((double)line - ref_line); };
  auto dist = [&](int i, double e) { return fabs(ps[i] - e); };
  if (np >= 2) {
    for (int line = t; line < nlines; line += kLT) {
      const double e = expect_of(line);
      int lo = 0, hi = np;  // first start strictly after e
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ps[mid] - e > 0.0) hi = mid;
        else lo = mid + 1;
      }
      int sx;
      if (lo >= 1 && lo < np && dist(lo, e) > dist(lo - 1, e)) {
        sx = lo - 1;
      } else {
        sx = min(lo, np - 1);
        while (sx + 1 < np && !(dist(sx + 1, e) > dist(sx, e))) sx++;
      }
      sx = min(sx, np - 2);
      stop[line] = (sx << 1) | (dist(sx, e) <= max_dist ? 1 : 0);
      taken[line] = -1;
    }
  }
  __syncthreads();
  if (clk && t == 0) clk[31] = clock64();
  if (t < 32) {
    const int lane = t;
    int cur = 0;
    // a cursor at the last start (or past it) takes no more pulses: the walk ends
    for (int g = 0; g < nlines && cur < np - 1; g += 32) {
      const int line = g + lane;
      const bool in = line < nlines && np >= 2;
      const int code = in ? stop[line] : 0;
      const int sx = code >> 1;
      const bool near = (code & 1) != 0;
      int k = 0;  // lanes below k are settled
      while (k < 32 && g + k < nlines && cur < np - 1) {
        // cursor met by each lane if lanes k .. lane-1 all stop at their S
        int incl = (in && lane >= k && near) ? sx + 1 : INT_MIN;
        for (int off = 1; off < 32; off <<= 1) {
          const int o = __shfl_up_sync(0xffffffffu, incl, off);
          if (lane >= off) incl = max(incl, o);
        }
        int excl = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) excl = INT_MIN;
        const int c = max(cur, excl);
        const unsigned behind = __ballot_sync(0xffffffffu, in && lane >= k && c > sx);
        const int kb = behind ? __ffs(behind) - 1 : 32;
        if (lane >= k && lane < kb && line < nlines) taken[line] = (in && near) ? sx : -1;
        const int settled = __shfl_sync(0xffffffffu, max(cur, incl), max(kb - 1, 0));
        if (kb > k) cur = settled;
        if (kb >= 32 || g + kb >= nlines) break;
        // line g + kb: its pulse is behind the cursor; walk from the cursor
        int nc = cur;
        if (lane == kb) {
          int got = -1;
          if (cur < np - 1) {
            const double e = expect_of(line);
            int w = cur;
            while (w + 1 < np && !(dist(w + 1, e) > dist(w, e))) w++;
            w = min(w, np - 2);
            if (dist(w, e) <= max_dist) {
              got = w;
              nc = w + 1;
            }
          }
          taken[line] = got;
        }
        cur = __shfl_sync(0xffffffffu, nc, kb);
        k = kb + 1;
      }
    }
  }
  __syncthreads();
  for (int line = t; line < nlines; line += kLT) {
    const int k = np >= 2 ? taken[line] : -1;
    locs[line] = k >= 0 ? ps[k] : expect_of(line);
  }
  __syncthreads();
}

__device__ VList field_vlist(const LineLocArgs& a, int f) {
  VList v;
  const size_t o = (size_t)f * kMaxValid;
  v.s = a.vs + o;
  v.l = a.vl + o;
  v.tg = a.vt + o;
  v.d = a.vd + o;
  v.n = a.vn[f];
  return v;
}

// Grid (num_fields): the stateless part of one field's line location, and
// the speculative anchor + grid when the field's pattern fixes its order.
template <class Src>
__global__ void __launch_bounds__(kLT, 1) prepare_kernel(const __grid_constant__ Src src) {
  const LineLocArgs& a = src.get();
  chain_wait();
  extern __shared__ double smem_d[];
  FieldSmem& sm = *reinterpret_cast<FieldSmem*>(smem_d);
  const int f = blockIdx.x, t = threadIdx.x;
  if (f >= a.win->fields) return;
  phase_clock(a, f, 0);
  const int n = min(max(a.pn[f], 0), kMaxPulses);
  for (int i = t; i < n; i += kLT) {
    sm.ps[i] = a.ps[(size_t)f * kMaxPulses + i];
    sm.pl[i] = a.pl[(size_t)f * kMaxPulses + i];
  }
  __syncthreads();
  phase_clock(a, f, 1);
  VList vg = field_vlist(a, f);
  vg.n = n > 0 ? validate(a, sm, n, vg) : 0;
  phase_clock(a, f, 2);
  if (t == 0) a.vn[f] = vg.n;
  VList v = vg;
  if (vg.n <= kSmemValid) {  // work from shared memory
    for (int k = t; k < vg.n; k += kLT) {
      sm.vs[k] = vg.s[k];
      sm.vt[k] = vg.tg[k];
    }
    v.s = sm.vs;
    v.tg = sm.vt;
    v.d = sm.sort;  // anchor-offset terms; the sort that reuses it comes after
    __syncthreads();
  }
  phase_clock(a, f, 3);
  const double mll = mean_line(sm, v, (double)a.fmt.samples_per_line);
  phase_clock(a, f, 4);
  const BlankingScan scan = scan_blanking(sm, v, mll, a.fmt);
  phase_clock(a, f, 5);
  FieldPrep p;
  p.mll = mll;
  p.n_raw = n;
  p.vn = vg.n;
  p.raw0 = n > 0 ? (double)sm.ps[0] : 0.0;
  p.scan = scan;
  p.spec_first = -1;
  pattern_vote(scan, p);
  const int pf = v.n > 0 ? pattern_first(p, kAnchorConfidence) : -1;
  if (f == 0) {
    // the chunk's first field: its incoming state is the chunk's, so the
    // in-order pass's fit is computed here
    const LineLocState st = *a.state;
    p.exact = 1;
    if (v.n > 0 && mll > 0.0) {
      const bool first = decide_first(p, st.prev_first_field, st.prev_first_hsync_loc, kAnchorConfidence);
      const long long readloc = a.raw_offset + a.offs[0];
      const double prev_off = (st.prev_first_hsync_readloc != -1 && mll > 0.0)
                                  ? ((double)st.prev_first_hsync_readloc - (double)readloc) / mll
                                  : 0.0;
      const AnchorFit fit = fit_anchor(sm, scan, v, mll, a.fmt, first, prev_off, st.prev_first_hsync_loc,
                                       st.prev_first_hsync_diff, a.dbg_clk ? a.dbg_clk + (size_t)f * kPhaseSlots : nullptr);
      phase_clock(a, f, 6);
      if (fit.cnt > 0)
        snap_lines(sm, v, fit.loc, fit.hsync_line, mll, a.fmt.lines_per_frame, a.ll + (size_t)f * a.fmt.lines_per_frame,
                   a.dbg_clk ? a.dbg_clk + (size_t)f * kPhaseSlots : nullptr);
      phase_clock(a, f, 7);
      p.exact_first = first ? 1 : 0;
      p.spec = fit;
    }
  } else if (pf >= 0) {
    const AnchorFit fit = fit_anchor(sm, scan, v, mll, a.fmt, pf == 1, 0.0, 1.0, 0.0,
                                     a.dbg_clk ? a.dbg_clk + (size_t)f * kPhaseSlots : nullptr);
    phase_clock(a, f, 6);
    if (fit.cnt > 0 && !fit.used_prediction) {
      snap_lines(sm, v, fit.loc, fit.hsync_line, mll, a.fmt.lines_per_frame, a.ll + (size_t)f * a.fmt.lines_per_frame,
                 a.dbg_clk ? a.dbg_clk + (size_t)f * kPhaseSlots : nullptr);
      p.spec_first = pf;
      p.spec = fit;
    }
    phase_clock(a, f, 7);
  }
  if (t == 0) a.prep[f] = p;
  phase_clock(a, f, 8);
  if (a.dbg_clk && t == 0) {
    a.dbg_clk[(size_t)f * kPhaseSlots + 9] = vg.n;
    a.dbg_clk[(size_t)f * kPhaseSlots + 10] = pf;
    a.dbg_clk[(size_t)f * kPhaseSlots + 11] = n;
  }
  // validated pulses for inspection (the first kMaxPulses)
  if (a.dbg_vn) {
    const int kept = min(v.n, kMaxPulses);
    for (int k = t; k < kept; k += kLT) {
      a.dbg_vs[(size_t)f * kMaxPulses + k] = v.s[k];
      a.dbg_vl[(size_t)f * kMaxPulses + k] = v.l[k];
      a.dbg_vt[(size_t)f * kMaxPulses + k] = vtype(v, k);
    }
    if (t == 0) a.dbg_vn[f] = kept;
  }
}

// One CTA: the fields in order with the carried state (pipeline.cu:1717-1778).
// Thread 0 walks the fields' records (fetched kPrepBatch at a time into shared
// memory) with the state in shared memory: where a field's speculative grid
// stands -- its pattern fixed the order the walk decides, and a previous field
// anchored the capture -- the step is a few integer decisions.  A field that
// needs its anchor fitted (the capture's first field, or an order its own
// pattern did not fix) stops the walk; the whole CTA fits and snaps it from
// its validated list staged in shared memory, and the walk goes on.  The
// carried hsync difference, a few FP64 divisions, is formed only when a fit
// or the next chunk reads it.
constexpr int kPrepBatch = 64;
template <class Src>
__global__ void __launch_bounds__(kLT, 1) finish_kernel(const __grid_constant__ Src src) {
  const LineLocArgs& a = src.get();
  chain_wait();
  extern __shared__ double smem_d[];
  FieldSmem& sm = *reinterpret_cast<FieldSmem*>(smem_d);
  __shared__ FieldPrep preps[kPrepBatch];
  __shared__ long long readlocs[kPrepBatch];
  __shared__ unsigned char fallback[kPrepBatch];
  __shared__ int fit_j, fit_first;
  __shared__ double prev_off_s, prev_loc_s, prev_diff_s;
  const int t = threadIdx.x;
  const int P = a.win->fields;
  const int LPF = a.fmt.lines_per_frame;
  // The carried state lives in thread 0's registers for the whole walk.
  // The hsync difference is formed only when a fit or the next chunk reads
  // it: from the last anchored field's rounded anchor, mll, order, the
  // previous anchor's read location and location, and its own read location.
  LineLocState st;
  bool diff_due = false;
  double d_round = 0.0, d_mll = 0.0, d_prev_loc = 0.0;
  long long d_prev_read = -1, d_read = 0;
  bool d_first = false;
  auto prev_off_of = [&](long long prev_read, long long read, double mll) {
    return (prev_read != -1 && mll > 0.0) ? ((double)prev_read - (double)read) / mll : 0.0;
  };
  auto settle_diff = [&]() {
    if (!diff_due) return;
    AnchorFit f;
    f.loc_round = d_round;
    st.prev_first_hsync_diff =
        hsync_diff_after(f, a.fmt, d_first, d_mll, prev_off_of(d_prev_read, d_read, d_mll), d_prev_loc);
    diff_due = false;
  };
  // a field anchored with this order and fit (from the per-field pass or a fit here)
  auto anchored = [&](int f, long long readloc, bool first, const AnchorFit& fit, double mll, bool diff_lazy,
                      double prev_off) {
    a.is_first[f] = first ? 1 : 0;
    if (!fit.used_prediction) {
      if (diff_lazy) {
        diff_due = true;
        d_round = fit.loc_round;
        d_mll = mll;
        d_first = first;
        d_prev_read = st.prev_first_hsync_readloc;
        d_prev_loc = st.prev_first_hsync_loc;
        d_read = readloc;
      } else {
        diff_due = false;
        st.prev_first_hsync_diff = hsync_diff_after(fit, a.fmt, first, mll, prev_off, st.prev_first_hsync_loc);
      }
    }
    st.prev_first_field = first ? 1 : 0;
    st.prev_progressive_field = 0;
    st.prev_first_hsync_readloc = readloc;
    st.prev_first_hsync_loc = fit.loc;
  };
  if (t == 0) st = *a.state;
  if (P > 0) phase_clock(a, 0, 16);
  for (int b0 = 0; b0 < P; b0 += kPrepBatch) {
    const int nb = min(kPrepBatch, P - b0);
    __syncthreads();  // the previous batch's records are no longer read
    for (int i = t; i < nb; i += kLT) {
      preps[i] = a.prep[b0 + i];
      readlocs[i] = a.raw_offset + a.offs[b0 + i];
      fallback[i] = 0;
    }
    __syncthreads();
    int j = 0;
    while (j < nb) {
      if (t == 0) {
        for (; j < nb; j++) {
          const int f = b0 + j;
          const FieldPrep& p = preps[j];
          const long long readloc = readlocs[j];
          if (!(p.vn > 0 && p.mll > 0.0)) {
            a.is_first[f] = st.prev_first_field >= 0 ? (1 - st.prev_first_field) : 1;
            fallback[j] = 1;
            continue;
          }
          if (p.exact) {  // fitted with this state by the per-field pass
            if (p.spec.cnt > 0) {
              anchored(f, readloc, p.exact_first != 0, p.spec, p.mll, true, 0.0);
            } else {
              a.is_first[f] = st.prev_first_field >= 0 ? (1 - st.prev_first_field) : 1;
              fallback[j] = 1;
            }
            continue;
          }
          const double prev_loc = st.prev_first_hsync_loc;
          const bool first = decide_first(p, st.prev_first_field, prev_loc, kAnchorConfidence);
          if (!(p.spec_first == (first ? 1 : 0) && prev_loc > 0.0)) {
            // fit this field: the previous state is final up to here
            settle_diff();
            fit_first = first;
            prev_off_s = prev_off_of(st.prev_first_hsync_readloc, readloc, p.mll);
            prev_loc_s = prev_loc;
            prev_diff_s = st.prev_first_hsync_diff;
            break;
          }
          anchored(f, readloc, first, p.spec, p.mll, true, 0.0);  // the speculative anchor stands
        }
        fit_j = j;
      }
      __syncthreads();
      j = fit_j;
      if (j >= nb) break;
      // field b0 + j: fit and snap with the whole CTA
      const int f = b0 + j;
      const FieldPrep& p = preps[j];
      VList v = field_vlist(a, f);
      if (v.n <= kSmemValid) {
        for (int k = t; k < v.n; k += kLT) {
          sm.vs[k] = v.s[k];
          sm.vt[k] = v.tg[k];
        }
        v.s = sm.vs;
        v.tg = sm.vt;
        v.d = sm.sort;  // anchor-offset terms; the sort that reuses it comes after
        __syncthreads();
      }
      phase_clock(a, f, 17);
      const AnchorFit fit = fit_anchor(sm, p.scan, v, p.mll, a.fmt, fit_first != 0, prev_off_s, prev_loc_s, prev_diff_s);
      phase_clock(a, f, 18);
      if (fit.cnt > 0) snap_lines(sm, v, fit.loc, fit.hsync_line, p.mll, LPF, a.ll + (size_t)f * LPF);
      phase_clock(a, f, 19);
      if (t == 0) {
        if (fit.cnt > 0) {
          anchored(f, readlocs[j], fit_first != 0, fit, p.mll, false, prev_off_s);
        } else {
          a.is_first[f] = st.prev_first_field >= 0 ? (1 - st.prev_first_field) : 1;
          fallback[j] = 1;
        }
      }
      j++;
      __syncthreads();
    }
    // fields with no anchor: the nominal grid from their first pulse
    for (int jj = 0; jj < nb; jj++) {
      if (!fallback[jj]) continue;
      double* locs = a.ll + (size_t)(b0 + jj) * LPF;
      for (int line = t; line < LPF; line += kLT) locs[line] = preps[jj].raw0 + preps[jj].mll * (double)line;
    }
  }
  if (t == 0) {
    settle_diff();
    *a.state = st;
  }
  if (P > 0) phase_clock(a, 0, 20);
}

// ------------------------------------------------------------ single pass

// Grid (num_fields): the reference's single-pass locator (line_locs.cu:62-543)
// for one field: width classes adapted to the field's mean hsync width, the
// blanking state machine for the reference pulse and the parity, the mean
// line from the longest hsync run, and the nominal grid snapped to the
// nearest hsync marker.  No carried state.
template <class Src>
__global__ void __launch_bounds__(kLT) single_pass_kernel(const __grid_constant__ Src src) {
  const LineLocArgs& a = src.get();
  chain_wait();
  extern __shared__ double smem_d[];
  FieldSmem& sm = *reinterpret_cast<FieldSmem*>(smem_d);
  __shared__ int mk_s[kMaxPulses], mk_l[kMaxPulses], hs[kMaxPulses];
  __shared__ int warp_cnt[kLT / 32];
  __shared__ double ref_pos_s, ref_line_s, mll_s;
  __shared__ int nm_s;
  const int f = blockIdx.x, t = threadIdx.x;
  if (f >= a.win->fields) return;
  const Format& fmt = a.fmt;
  const int n = min(max(a.pn[f], 0), kMaxPulses);
  for (int i = t; i < n; i += kLT) {
    sm.ps[i] = a.ps[(size_t)f * kMaxPulses + i];
    sm.pl[i] = a.pl[(size_t)f * kMaxPulses + i];
  }
  __syncthreads();
  const int* starts = sm.ps;
  const int* lengths = sm.pl;
  unsigned char* type = sm.cls;
  const double tol = 0.5e-6 * fmt.fs_hz;
  const double inl = (double)fmt.samples_per_line;
  const double hnom = fmt.hsync_width, enom = fmt.eq_pulse_width, vnom = fmt.vsync_width;
  // width classes shifted by the field's mean hsync width (line_locs.cu:99-135)
  const double loose_lo = fma(-3.5, tol, hnom), loose_hi = fma(4.0, tol, hnom);
  long long hsum = 0, hcnt = 0;
  for (int i = t; i < n; i += kLT) {
    const double len = (double)lengths[i];
    if (len >= loose_lo && len <= loose_hi) {
      hsum += lengths[i];
      hcnt++;
    }
  }
  hsum = block_sum_ll(hsum, sm.red);
  hcnt = block_sum_ll(hcnt, sm.red);
  const double shift = (hcnt > 0 ? (double)hsum / (double)hcnt : hnom) - hnom;
  const double h_lo = hnom + shift - tol, h_hi = hnom + shift + tol;
  const double e_lo = enom + shift - tol, e_hi = enom + shift + tol;
  const double v_lo = (vnom + shift) * 0.5, v_hi = fma(2.0, tol, vnom + shift);
  for (int i = t; i < n; i += kLT) {
    const double len = (double)lengths[i];
    unsigned char ty = kHsync;  // unclassified widths count as hsync
    if (len >= v_lo && len <= v_hi) ty = kVsync;
    else if (len >= h_lo && len <= h_hi) ty = kHsync;
    else if (len >= e_lo && len <= e_hi) ty = kEq1;
    type[i] = ty;
  }
  __syncthreads();
  if (t == 0) {
    // blanking state machine: the first hsync after the vertical interval (line_locs.cu:148-201)
    int ref = -1, last_h = -1, first_eq = -1, last_eq2 = -1, state = -1;
    for (int i = 0; i < n; i++) {
      const int ty = type[i];
      if (state == -1) {
        if (ty == kHsync) {
          state = kHsync;
          last_h = i;
        }
      } else if (state == kHsync) {
        if (ty == kHsync) last_h = i;
        else if (ty == kEq1) {
          state = kEq1;
          first_eq = i;
        } else if (ty == kVsync) state = kVsync;
      } else if (state == kEq1) {
        if (ty == kVsync) state = kVsync;
        else if (ty == kHsync) {
          state = kHsync;
          last_h = i;
          first_eq = -1;
        }
      } else if (state == kVsync) {
        if (ty == kEq1) {
          state = kEq2;
          last_eq2 = i;
        } else if (ty == kHsync) {
          ref = i;
          break;
        }
      } else if (state == kEq2) {
        if (ty == kEq1) last_eq2 = i;
        else if (ty == kHsync) {
          if (last_eq2 < 0) last_eq2 = i - 1;
          ref = i;
          break;
        }
      }
    }
    // field parity from the half-line spacing entering or leaving the interval (line_locs.cu:203-236)
    const bool ntsc = fmt.system == kNtsc;
    int par = -1;
    if (ref >= 0 && last_h >= 0 && first_eq >= 0) {
      const double lines = (double)(starts[first_eq] - starts[last_h]) / inl;
      par = ntsc ? (lines > 0.75 ? 1 : 0) : (lines > 0.75 ? 0 : 1);
    }
    if (par < 0 && ref >= 0 && last_eq2 >= 0) {
      const double lines = (double)(starts[ref] - starts[last_eq2]) / inl;
      par = ntsc ? (lines > 0.75 ? 1 : 0) : (lines > 0.75 ? 0 : 1);
    }
    a.is_first[f] = par;
    // mean line length over the longest hsync run (line_locs.cu:246-284)
    int best_s = -1, best_n = 0, cur_s = -1, cur_n = 0;
    for (int i = 0; i < n; i++) {
      if (type[i] == kHsync) {
        if (cur_s == -1) {
          cur_s = i;
          cur_n = 1;
        } else {
          cur_n++;
        }
      } else {
        if (cur_n > best_n) {
          best_s = cur_s;
          best_n = cur_n;
        }
        cur_s = -1;
        cur_n = 0;
      }
    }
    if (cur_n > best_n) {
      best_s = cur_s;
      best_n = cur_n;
    }
    double mll = inl;
    if (best_n >= 2) {
      long long sum = 0;
      int cnt = 0;
      for (int i = best_s + 1; i < best_s + best_n; i++) {
        const double sp = (double)(starts[i] - starts[i - 1]);
        if (sp >= inl * 0.95 && sp <= inl * 1.05) {
          sum += starts[i] - starts[i - 1];
          cnt++;
        }
      }
      if (cnt > 0) mll = (double)sum / cnt;
    }
    // reference position and line (line_locs.cu:295-337)
    double ref_pos, ref_line;
    if (ref >= 0) {
      ref_pos = (double)starts[ref];
      ref_line = 10.0;
      if (ref > n / 2) {
        const double back = ref_pos - (double)fmt.samples_per_field;
        if (back > 0.0) ref_pos = back;
      }
    } else {
      ref = 0;
      for (int i = 0; i < n; i++)
        if (type[i] == kHsync) {
          ref = i;
          break;
        }
      ref_pos = n > 0 ? (double)starts[ref] : 0.0;
      ref_line = 0.0;
    }
    ref_pos_s = ref_pos;
    ref_line_s = ref_line;
    mll_s = mll;
  }
  __syncthreads();
  // line markers: an EQ pulse followed closely by a tiny hsync fragment stands
  // for the line, and the fragment is dropped (line_locs.cu:365-399); ordered compaction
  const double tiny = hnom * 0.75, gap = inl * 0.25;
  int base = 0;
  for (int i0 = 0; i0 < n; i0 += kLT) {
    const int i = i0 + t;
    bool keep = false;
    if (i < n) {
      const bool eq = type[i] == kEq1 || type[i] == kEq2;
      const bool surrogate = eq && i + 1 < n && type[i + 1] == kHsync && (double)lengths[i + 1] <= tiny &&
                             (double)(starts[i + 1] - starts[i]) <= gap;
      const bool fragment = type[i] == kHsync && (double)lengths[i] <= tiny && i > 0 &&
                            (type[i - 1] == kEq1 || type[i - 1] == kEq2) && (double)(starts[i] - starts[i - 1]) <= gap;
      keep = surrogate || (type[i] == kHsync && !fragment);
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if ((t & 31) == 0) warp_cnt[t >> 5] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < kLT / 32; w++) {
      if (w < (t >> 5)) before += warp_cnt[w];
      total += warp_cnt[w];
    }
    if (keep) {
      const int k = base + before + __popc(m & ((1u << (t & 31)) - 1u));
      mk_s[k] = starts[i];
      mk_l[k] = lengths[i];
    }
    base += total;
    __syncthreads();
  }
  if (t == 0) {
    // one marker per line interval: the one nearest the nominal hsync width (line_locs.cu:401-425)
    const double dup = inl * 0.75;
    const int nm = base;
    int nh = 0;
    for (int c0 = 0; c0 < nm;) {
      int best = c0;
      double score = fabs((double)mk_l[c0] - hnom);
      int c1 = c0 + 1;
      while (c1 < nm && (double)(mk_s[c1] - mk_s[c0]) < dup) {
        const double sc = fabs((double)mk_l[c1] - hnom);
        if (sc < score || (sc == score && mk_s[c1] < mk_s[best])) {
          best = c1;
          score = sc;
        }
        c1++;
      }
      hs[nh++] = mk_s[best];
      c0 = c1;
    }
    nm_s = nh;
    // nominal grid snapped to the nearest marker ahead of a monotonic cursor (line_locs.cu:429-470)
    const double mll = mll_s, ref_pos = ref_pos_s, ref_line = ref_line_s;
    const double max_d = mll / 1.5;
    double* locs = a.ll + (size_t)f * fmt.lines_per_frame;
    int cur = 0;
    for (int line = 0; line < fmt.lines_per_frame; line++) {
      const double expected = fma(mll, (double)line - ref_line, ref_pos);
      locs[line] = expected;
      if (cur >= nh) continue;
      double best_d = max_d;
      int best_pos = -1;
      for (int s = cur; s < nh; s++) {
        const double d = fabs((double)hs[s] - expected);
        if (d <= best_d) {
          best_d = d;
          best_pos = hs[s];
          cur = s;
        }
        if (s + 1 < nh) {
          if (fabs((double)hs[s + 1] - expected) > d) break;
        } else {
          break;
        }
      }
      if (best_pos >= 0) {
        locs[line] = (double)best_pos;
        cur++;
      }
    }
  }
  // the raw pulses with their nominal classes stand for the validated list
  // when inspected (line_locs.cu:18-49 with the thresholds of :551-558)
  if (a.dbg_vn) {
    const double ntol = 0.5e-6 * fmt.fs_hz;
    for (int i = t; i < n; i += kLT) {
      const double len = (double)lengths[i];
      int ty = kHsync;
      if (len >= fmt.vsync_width * 0.5 && len <= fmt.vsync_width + 1.0e-6 * fmt.fs_hz) ty = kVsync;
      else if (len >= fmt.hsync_width - ntol && len <= fmt.hsync_width + ntol) ty = kHsync;
      else if (len >= fmt.eq_pulse_width - ntol && len <= fmt.eq_pulse_width + ntol) ty = kEq1;
      a.dbg_vs[(size_t)f * kMaxPulses + i] = starts[i];
      a.dbg_vl[(size_t)f * kMaxPulses + i] = lengths[i];
      a.dbg_vt[(size_t)f * kMaxPulses + i] = ty;
    }
    if (t == 0) a.dbg_vn[f] = n;
  }
}

}  // namespace

size_t lineloc_smem_bytes() { return sizeof(FieldSmem); }

namespace {
template <class S>
cudaError_t windows_launch(const S& src, int portions, cudaStream_t st) {
  const size_t smem = fieldwin_smem_bytes();
  const cudaError_t e =
      cudaFuncSetAttribute(fieldwin_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return launch_chained(fieldwin_kernel<S>, dim3(1, 1, portions), dim3(kWinThreads), smem, st, src);
}

template <class S>
cudaError_t pulses_launch(const S& src, int portions, int max_fields, cudaStream_t st) {
  if (max_fields <= 0) return cudaSuccess;
  return launch_chained(pulses_kernel<S>, dim3(max_fields, 1, portions), dim3(kLT), 0, st, src);
}

template <class S>
cudaError_t lines_launch(const S& src, bool single_pass, int portions, int max_fields, cudaStream_t st) {
  if (max_fields <= 0) return cudaSuccess;
  const size_t smem = sizeof(FieldSmem);
  cudaError_t e;
  if (single_pass) {
    e = cudaFuncSetAttribute(single_pass_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return launch_chained(single_pass_kernel<S>, dim3(max_fields, 1, portions), dim3(kLT), smem, st, src);
  }
  e = cudaFuncSetAttribute(prepare_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(finish_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = launch_chained(prepare_kernel<S>, dim3(max_fields, 1, portions), dim3(kLT), smem, st, src);
  if (e != cudaSuccess) return e;
  return launch_chained(finish_kernel<S>, dim3(1, 1, portions), dim3(kLT), smem, st, src);
}
}  // namespace

cudaError_t launch_field_windows(const LineLocArgs& a, cudaStream_t st) {
  return windows_launch(ArgsOne<LineLocArgs>{a}, 1, st);
}

cudaError_t launch_field_pulses(const LineLocArgs& a, cudaStream_t st) {
  return pulses_launch(ArgsOne<LineLocArgs>{a}, 1, a.num_fields, st);
}

cudaError_t launch_line_locations(const LineLocArgs& a, cudaStream_t st) {
  return lines_launch(ArgsOne<LineLocArgs>{a}, a.single_pass != 0, 1, a.num_fields, st);
}

cudaError_t launch_field_windows_many(const ArgsMany<LineLocArgs>& p, int portions, cudaStream_t st) {
  return portions > 0 ? windows_launch(p, portions, st) : cudaSuccess;
}

cudaError_t launch_field_pulses_many(const ArgsMany<LineLocArgs>& p, int portions, int max_fields, cudaStream_t st) {
  return portions > 0 ? pulses_launch(p, portions, max_fields, st) : cudaSuccess;
}

cudaError_t launch_line_locations_many(const ArgsMany<LineLocArgs>& p, int portions, int max_fields,
                                       cudaStream_t st) {
  return portions > 0 ? lines_launch(p, p.a[0].single_pass != 0, portions, max_fields, st) : cudaSuccess;
}

}  // namespace cuvhs
