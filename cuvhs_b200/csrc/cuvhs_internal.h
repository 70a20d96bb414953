// Internal interfaces of libcuvhs: NTSC format constants, the filter design
// that turns the reference's frequency responses into short time-domain
// kernels for shared-memory overlap-save, the device kernels' launchers and
// the host-side line-location logic.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace cuvhs {

constexpr int kOverlap = 2048;        // overlap-save history of every demod tile
constexpr int kFieldMarginLines = 20;  // extra lines per tile beyond one field
constexpr int kMaxPulses = 800;        // pulses kept per field
constexpr int kPhaseSlots = 32;        // phase clocks recorded per field or sample (inspection)
constexpr int kMaxDropouts = 512;      // TBC dropout entries per field
constexpr int kMaxRfDropouts = 128;    // RF-domain dropout spans per field
constexpr int kMaxBurstLen = 48;       // burst window width bound, output samples (NTSC 36, PAL 40)
enum PulseType { kHsync = 0, kEq1 = 1, kVsync = 2, kEq2 = 3 };
enum VideoSystem { kNtsc = 0, kPal = 1 };

// Format constants of the video system, derived from the capture rate
// (reference: src/format/video_format.cpp:23-104; the members' initial
// values are NTSC's).
struct Format {
  int system = kNtsc;
  double fs_hz = 0;
  int lines_per_frame = 525;
  int output_line_len = 910;
  int output_field_lines = 263;
  int field_lines_first = 263, field_lines_second = 262;
  int num_eq_pulses = 6;
  int active_line_start = 10;
  double line_rate = 15734.264;
  double fsc = 3579545.0;
  double chroma_under = 0;
  double hz_ire = 0, ire0 = 0, vsync_ire = -40.0;
  double pulse_threshold_hz = 0;
  double output_zero = 1024.0, output_scale = 0;
  double output_rate = 0;
  double burst_abs_ref = 4416.0, burst_start_us = 5.3, burst_end_us = 7.8;
  int samples_per_line = 0, samples_per_field = 0;
  int spp = 0;  // tile stride: samples_per_field + 20 lines
  double hsync_width = 0, eq_pulse_width = 0, vsync_width = 0;
  int burst_start = 0, burst_end = 0;  // in output samples
  int burst_len = 0;                   // burst_end - burst_start
  int lines_per_field = 263;
  int line_fft = 1024;                 // chroma per-line transform: next power of 2 >= output_line_len
  void init(double mhz, int system = kNtsc);
};

// Filter kernels for the three overlap-save stages.  Every stage reproduces a
// circular convolution over one reference tile (length `tile`), evaluated
// block by block: a block of N samples yields N - (neg + pos) outputs.
struct Design {
  int tile = 0;     // demod tile length: 7-smooth >= spp + 2048
  int bins = 0;     // tile/2 + 1
  // K1a: u8 -> analytic signal (RF band-pass x Hilbert weighting)
  static constexpr int kNa = 4096;
  int a_neg = 0, a_pos = 0, a_out = 0;
  std::vector<float2> ga;       // block spectrum of the truncated analytic kernel / kNa
  double a_tail = 0;            // relative l2 energy outside the kept support
  float rot_re = 1, rot_im = 0;  // e^{-i d0}: nominal carrier phase step removed before atan2
  double d0 = 0;                 // nominal phase step (rad/sample) at ire0
  float demod_scale = 0;         // fs / 2pi
  float demod_offset = 0;        // d0 * fs/2pi - ire0 (Hz)
  // K1b: demod -> video (real part) + sync (imag part)
  static constexpr int kNb = 8192;
  int b_neg = 0, b_pos = 0, b_out = 0;
  std::vector<float2> gb;
  double b_tail = 0;
  float corr_video = 0, corr_sync = 0;
  // chroma colour-under pre-band-pass (zero-padded tile of length ctile)
  static constexpr int kNc = 16384;
  int ctile = 0;
  int c_half = 0, c_out = 0;  // kernel half-width, outputs per half block
  std::vector<float> gc;       // real block spectrum / kNc
  double c_tail = 0;
  // FP64 taps for re-evaluating sync samples near the pulse threshold (the
  // guard band): the K1a analytic kernel at offsets [-ga64_half, ga64_half]
  // (interleaved re, im) and the sync kernel at [-hs64_half, hs64_half], each
  // wide enough that every dropped tap lies below kGuardTailRel of the largest.
  static constexpr double kGuardTailRel = 1e-13;
  static constexpr int kGuardMaxHalf = 4096;
  int ga64_half = 0, hs64_half = 0;
  std::vector<double> ga64, hs64;
  // the guard's overlap-save form of ga64: its kGuardN-point FFT (taps at
  // offset m placed at m mod kGuardN) divided by kGuardN, and the FFT's
  // twiddles exp(-2 pi i k / kGuardN); interleaved re, im
  static constexpr int kGuardN = 4096;
  std::vector<double> guard_g, guard_tw;
  // twiddle tables W_N^m
  std::vector<float2> tw_a, tw_b, tw_c, tw_line;
  // chroma per-line constants
  double het_scale = 0;
  int fsc_bin = 0, bw_bins = 0;
  void build(const Format& fmt);
  // build() once per sample rate per process; later calls copy the result
  // (thread-safe).  Contexts of one rate then share the FP64 design work.
  void build_cached(const Format& fmt);
};

// Half-support (samples each side) of the truncated K1a kernel at a capture
// rate: a K1a block of Design::kNa samples yields kNa - 2 * h - 1 outputs,
// the first at block position h + 1 (Design::a_pos, Design::a_out).
int k1a_half_support(double fs_hz);

// Kernel arguments of one capture's chunk, or of the chunks of several
// captures decoded together (a batched round: grid.z picks the capture, and
// every kernel runs the one-capture code on that capture's arguments).  Both
// travel as __grid_constant__ kernel parameters (kMaxPortions sets of the
// largest argument struct fit the 32 KB parameter space).  A single chunk's
// arguments are a set of one, read the same way (indexed by grid.z, which is
// 0), so a kernel compiles to the same arithmetic for one capture or many
// and a batched capture decodes bit for bit as it does alone.
constexpr int kMaxPortions = 64;
template <class A>
struct ArgsOne {
  A a[1];
#ifdef __CUDACC__
  __device__ __forceinline__ const A& get() const { return a[blockIdx.z]; }
#endif
};
template <class A>
struct ArgsMany {
  A a[kMaxPortions];
#ifdef __CUDACC__
  __device__ __forceinline__ const A& get() const { return a[blockIdx.z]; }
#endif
};

// ---------------------------------------------------------------- kernels
struct DemodArgs {
  const uint8_t* raw;  // chunk samples in the input format (raw_input.cuh)
  int in_fmt;          // InputFormat
  int n_read;          // samples read; chunk positions past them are 0
  const float* dc;     // device scalar subtracted from every sample read, or null
  long long total;     // T * spp (clamp bound of the tile gathers)
  int tiles, spp, tile;
  const float2* ga;
  const float2* gb;
  const float2* tw_a;
  const float2* tw_b;
  // The inverse transforms read their own copies of the twiddle tables, so the
  // compiler cannot merge the two transforms' twiddle loads and keep them all
  // live at once.
  const float2* tw_a_inv;
  const float2* tw_b_inv;
  int a_pos, a_out, b_pos, b_out;
  float rot_re, rot_im, d0, demod_scale, demod_offset;
  float corr_video, corr_sync;
  float* dem;      // [T*spp] demod - ire0 (Hz)
  float* env;      // [T*spp] |analytic|
  double* env_part;  // [T * env_blocks] per-block envelope sums
  int env_blocks;    // blocks per tile of the K1a grid
  float* video;    // [T*spp] video - ire0
  float* sync;     // [T*spp] sync - ire0
  // Guard band: K1b lists every sync sample it writes within guard_hz of
  // thr_rel (chunk index into guard_list); the count may exceed guard_cap,
  // which the host reports.  guard_list == null: off.
  // In-pulse bits (sync <= thr_rel, FP32): bit p of pulse_bits is set by K1b
  // for chunk position p in a pulse (the array zeroed before K1b); null: off.
  unsigned* pulse_bits = nullptr;
  float thr_rel = 0.0f, guard_hz = 0.0f;
  unsigned* guard_list = nullptr;
  int* guard_count = nullptr;
  int guard_cap = 0;
};

// FP64 re-evaluation of the listed sync samples (kernels_guard.cu).
constexpr float kGuardHz = 8.0f;   // half-width of the guard band: >= 4x the largest FP32 sync error measured
constexpr int kGuardCap = 65536;    // flagged samples one chunk can list
struct GuardArgs {
  const uint8_t* raw;
  int in_fmt, n_read;
  const float* dc;
  long long total;  // T * spp: the demodulated chunk extent
  int spp, tile;
  const double2* gfft;  // [Design::kGuardN] FFT of the K1a taps (offsets [-ha, ha]) / kGuardN
  const double2* tw;    // [Design::kGuardN] exp(-2 pi i k / kGuardN)
  int ha;
  const double* hs64;  // sync taps, offsets [-hb, hb]
  int hb;
  double scale;        // fs / 2pi
  double ire0, thr_hz;  // absolute Hz: the reference's threshold
  float thr_rel;        // the FP32 threshold the edge kernels compare with
  float* sync;          // corrected in place
  const unsigned* list;
  const int* count;
  int cap;
  double* values;  // optional [cap]: the FP64 sync value of each listed sample
  int* flips = nullptr;  // optional: counts samples whose FP64 side differs from their FP32 value's
  long long* dbg_clk = nullptr;  // optional [kGuardClockSamples][kPhaseSlots]: SM clock at each phase of a sample's CTA
};
constexpr int kGuardClockSamples = 1024;
// Whether the guard handles these tap supports, and its shared memory.
bool guard_supported(int ha, int hb);
size_t guard_smem_bytes(int hb);
cudaError_t launch_sync_guard(const GuardArgs& g, cudaStream_t st);
cudaError_t launch_sync_guard_many(const ArgsMany<GuardArgs>& p, int portions, cudaStream_t st);
// K1a over tiles [f0, f0 + nf).
void launch_k1a(const DemodArgs& a, int f0, int nf, cudaStream_t st);
// K1a / K1b over every tile of `portions` captures' chunks (one launch each).
void launch_k1a_many(const ArgsMany<DemodArgs>& p, int portions, int max_tiles, cudaStream_t st);
void launch_k1b_many(const ArgsMany<DemodArgs>& p, int portions, int max_tiles, cudaStream_t st);
// DC correction: *dc = mean of the n converted samples of raw (exact integer
// sum, one FP64 division, as the reference's FP64 loop), as FP32.
// sum is scratch for one unsigned long long.
void launch_dc_mean(const uint8_t* raw, int n, int in_fmt, unsigned long long* sum, float* dc, cudaStream_t st);
// K1b over tiles [f0, f0 + nf): every tile is filtered on its own, so it can
// follow K1a tile range by tile range.
void launch_k1b(const DemodArgs& a, int f0, int nf, cudaStream_t st);

// Threshold edges of the sync signal in sample order: falling (x<=thr after
// x>thr, or at 0) and rising (x>thr after x<=thr).  counts[0..1] = totals;
// blk is scratch of edge_blocks(total) entries.
int edge_blocks(long long total);
// masks: scratch of edge_mask_words(total) words (per-thread edge bit masks)
size_t edge_mask_words(long long total);
// Threshold edges from K1b's in-pulse bits (the same lists as launch_edges on
// the FP32 sync it wrote).
struct EdgeArgs {
  const unsigned* bits;
  long long total;
  int2* blk;    // per-CTA counts, then offsets
  int* counts;  // [0] falling, [1] rising
  unsigned *fall, *rise;
  int cap;
};
void launch_edges_bits(const unsigned* bits, long long total, unsigned* fall, unsigned* rise, int* counts, int cap,
                       int2* blk, cudaStream_t st);
size_t pulse_bit_words(long long total);
void launch_edges_bits_many(const ArgsMany<EdgeArgs>& e, int portions, long long max_total, cudaStream_t st);
void launch_edges(const float* sync, long long total, float thr_rel, unsigned* fall, unsigned* rise,
                  int* counts, int cap, int2* blk, unsigned* masks, cudaStream_t st);

struct LineArgs {
  const float* video;
  const float* sync;
  double* ll;  // [P*525]
  int fields;
  long long total;  // P * spp
  int lines_per_frame, active_line_start;
  float thr_rel;
  double one_us, hsync_width, right_edge_offset;
  // luma resample
  uint16_t* luma;  // [P*263*910]
  int out_w, out_h;
  float luma_gain, luma_offset;  // u16 = video_rel * gain + offset
  uint16_t oob_value;            // pixels outside the signal: output_zero (tbc_resample.cu:91-96)
  const double* col_frac;        // [out_w]: (double)col / (double)out_w
};
void launch_hsync_refine(const LineArgs& a, cudaStream_t st);
void launch_luma(const LineArgs& a, cudaStream_t st);
void launch_hsync_refine_many(const ArgsMany<LineArgs>& p, int portions, int max_fields, cudaStream_t st);
void launch_luma_many(const ArgsMany<LineArgs>& p, int portions, int max_fields, cudaStream_t st);

struct ChromaArgs {
  const uint8_t* raw;  // as DemodArgs
  int in_fmt, n_read;
  const float* dc;
  float* pre;  // [P*spp]
  int fields, spp, ctile, c_half, c_out;
  const float* gc;
  const float2* tw_c;
  const float2* tw_line;
  const float2* tw_c_inv;
  const float2* tw_line_inv;
  const double* ll;
  long long total;  // P * spp
  const int* track;  // per field
  double het_scale;
  int fsc_bin, bw_bins, burst_start, burst_len;
  int line_fft;      // per-line transform size (1024 or 2048)
  int out_w, out_h, lines_per_frame;
  float burst_abs_ref;
  uint16_t* chroma;  // [P*out_h*out_w]
  float* burst;      // [P*out_h*burst_len] band-passed burst window (scaled)
  double* metric;    // per field burst cancellation metric
  const double* col_frac;  // [out_w]: (double)col / (double)out_w
};
void launch_chroma_prefilter(const ChromaArgs& a, cudaStream_t st);
// Lines [field0*out_h, (field0+nfields)*out_h) of the chunk.
void launch_chroma_lines(const ChromaArgs& a, int field0, int nfields, bool write_output, cudaStream_t st);
void launch_burst_metric(const ChromaArgs& a, int field0, int nfields, cudaStream_t st);
// The same over `portions` captures (grid.z): the pre-band-pass over each
// capture's a.fields tiles; chroma lines of fields [0, nfields) of each
// (nfields < 0: each capture's a.fields) and their burst metrics.
void launch_chroma_prefilter_many(const ArgsMany<ChromaArgs>& p, int portions, int max_tiles, cudaStream_t st);
void launch_chroma_lines_many(const ArgsMany<ChromaArgs>& p, int portions, int nfields, int max_fields,
                              bool write_output, cudaStream_t st);
void launch_burst_metric_many(const ArgsMany<ChromaArgs>& p, int portions, int max_fields, cudaStream_t st);

// Track detection on the device (chroma_decode.cu:684-743): the burst
// cancellation metric of both trial passes over field 0 (burst0: track 0,
// burst1: track 1), summed in the host's order, picks the track with the
// lower metric; track[f] for f < fields alternates from it, *pick = it.
struct TrackPickArgs {
  const float* burst0;
  const float* burst1;
  int out_h, burst_len, fields;
  int* track;
  int* pick;
};
void launch_track_pick(const TrackPickArgs& a, cudaStream_t st);

struct DropoutArgs {
  const float* env;
  const double* env_part;
  int env_blocks;
  const double* ll;
  int fields, spp, lines_per_frame, active_line_start, out_w, out_h;
  uint16_t* luma;
  uint16_t* chroma;
  int* do_count;
  int* do_lines;
  int* do_starts;
  int* do_ends;
  unsigned char* cls = nullptr;  // two-pass form: [fields * max_blocks]
  int max_blocks = 0;            // 16-sample blocks per field slot, dropout_class_bytes_per_field(spp)
};
// Dynamic shared memory cap of the kernels that hold one field's class bytes
// (dropout_class_bytes_per_field(spp) must not exceed it).
constexpr int kMaxClassBytes = 200 * 1024;
// Fused form: one CTA per field, no scratch beyond env_part.  Returns the
// error of the attribute set or of the launch.
cudaError_t launch_dropouts(const DropoutArgs& a, cudaStream_t st);
// Two-pass form: wide class kernel over every field, then a per-field scan
// that maps the entries and conceals the luma; chroma concealment follows
// once the chroma planes are final.
// Class bytes per field slot of spp samples: one per 16-sample block, rounded
// up to a multiple of 16.
size_t dropout_class_bytes_per_field(int spp);
void launch_dropouts_two_pass(const DropoutArgs& a, cudaStream_t st);
// Chroma concealment of fields [f0, f0 + nf) (their chroma lines final).
void launch_dropout_conceal_chroma(const DropoutArgs& a, int f0, int nf, cudaStream_t st);
void launch_dropouts_two_pass_many(const ArgsMany<DropoutArgs>& p, int portions, int max_fields, cudaStream_t st);
void launch_dropout_conceal_chroma_many(const ArgsMany<DropoutArgs>& p, int portions, int max_fields,
                                        cudaStream_t st);

// ---------------------------------------------------------------- line locations
// Per-field pulse validation, mean line length, vertical-blanking anchor and
// line-location snapping (reference: src/pipeline/pipeline.cu:410-893), with
// the state carried from field to field (pipeline.h:92-97).
struct LineLocState {
  int prev_first_field = -1;
  int prev_progressive_field = -1;
  long long prev_first_hsync_readloc = -1;
  double prev_first_hsync_loc = -1.0;
  double prev_first_hsync_diff = -1.0;
};
constexpr int kAnchorConfidence = 75;  // pattern vote (percent) that fixes the field order
// Vertical-blanking pulses of one field and their half-line pattern.
struct BlankingScan {
  int vb_pulse[8];
  double order_len[4];
  double agree = 0.0, seen = 0.0;
};
// First-hsync anchor of one field for a given field order.
struct AnchorFit {
  int cnt = 0;                 // estimates combined (0: no anchor)
  bool used_prediction = false;
  double loc_round = 0.0;      // estimate before the hsync refinement
  double loc = 0.0;            // first-hsync location
  double hsync_line = 0.0;
};
constexpr int kMaxValid = kMaxPulses * 27;  // validated entries of one field: each raw pulse adds
                                            // itself, or up to 26 entries of a blanking sequence

// The stateless part of one field's line location (kernels_linelocs.cu):
// mean line length, blanking scan and, when the field's pattern fixes its
// order, the anchor of the speculative grid.
struct FieldPrep {
  double mll = 0.0;
  double raw0 = 0.0;    // first raw pulse start, the fallback grid origin
  int n_raw = 0;
  int vn = 0;           // validated entries
  int spec_first = -1;  // field order of the speculative anchor, -1 if none
  // the field-order vote of the blanking pattern, which needs no carried
  // state: the order with no previous field, and each order's vote (percent,
  // when the pattern saw any interval)
  int pat_default = 1;
  int c_first = 0, c_second = 0;
  // the chunk's first field is fitted with the chunk's incoming state (known
  // when the per-field pass runs): exact = 1, its order in exact_first and
  // its fit in spec
  int exact = 0, exact_first = 0;
  BlankingScan scan;
  AnchorFit spec;
};
// Field windows of one chunk (written by the field-window kernel).
struct WindowInfo {
  int fields = 0;  // windows (fields) in the chunk
  int ncand = 0;   // VSYNC candidates
  int err = 0;     // 1: an edge list overflowed
  int pad = 0;
  long long next_rel = 0;  // start of the next chunk, relative to this one
};
// Arguments of the line-location kernels.
struct LineLocArgs {
  Format fmt;
  const unsigned* fall;  // sorted threshold edges of the chunk
  const unsigned* rise;
  const int* counts;     // [0] falling, [1] rising edges
  int edge_cap;
  long long total;       // T * spp
  int tiles, num_fields;
  int minw, maxw;        // VSYNC run widths (samples)
  WindowInfo* win;
  long long* offs;       // [num_fields] window starts, chunk positions
  int* cand;             // [cand_cap] VSYNC candidates
  int cand_cap;
  int *ps, *pl, *pn;     // [num_fields][kMaxPulses] window pulses, [num_fields] counts
  int *vs, *vl;          // [num_fields][kMaxValid] validated pulses
  unsigned char* vt;     // type | good << 2
  double* vd;            // [num_fields][kMaxValid] scratch
  int* vn;               // [num_fields]
  FieldPrep* prep;       // [num_fields]
  LineLocState* state;   // carried from field to field and chunk to chunk
  double* ll;            // [num_fields][lines_per_frame] line starts
  int* is_first;         // [num_fields] 1 first, 0 second (single pass: -1 undetermined)
  long long raw_offset;  // capture position of the chunk
  int single_pass;
  int *dbg_vs = nullptr, *dbg_vl = nullptr, *dbg_vt = nullptr, *dbg_vn = nullptr;  // optional: validated pulses
  long long* dbg_clk = nullptr;  // optional [num_fields][kPhaseSlots]: SM clock at each phase of a field's CTAs
};
size_t lineloc_smem_bytes();
// VSYNC clustering into field windows (one CTA).
cudaError_t launch_field_windows(const LineLocArgs& a, cudaStream_t st);
// The pulses of every field window.
cudaError_t launch_field_pulses(const LineLocArgs& a, cudaStream_t st);
// Line locations of every field window: the validated host path of the
// reference (per-field CTAs, then one CTA in field order), or the single-pass
// locator.
cudaError_t launch_line_locations(const LineLocArgs& a, cudaStream_t st);
// The same over `portions` captures' chunks (grid.z), fields per capture up
// to max_fields (each capture's own count in its arguments).
cudaError_t launch_field_windows_many(const ArgsMany<LineLocArgs>& p, int portions, cudaStream_t st);
cudaError_t launch_field_pulses_many(const ArgsMany<LineLocArgs>& p, int portions, int max_fields, cudaStream_t st);
cudaError_t launch_line_locations_many(const ArgsMany<LineLocArgs>& p, int portions, int max_fields,
                                       cudaStream_t st);

}  // namespace cuvhs
