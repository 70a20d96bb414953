// Decoder context: device buffers (allocated once), one CUDA stream, the
// state carried from chunk to chunk, and host copies of the last chunk's
// intermediates for inspection.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cuvhs.h"
#include "cuvhs_internal.h"

namespace cuvhs {

// Per-slot regions of the chunk buffers a batched round gives each capture:
// the capture whose chunk starts at slot s0 uses [s0 * per_slot, ...).
inline size_t kBitWordsPerSlot(int spp) { return (size_t)(spp + 31) / 32 + 1; }
inline size_t kEdgesPerSlot(int spp) { return (size_t)spp / 4 + 64; }
inline size_t kEdgeBlocksPerSlot(int spp) { return (size_t)(spp + 8191) / 8192 + 2; }
constexpr int kGuardPerSlot = 2048;  // near-threshold sync samples one field slot of a batched round can list

extern const int kPhaseCycle[8];
int phase_id_for(int is_first, int quadrant);
double host_burst_metric(const float* b, int H, int bl);
double host_burst_phase(const float* b, int H, const Format& fmt);

struct ChunkResult {
  int fields = 0;
  uint64_t next_raw_offset = 0;
  bool outputs_copied = false;  // luma/chroma already in the caller's host buffers
  std::vector<cuvhs_field_info> field_info;
};

// What one capture carries from chunk to chunk when it is decoded in batched
// rounds (a single-capture context keeps the same in its own members).
struct PortionState {
  LineLocState lls;
  bool chroma_valid = false;
  int chroma_track = 0;
  double chroma_threshold = 0.0;
  int chroma_cycle_start = 0;
  bool last_parity = true;
};
// One capture's chunk in a batched round.
struct Portion {
  const uint8_t* src = nullptr;  // host samples from raw_offset (u8)
  size_t n_avail = 0;
  uint64_t raw_offset = 0;
  int num_fields = 0;  // the chunk size
  int slot0 = 0;       // first field slot (the round's portions fill consecutive slots)
  PortionState* st = nullptr;
  uint16_t* dst_luma = nullptr;  // host planes for the chunk's fields, or null
  uint16_t* dst_chroma = nullptr;
  // filled in
  ChunkResult res;
  int T = 0, n_read = 0;
};

enum Stage {
  kStageK1a = 0,
  kStageK1b,
  kStageEdges,
  kStageHsync,
  kStageLuma,
  kStageChromaPre,
  kStageChromaLines,
  kStageBurstMetric,
  kStageDropouts,
  kStageGuard,    // FP64 re-evaluation of near-threshold sync samples
  kStageWindows,  // VSYNC clustering into field windows
  kStageLines,    // line locations (pulses, validation, anchors, snap), on the line stream
  // host phases (wall time on the calling thread)
  kHostWindowsWait,  // waiting for the chunk's field count and window offsets
  kHostChromaWait,
  kHostFinalWait,
  kNumStages
};
constexpr int kFirstHostStage = kHostWindowsWait;
extern const char* const kStageNames[kNumStages];

struct Context {
  cuvhs_config cfg{};
  Format fmt;
  Design des;
  int device = -1;
  int batch = 0;
  int spp = 0;
  int env_blocks = 0;
  int edge_cap = 0;
  int in_fmt = 0;         // InputFormat of the capture samples
  int bps = 1;            // bytes per capture sample
  bool dc_correct = false;
  bool single_pass = false;  // the single-pass line locator (config or CUVHS_K2B_DISABLE, read per chunk)
  int cur_n_read = 0;     // samples read into the current chunk window
  float* d_dc = nullptr;  // chunk DC mean (DC correction)
  unsigned long long* d_dcsum = nullptr;
  cudaStream_t stream = nullptr;
  // Copy stream: host input arrives in pieces (K1a starts on each piece as it
  // lands) and the finished luma leaves while chroma is still being decoded.
  cudaStream_t xstream = nullptr;
  // Output stream: the TBC planes leave on their own stream, so the small
  // copies the host waits on (window records, dropout lists) never queue
  // behind a chunk's or round's plane copies.
  cudaStream_t ostream = nullptr;
  static constexpr int kInputPieces = 8;
  cudaEvent_t ev_piece[kInputPieces] = {};
  cudaEvent_t ev_luma = nullptr;
  cudaEvent_t ev_edges = nullptr;
  // Cross-chunk pipelining of a capture held in host memory: while a chunk
  // decodes, the next chunk's window is copied into the other raw buffer on
  // the prefetch stream, and with page-locked destinations a chunk's planes
  // leave from one of two output sets while the next chunk already runs.
  cudaStream_t hstream = nullptr;  // host->device input copies
  // Line location: its own high-priority stream, so the field kernels run
  // beside the chroma prefilter; hsync waits on ev_ll.  ev_win marks the
  // field windows (the host reads the field count and offsets after it).
  cudaStream_t lstream = nullptr;
  cudaEvent_t ev_ll = nullptr, ev_win = nullptr, ev_winhost = nullptr;
  // Chroma pre-band-pass: its own stream, after K1b (ev_k1b), beside the
  // sync and line-location kernels; the chroma lines wait on ev_pre.
  cudaStream_t pstream = nullptr;
  cudaEvent_t ev_k1b = nullptr, ev_pre = nullptr;
  // FP64 guard: its own stream after K1b, beside the edges and line
  // locations, which run on K1b's FP32 in-pulse bits.  ev_guard marks the
  // guard and its listed / flipped counts in pinned memory; when it flipped
  // a threshold decision, the edges, windows and line locations run again on
  // the corrected sync (rare), from the line-location state saved before.
  cudaStream_t gstream = nullptr;
  cudaEvent_t ev_guard = nullptr;
  // Chroma track detection of a chunk without carried chroma state: both
  // trial passes over field 0 (one launch) and the device pick follow the
  // hsync refinement on the pre-band-pass stream, beside luma and dropouts;
  // ev_trial marks the pick (d_track set), ev_trialh the trial windows and the
  // pick in hp_burst / hp_pick.
  cudaEvent_t ev_hs = nullptr, ev_trial = nullptr, ev_trialh = nullptr;  // ev_trialh: the copies to the host
  cudaEvent_t ev_cpass = nullptr;  // a chroma pass on its stream, before its concealment
  int* d_trial = nullptr;        // {0, 1}: the trial tracks
  float* d_burst_trial = nullptr;  // [2][out_h * burst_len]
  int* d_pick = nullptr;
  int* hp_pick = nullptr;
  uint8_t* d_raw_set[2] = {};
  uint16_t* d_luma_set[2] = {};
  uint16_t* d_chroma_set[2] = {};
  int raw_set = 0, out_set = 0;
  cudaEvent_t ev_prefetch = nullptr, ev_small = nullptr, ev_chroma = nullptr;
  cudaEvent_t ev_out_done[2] = {};
  struct Prefetch {
    bool valid = false;
    uint64_t raw_offset = 0;
    size_t n_read = 0, total = 0;
    int set = 0;
  } pf;
  std::string err;
  cuvhs_status status = CUVHS_OK;
  std::vector<void*> allocations;
  std::vector<void*> host_allocations;
  cudaEvent_t ev_host = nullptr;
  int last_fields = 0;

  uint8_t* d_raw = nullptr;
  float *d_dem = nullptr, *d_env = nullptr, *d_video = nullptr, *d_sync = nullptr;
  double* d_env_part = nullptr;
  unsigned *d_fall = nullptr, *d_rise = nullptr;
  int* d_counts = nullptr;
  int2* d_edge_blk = nullptr;
  unsigned* d_edge_mask = nullptr;
  double* d_ll = nullptr;
  uint16_t *d_luma = nullptr, *d_chroma = nullptr;
  float* d_burst = nullptr;
  int* d_track = nullptr;
  int *d_do_count = nullptr, *d_do_lines = nullptr, *d_do_starts = nullptr, *d_do_ends = nullptr;
  unsigned char* d_do_cls = nullptr;
  double* d_col_frac = nullptr;
  // line location (kernels_linelocs.cu)
  WindowInfo* d_win = nullptr;
  long long* d_offs = nullptr;
  int* d_cand = nullptr;
  int *d_ps = nullptr, *d_pl = nullptr, *d_pn = nullptr;
  int *d_vs = nullptr, *d_vl = nullptr, *d_vn = nullptr;
  unsigned char* d_vt = nullptr;
  double* d_vd = nullptr;
  FieldPrep* d_prep = nullptr;
  LineLocState* d_lls = nullptr;
  int* d_is_first = nullptr;
  int *d_dbg_vs = nullptr, *d_dbg_vl = nullptr, *d_dbg_vt = nullptr, *d_dbg_vn = nullptr;
  long long *d_dbg_clk_ll = nullptr, *d_dbg_clk_guard = nullptr;  // phase clocks (debug)
  // guard band of the sync threshold (kernels_guard.cu)
  double2 *d_guard_g = nullptr, *d_guard_tw = nullptr;
  double* d_hs64 = nullptr;
  unsigned* d_guard_list = nullptr;
  int* d_guard_count = nullptr;
  double* d_guard_vals = nullptr;
  int* hp_guard = nullptr;  // pinned: the chunk's listed count, then its flipped count (per capture in a round)
  LineLocState* hp_lls = nullptr;  // pinned: line-location states of a round's captures
  unsigned* d_pulse_bits = nullptr;
  int* d_guard_flips = nullptr;
  LineLocState* d_lls_save = nullptr;
  // Guard launch over the current chunk's sync (T tiles), after the last K1b;
  // every later threshold decision reads the corrected samples.
  GuardArgs guard_args(const DemodArgs& da) const;
  float2 *d_ga = nullptr, *d_gb = nullptr, *d_twa = nullptr, *d_twb = nullptr, *d_twc = nullptr, *d_twl = nullptr;
  float2 *d_twa_inv = nullptr, *d_twb_inv = nullptr, *d_twc_inv = nullptr, *d_twl_inv = nullptr;
  float* d_gc = nullptr;

  // carried state (the line-location part lives on the device, d_lls)
  bool chroma_valid = false;
  int chroma_track = 0;
  double chroma_threshold = 0.0;
  int chroma_cycle_start = 0;
  bool last_parity = true;

  // host scratch (kept to avoid reallocation)
  std::vector<int> h_phase, computed_track;
  // pinned staging
  int* hp_counts = nullptr;
  WindowInfo* hp_win = nullptr;
  long long* hp_offs = nullptr;
  int* hp_is_first = nullptr;
  int *hp_track = nullptr, *hp_trial = nullptr;
  float* hp_burst = nullptr;
  double* hp_metric = nullptr;  // mapped: the metric kernel writes it directly
  double* dp_metric = nullptr;  // device alias of hp_metric
  int *hp_do_count = nullptr, *hp_do_lines = nullptr, *hp_do_starts = nullptr, *hp_do_ends = nullptr;

  // last-chunk intermediates (debug)
  bool debug = false;
  int debug_tiles = 2;
  std::vector<int> dbg_meta, dbg_vsync, dbg_k2c, dbg_k2s, dbg_k2l, dbg_k2bc, dbg_k2bs, dbg_k2bl, dbg_k2bt, dbg_is_first;
  std::vector<long long> dbg_offs;
  std::vector<double> dbg_ll_coarse, dbg_ll, dbg_guard_vals;
  std::vector<long long> dbg_guard_pos, dbg_clk_ll, dbg_clk_guard;
  std::vector<float> dbg_demod, dbg_video, dbg_sync, dbg_env, dbg_pre;

  // per-stage device time (CUDA events on the decode stream) and launch count
  bool timing = false;
  unsigned timing_mask = ~0u;  // device stages bracketed by events while timing (bit = Stage)
  double stage_ms[kNumStages] = {};
  long long stage_launches[kNumStages] = {};
  long long launches = 0;
  struct Mark {
    int stage;
    cudaEvent_t a, b;
  };
  std::vector<Mark> marks;
  // the last chunk's device stage intervals, ms from its first timed event
  struct Span {
    int stage;
    double start, end;
  };
  std::vector<Span> timeline;
  cudaEvent_t ev_t0 = nullptr;  // first timed event of the current chunk
  bool t0_pending = false;      // the next begin_stage opens a new chunk's timeline
  std::vector<cudaEvent_t> event_pool;
  size_t pool_used = 0;
  cudaEvent_t next_event();
  void begin_stage(int stage, cudaEvent_t& a) { begin_stage_on(stage, a, stream); }
  void end_stage(int stage, cudaEvent_t a, int kernels = 1) { end_stage_on(stage, a, stream, kernels); }
  void begin_stage_on(int stage, cudaEvent_t& a, cudaStream_t st);
  void end_stage_on(int stage, cudaEvent_t a, cudaStream_t st, int kernels = 1);
  void collect_stage_times();
  double host_clock() const;
  void host_phase(int stage, double t0) {
    if (timing) stage_ms[stage] += host_clock() - t0;
  }

  ~Context();
  bool init(const cuvhs_config& c);
  bool alloc_buffers();  // for `batch` fields; false (err set) when an allocation fails
  void free_buffers();
  size_t dev_limit = 0, dev_used = 0;  // device bytes this context may allocate (0: no limit), allocated
  void release();
  void reset_state();
  bool check_cuda(const char* where);
  bool sync(const char* where);
  bool wait_host_event(const char* where);
  // dst_luma / dst_chroma: optional page-locked host destinations for the
  // chunk's fields (num_fields fields of room each); when given, the planes
  // are copied there as soon as each is final and res.outputs_copied is set.
  // cap_base / cap_n: the whole host capture `src` lies in (src = cap_base +
  // raw_offset); when given, the next chunk's window is prefetched.  defer:
  // return before the plane copies end (drain_copies() waits for them).
  bool decode_chunk(const uint8_t* src, bool src_on_device, size_t n_avail, uint64_t raw_offset, int num_fields,
                    ChunkResult& res, uint16_t* dst_luma = nullptr, uint16_t* dst_chroma = nullptr,
                    const uint8_t* cap_base = nullptr, size_t cap_n = 0, bool defer = false);
  // Waits for deferred plane copies and input prefetches; returns false on a CUDA error.
  bool drain_copies();
  // The next chunk of up to kMaxPortions captures in one pass of batched
  // launches (round.cpp); res of each portion as decode_chunk's, its dropout
  // lists at hp_do_* + slot0 * kMaxDropouts.
  // next_plan, when given, is called once the round's field windows are
  // known (each portion's res.fields and next_raw_offset set) and returns the
  // next round's portions, whose input windows are then copied into the other
  // raw buffer while this round finishes; a next call with exactly those
  // portions reads them there.
  using RoundPlan = std::function<void(const std::vector<Portion>&, std::vector<Portion>&)>;
  bool decode_round(std::vector<Portion>& ps, const RoundPlan& next_plan = nullptr);
  struct RoundPrefetch {
    bool valid = false;
    int set = 0;
    std::vector<std::pair<const uint8_t*, long long>> sig;  // (src, n_read << 20 | slot0) per portion
  } rpf;
  int round_raw_set = 0;
  float* hp_round_burst = nullptr;  // pinned: trial-pass burst windows of a round's captures (on first use)
  // K1 arguments over T tiles of the current raw buffer into the context's buffers.
  DemodArgs demod_args(int T) const;
  // Kernel arguments on the context's buffers: chroma over T tiles of `raw`,
  // lines and dropouts over P fields.
  ChromaArgs chroma_args(const uint8_t* raw, int n_read, const float* dc, int T) const;
  LineArgs line_args(int P) const;
  DropoutArgs dropout_args(int P) const;
  // Chroma lines of fields [0, P) of ca (pre-band-passed already) with the
  // track/phase decisions and the carried chroma state; sets h_phase.  With
  // `conceal`, fields are concealed as they are decoded; with dst_chroma (page
  // -locked host planes), sent there on the copy stream as well.
  // trial_on_device: the trial passes and the device pick were enqueued
  // (ev_trial) for a context without carried chroma state.
  // chroma_stream: the stream of the chroma passes (nullptr: the decode
  // stream); it must already follow the hsync refinement and the pre-band-pass.
  bool chroma_fields(ChromaArgs& ca, int P, const DropoutArgs* conceal = nullptr, uint16_t* dst_chroma = nullptr,
                     bool trial_on_device = false, cudaStream_t chroma_stream = nullptr);
  // Sync edges of `sync` over [0, total) and the field windows clustered
  // from them (at most num_fields), read back into hp_win / hp_offs
  // (synchronous).
  bool field_windows(const float* sync, long long total, int tiles, int num_fields);
  // Line-location kernel arguments for the current chunk.
  LineLocArgs lineloc_args(int tiles, int num_fields, long long raw_offset) const;
  // The device line-location state (d_lls) to and from the host.
  bool read_lls(LineLocState& st);
  bool write_lls(const LineLocState& st);
  // False (with the error set) when a chunk listed more near-threshold sync
  // samples than the guard's capacity.
  bool guard_ok(int listed);
};

// .tbc.json text (reference format, src/io/tbc_writer.cpp:89-175).
std::string tbc_json(const Format& fmt, const cuvhs_field_info* fields, size_t n, const int32_t* dl,
                     const int32_t* ds, const int32_t* de);

}  // namespace cuvhs

// The C ABI's opaque context handle.
struct cuvhs_ctx {
  cuvhs::Context c;
};
