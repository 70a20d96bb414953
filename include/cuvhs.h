/* libcuvhs: B200 (sm_100a) VHS RF decoder, C ABI.
 *
 * Drop-in for the decode path of hunterschuler/cuVHS: an NTSC or PAL VHS RF
 * capture (u8, s16 or u16 samples) in, u16 luma and chroma TBC fields (910x263
 * NTSC, 1135x313 PAL) plus .tbc.json field/line/dropout metadata out.  Every entry point returns a cuvhs_status; no C++ types or
 * exceptions cross the boundary.  A context owns one CUDA stream and all of its
 * device memory, allocated once in cuvhs_create.  Contexts are independent;
 * one context is not safe to use from two threads at once.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   cuvhs_create / cuvhs_destroy      Pipeline::Pipeline + allocate_buffers +
 *                                     FMDemodState::init (src/pipeline/pipeline.h:28-33,
 *                                     src/pipeline/pipeline.cu:1383-1475,
 *                                     src/pipeline/fm_demod.cu:273-374)
 *   cuvhs_decode_chunk                Pipeline::process_chunk (src/pipeline/pipeline.cu:1525-2624)
 *   cuvhs_decode_capture              Pipeline::run chunk loop (src/pipeline/pipeline.cu:2626-2713)
 *   cuvhs_decode_file                 main + RawReader + TBCWriter (src/main.cpp:97-165,
 *                                     src/io/raw_reader.cpp:128-151, src/io/tbc_writer.cpp:10-175)
 *   cuvhs_json                        TBCWriter::write_json (src/io/tbc_writer.cpp:89-175)
 *   cuvhs_stage_*                     the stage functions fm_demod, discover_vsyncs,
 *                                     sync_pulses, hsync_refine, tbc_resample,
 *                                     chroma_decode and the K2b host line locations
 *                                     (src/pipeline/{fm_demod,vsync_discover,...}.h;
 *                                     pipeline.cu:1557-2548)
 *   cuvhs_decode_chunk_async,         no counterpart (the reference's calls are
 *   cuvhs_flush                       synchronous): chunk decode whose plane copies
 *                                     overlap the next chunk, and the wait for them
 *   cuvhs_debug_array                 the stage outputs the reference keeps in device
 *                                     buffers (d_pulse_*, d_linelocs, d_is_first_field,
 *                                     d_do_*; src/pipeline/pipeline.h:52-87)
 *   cuvhs_adjoint_*                   no counterpart: the reference has no gradients; a
 *                                     differentiable decode model with adjoint kernels for
 *                                     tape parameter calibration
 *   cuvhs_batch_*                     no counterpart: the reference decodes one capture per
 *                                     process (src/main.cpp:97-165); a batch decodes many
 *                                     captures of mixed sample rates concurrently, each
 *                                     exactly as a single-capture decode would
 */
#ifndef CUVHS_H
#define CUVHS_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define CUVHS_FIELD_WIDTH 910
#define CUVHS_FIELD_HEIGHT 263
#define CUVHS_MAX_DROPOUTS_PER_FIELD 512

typedef enum cuvhs_status {
  CUVHS_OK = 0,
  CUVHS_ERR_INVALID_ARGUMENT = 1,
  CUVHS_ERR_CUDA = 2,
  CUVHS_ERR_OUT_OF_MEMORY = 3,
  CUVHS_ERR_IO = 4,
  CUVHS_ERR_CAPACITY = 5,    /* an internal fixed-size list overflowed */
  CUVHS_ERR_UNSUPPORTED = 6, /* e.g. a PAL context for the NTSC-only calibration model */
  CUVHS_ERR_EXISTS = 7       /* output exists and overwrite was not requested */
} cuvhs_status;

typedef struct cuvhs_ctx cuvhs_ctx;

typedef struct cuvhs_config {
  int system;             /* --system: 0 = NTSC, 1 = PAL (src/format/video_format.cpp:23-104) */
  double sample_rate_mhz; /* -f, capture rate */
  int device;             /* --gpu: CUDA device id, -1 = the one with most memory */
  int batch_fields;       /* fields per chunk; 0 = derive from free device memory */
  int stream_mode;        /* non-zero caps the chunk at 64 fields (pipe input) */
  int input_format;       /* --format: 0 = u8, 1 = s16, 2 = u16 (src/io/raw_reader.cpp:71-91) */
  int dc_correct;         /* --dc-correct: subtract each chunk's mean sample (raw_reader.cpp:93-99) */
  int single_pass_lines;  /* 1: the reference's single-pass line locator (src/pipeline/line_locs.cu) in
                             place of its validated host line location, as the reference runs with the
                             CUVHS_K2B_DISABLE environment variable set (which does the same here) */
  double guard_band_hz;   /* half-width of the band around the sync pulse threshold inside which sync
                             samples are re-evaluated in FP64 before any threshold decision; 0 = the
                             default (8 Hz, several times the FP32 sync error).  Wider bands cost time
                             and change nothing else; they exist to check the FP64 path */
  double device_memory_limit_mb; /* 0 = none; else the context allocates at most this much device
                             memory, as if other users held the rest: when batch_fields is 0 the
                             batch is sized from the free memory and halved after any allocation
                             that fails or passes the limit (the reference's VRAM back-off,
                             src/pipeline/pipeline.cu:1384-1475); an explicit batch_fields that does
                             not fit fails with CUVHS_ERR_OUT_OF_MEMORY */
} cuvhs_config;

/* Per-field metadata, one .tbc.json "fields" entry. */
typedef struct cuvhs_field_info {
  uint64_t file_loc;      /* capture sample where the field's window starts */
  int32_t is_first_field;
  int32_t field_phase_id; /* 1..4, 0 = unset */
  int32_t dropout_count;
  int32_t dropout_offset; /* first entry in the dropout arrays */
} cuvhs_field_info;

/* Caller-owned host output buffers. */
typedef struct cuvhs_output {
  uint16_t* luma;          /* [max_fields][field height][field width] */
  uint16_t* chroma;        /* [max_fields][field height][field width] */
  cuvhs_field_info* fields; /* [max_fields] */
  int32_t* dropout_line;   /* [max_dropouts] */
  int32_t* dropout_startx;
  int32_t* dropout_endx;
  size_t max_fields;
  size_t max_dropouts;
  /* filled in by the decoder */
  size_t fields_out;
  size_t dropouts_out;
  uint64_t next_raw_offset; /* chunk calls: where the next chunk starts */
} cuvhs_output;

void cuvhs_default_config(cuvhs_config* cfg);
cuvhs_status cuvhs_create(const cuvhs_config* cfg, cuvhs_ctx** out);
void cuvhs_destroy(cuvhs_ctx* ctx);
const char* cuvhs_last_error(const cuvhs_ctx* ctx);
const char* cuvhs_status_string(cuvhs_status s);

int cuvhs_batch_fields(const cuvhs_ctx* ctx);
/* Output field geometry of the context's system: 910 x 263 (NTSC) or
 * 1135 x 313 (PAL) u16 samples, and line locations per field (525 / 625).
 * CUVHS_FIELD_WIDTH / CUVHS_FIELD_HEIGHT are the NTSC values. */
int cuvhs_field_width(const cuvhs_ctx* ctx);
int cuvhs_field_height(const cuvhs_ctx* ctx);
int cuvhs_lines_per_frame(const cuvhs_ctx* ctx);
size_t cuvhs_samples_per_field(const cuvhs_ctx* ctx); /* samples_per_line * 263 (NTSC) or 313 (PAL) */
size_t cuvhs_tile_stride(const cuvhs_ctx* ctx);       /* samples per chunk field slot (+20 lines) */
/* Forget carried state (field parity, line-location and chroma track state). */
void cuvhs_reset(cuvhs_ctx* ctx);

/* The state a decode carries from one chunk to the next: the parity of the
 * last field written (the reference's static last_parity,
 * src/pipeline/pipeline.cu:2575), the line-location history (Pipeline's
 * k2b_prev_* members, src/pipeline/pipeline.h:92-97; prev_first_hsync_loc is
 * relative to the chunk it was found in, as the reference keeps it) and the
 * chroma track and phase cycle (ChromaState, src/pipeline/chroma_decode.h:9-15).
 * Reading it after a chunk and writing it into another context before the
 * next chunk continues the decode there exactly: a capture split into
 * segments decodes as one. */
typedef struct cuvhs_state {
  int32_t last_parity;
  int32_t prev_first_field;
  int32_t prev_progressive_field;
  int32_t chroma_valid;
  int64_t prev_first_hsync_readloc;
  double prev_first_hsync_loc;
  double prev_first_hsync_diff;
  double chroma_threshold;
  int32_t chroma_track;
  int32_t chroma_cycle_start;
} cuvhs_state;
cuvhs_status cuvhs_get_state(const cuvhs_ctx* ctx, cuvhs_state* state);
cuvhs_status cuvhs_set_state(cuvhs_ctx* ctx, const cuvhs_state* state);

/* One chunk of at most batch_fields fields starting at capture sample raw_offset.
 * `samples` points at that sample in host memory, n_avail samples remain from
 * there.  Appends to `out` (fields_out, dropouts_out grow) and sets
 * out->next_raw_offset.  A chunk that yields no field leaves fields_out unchanged. */
cuvhs_status cuvhs_decode_chunk(cuvhs_ctx* ctx, const uint8_t* samples, size_t n_avail, uint64_t raw_offset,
                                int num_fields, cuvhs_output* out);

/* cuvhs_decode_chunk without waiting for the output planes: when out's luma
 * and chroma are page-locked host memory with room for the chunk, the call
 * returns once the field metadata and dropout lists are in `out`, while the
 * planes are still being copied there, so the next chunk's decode overlaps
 * them.  The planes are complete after cuvhs_flush.  With pageable planes it
 * is cuvhs_decode_chunk. */
cuvhs_status cuvhs_decode_chunk_async(cuvhs_ctx* ctx, const uint8_t* samples, size_t n_avail, uint64_t raw_offset,
                                      int num_fields, cuvhs_output* out);
/* Waits for everything the context still has in flight (plane copies of
 * cuvhs_decode_chunk_async, input prefetches); afterwards every result that a
 * call reported is in the caller's memory.  Returns the first CUDA error of
 * that work.  The reference's calls are synchronous and need no flush. */
cuvhs_status cuvhs_flush(cuvhs_ctx* ctx);

/* The same chunk decode on samples already in device memory; the luma/chroma
 * TBC and dropout results stay on the device (read them with
 * cuvhs_device_outputs).  *fields_out = fields decoded. */
cuvhs_status cuvhs_decode_chunk_device(cuvhs_ctx* ctx, const uint8_t* d_samples, size_t n_avail,
                                       uint64_t raw_offset, int num_fields, int* fields_out,
                                       uint64_t* next_raw_offset);
/* Device pointers to the last chunk's luma and chroma fields. */
cuvhs_status cuvhs_device_outputs(const cuvhs_ctx* ctx, const uint16_t** d_luma, const uint16_t** d_chroma);

/* A whole capture in host memory, chunk by chunk as the reference's run loop.
 * For every decode call, `samples` holds samples of the configured input
 * format (1 byte each for u8, 2 for s16/u16) and sizes count samples. */
cuvhs_status cuvhs_decode_capture(cuvhs_ctx* ctx, const uint8_t* samples, size_t n, cuvhs_output* out);

/* .tbc.json text for `out`'s fields; returns the length (excluding NUL) and
 * writes at most cap bytes including the NUL. */
long long cuvhs_json(const cuvhs_ctx* ctx, const cuvhs_output* out, char* dst, long long cap);

/* The CLI path: decode a u8 capture file (or "-" for stdin) to
 * <out_base>.tbc, <out_base>_chroma.tbc and <out_base>.tbc.json. */
cuvhs_status cuvhs_decode_file(const cuvhs_config* cfg, const char* in_path, const char* out_base,
                               int overwrite);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events against the decoder. */
void* cuvhs_stream(const cuvhs_ctx* ctx);

/* Per-stage device time: with timing on, every kernel launch is bracketed by
 * CUDA events on the decode stream and its duration accumulated per stage.
 * cuvhs_stage_times fills up to cap entries (ms, launches) and returns the
 * number of stages.  No counterpart in the reference, which has no
 * per-stage timers. */
void cuvhs_set_timing(cuvhs_ctx* ctx, int on);
/* Which device stages the timing brackets with events (bit i = stage i;
 * default all).  Each bracket costs host time on the decode's critical path,
 * so a throughput measurement times only the stage it reports. */
void cuvhs_set_timing_mask(cuvhs_ctx* ctx, unsigned mask);
int cuvhs_stage_count(void);
const char* cuvhs_stage_name(int i);
int cuvhs_stage_times(const cuvhs_ctx* ctx, double* ms, long long* launches, int cap);
void cuvhs_reset_stage_times(cuvhs_ctx* ctx);
/* With timing on, the last chunk decode's device stage intervals in launch
 * order: stage index and start / end in ms from the chunk's first timed event
 * (so the gaps between intervals are time the GPU spent waiting on the host).
 * Fills up to cap entries; returns the number of intervals. */
int cuvhs_stage_timeline(const cuvhs_ctx* ctx, int* stage, double* start_ms, double* end_ms, int cap);
/* Kernel launches issued since the last cuvhs_reset_stage_times. */
long long cuvhs_launch_count(const cuvhs_ctx* ctx);

/* Keep host copies of the last chunk's intermediates (costs copies). */
void cuvhs_set_debug(cuvhs_ctx* ctx, int on);
/* Copy an intermediate of the last chunk into dst (cap elements; dst NULL
 * queries the count).  int32: "meta"(raw_offset lo/hi words excluded: tiles,
 * fields, spp), "vsync_candidates", "k2_pulse_count", "k2_pulse_starts",
 * "k2_pulse_lengths", "k2b_pulse_count", "k2b_pulse_starts", "k2b_pulse_lengths",
 * "k2b_pulse_types", "is_first", "do_count", "do_lines", "do_starts", "do_ends";
 * int64: "field_offsets"; float64: "linelocs_coarse", "linelocs"; float32 (Hz
 * relative to the 0 IRE carrier, or raw units): "demod", "video", "sync",
 * "envelope", "chroma_prefilt".  Returns -1 for an unknown name. */
long long cuvhs_debug_array(const cuvhs_ctx* ctx, const char* name, void* dst, long long cap);

/* ---------------------------------------------------------------- stages
 * One stage of the decode at a time on caller-owned buffers, for parity tests
 * of single stages and for callers that compose their own pipeline.  Each
 * entry point is the counterpart of one stage function of the reference's
 * Pipeline::process_chunk (src/pipeline/pipeline.cu:1557-2548), runs the same
 * kernels and host code as cuvhs_decode_chunk on the context's stream and
 * scratch, shares its carried state (line-location history, chroma track and
 * phase cycle) and returns when its results are complete.
 *   A chunk is `tiles` field slots of cuvhs_tile_stride samples (tiles and
 * n_fields at most cuvhs_batch_fields); chunk positions count samples from
 * the chunk's first sample.  d_ arguments are device memory, the rest host
 * memory.  Signals are FP32: video and sync in Hz relative to the 0 IRE
 * frequency (cuvhs_ire0_hz), the envelope as |analytic signal| in the
 * reference's scale.  Line locations are FP64 chunk positions,
 * cuvhs_lines_per_frame per field; TBC fields have the cuvhs_field_width x
 * cuvhs_field_height geometry.
 * The dropout stage (dropout_detect, src/pipeline/dropout_detect.h:22-32) is
 * cuvhs_dropouts_noalloc below. */
#define CUVHS_MAX_PULSES_PER_FIELD 800
#define CUVHS_LINES_PER_FRAME 525 /* NTSC; cuvhs_lines_per_frame gives the context's */
double cuvhs_ire0_hz(const cuvhs_ctx* ctx);
/* The sync pulse threshold in Hz (0 IRE minus 20 IRE, VideoFormat's
 * pulse_threshold_hz, src/format/video_format.cpp:23-104): sync samples at or
 * below it are inside a pulse. */
double cuvhs_pulse_threshold_hz(const cuvhs_ctx* ctx);

/* fm_demod (src/pipeline/fm_demod.h:46-53): d_raw holds n_read samples of the
 * configured input format (positions past n_read count as 0, the reference's
 * zero fill); d_video, d_sync, d_envelope [tiles * tile_stride]. */
cuvhs_status cuvhs_stage_fm_demod(cuvhs_ctx* ctx, const void* d_raw, size_t n_read, int tiles, float* d_video,
                                  float* d_sync, float* d_envelope);

/* discover_vsyncs (src/pipeline/vsync_discover.h:6-11) and the clustering of
 * its candidates (src/pipeline/pipeline.cu:1567-1651): the field windows'
 * starts (field_offsets, room for max_fields), their count, and where the
 * next chunk starts (next_offset, may be NULL), all chunk positions.  Pass
 * the chunk's requested field count as max_fields, as the reference caps it
 * (pipeline.cu:1622-1624): a window can start past the last demodulated tile,
 * so n_fields may exceed tiles by one. */
cuvhs_status cuvhs_stage_discover_vsyncs(cuvhs_ctx* ctx, const float* d_sync, int tiles, int max_fields,
                                         int64_t* field_offsets, int* n_fields, int64_t* next_offset);

/* sync_pulses (src/pipeline/sync_pulses.h:20-27) with per-field offsets:
 * starts/lengths [n_fields * CUVHS_MAX_PULSES_PER_FIELD], counts [n_fields]. */
cuvhs_status cuvhs_stage_sync_pulses(cuvhs_ctx* ctx, const float* d_sync, int tiles, const int64_t* field_offsets,
                                     int n_fields, int32_t* starts, int32_t* lengths, int32_t* counts);

/* The host line locations that follow sync_pulses (src/pipeline/pipeline.cu:1717-1778):
 * pulse validation, field order, blanking anchor and the snapped line grid,
 * field by field with the field-order state carried across fields and calls.
 * raw_offset is the capture sample of the chunk's first sample.  linelocs
 * [n_fields * lines_per_frame]; is_first_field [n_fields] (may be NULL) = 1, 0, or -1. */
cuvhs_status cuvhs_stage_line_locations(cuvhs_ctx* ctx, uint64_t raw_offset, const int64_t* field_offsets,
                                        int n_fields, const int32_t* starts, const int32_t* lengths,
                                        const int32_t* counts, double* linelocs, int32_t* is_first_field);

/* hsync_refine (src/pipeline/hsync_refine.h:18-22): refines d_linelocs
 * [n_fields * lines_per_frame] in place.  d_sync holds `tiles` slots; the refinement
 * reads min(n_fields, tiles) * tile_stride samples of it (the reference's
 * total_demod_samples = n_fields * tile_stride when the buffer covers them). */
cuvhs_status cuvhs_stage_hsync_refine(cuvhs_ctx* ctx, const float* d_sync, int tiles, double* d_linelocs,
                                      int n_fields);

/* tbc_resample (src/pipeline/tbc_resample.h:16-27): d_luma [n_fields][height][width];
 * d_video holds `tiles` slots, read as hsync_refine reads d_sync. */
cuvhs_status cuvhs_stage_tbc_resample(cuvhs_ctx* ctx, const float* d_video, int tiles, const double* d_linelocs,
                                      int n_fields, uint16_t* d_luma);

/* chroma_decode (src/pipeline/chroma_decode.h:38-46): the colour-under chroma
 * of n_fields fields from the raw chunk (n_read samples of the configured
 * format) into d_chroma [n_fields][height][width]; field_phase_ids [n_fields] (may
 * be NULL) receives the NTSC field phase IDs.  The first call after create or
 * cuvhs_reset detects the track and phase cycle; later calls carry them. */
cuvhs_status cuvhs_stage_chroma_decode(cuvhs_ctx* ctx, const void* d_raw, size_t n_read, const double* d_linelocs,
                                       int n_fields, uint16_t* d_chroma, int32_t* field_phase_ids);

/* Dropout detection and concealment on caller-owned device buffers, allocating
 * no device memory, for NTSC fields (525 line locations, 910x263 TBC fields,
 * active lines from 10).  No counterpart in the reference (its dropout stage
 * allocates a temporary on every call).  For callers that cannot call
 * cudaMalloc: code running while its stream is captured into a CUDA graph,
 * real-time capture loops that must not block in the allocator, and hosts
 * whose device memory belongs to another allocator.
 *   d_envelope  [fields * tile_stride] f32 RF envelope; field f's slot starts
 *               at f * tile_stride (the decoder's layout, see cuvhs_tile_stride)
 *   d_linelocs  [fields * 525] f64 line starts in the same sample units
 *   d_luma, d_chroma  [fields][263][910] u16 TBC fields, concealed in place
 *   d_count [fields], d_lines/d_startx/d_endx [fields * 512]  outputs
 *   stream      a cudaStream_t (NULL = default stream); the call is asynchronous
 * The only scratch is a fixed device array of CUVHS_NOALLOC_MAX_PARTIALS
 * doubles (256 KiB, one per envelope block of the decoder's demodulator:
 * 3,327 samples at 28 MHz, 2,943 at 40 MHz), shared by all calls on a device
 * and held by every GPU that loads the library until the process exits:
 * calls that overlap on the GPU race on it.  Sizes needing more partial sums
 * (about 215 fields at 28 MHz, 156 at 35.8 MHz, 133 at 40 MHz) return
 * CUVHS_ERR_CAPACITY.  The first call on each device (and again in a new
 * context, e.g. after cudaDeviceReset) looks up the array's device address;
 * make that first call before any stream capture.  An error left pending by
 * an earlier CUDA call is left pending and the call returns CUVHS_ERR_CUDA
 * without launching anything. */
#define CUVHS_NOALLOC_MAX_PARTIALS 32768
cuvhs_status cuvhs_dropouts_noalloc(const float* d_envelope, const double* d_linelocs, int fields, int tile_stride,
                                    uint16_t* d_luma, uint16_t* d_chroma, int32_t* d_count, int32_t* d_lines,
                                    int32_t* d_startx, int32_t* d_endx, void* stream);

/* ---------------------------------------------------------------- batches
 * Many independent captures (mixed sample rates and lengths) decoded together
 * on one GPU.  Captures of one sample rate are decoded in rounds: each round
 * takes the next chunk of up to 64 captures, places them in consecutive field
 * slots of one context's buffers and runs every stage as one launch over all
 * of them (grid.z picks the capture), so a stage's launch, its host waits and
 * the GPU's fill are shared by the whole round.  `lanes` host threads each
 * drive rounds on their own contexts (one per sample rate), so one lane's
 * host decisions overlap another's kernels.  The field slots per round come
 * from an autotuner (timed rounds of a synthetic probe at each candidate
 * size, once per sample rate and batch object) unless round_fields is given.
 * Every capture is decoded from a fresh state exactly as cuvhs_decode_capture
 * on a new context with a chunk of max_fields fields would decode it: outputs
 * do not depend on the lane count, the round size or the order of the items. */
typedef struct cuvhs_batch cuvhs_batch;

typedef struct cuvhs_batch_config {
  int device;       /* CUDA device id, -1 = the one with most memory */
  int lanes;        /* concurrent round drivers; 0 = 4 */
  int max_fields;   /* chunk size of every capture; 0 = 256 (one chunk per capture of up
                       to 256 fields, as a single-capture decode with the default
                       chunk size) */
  int round_fields; /* field slots per round (at least max_fields); 0 = autotune */
} cuvhs_batch_config;

typedef struct cuvhs_batch_item {
  const uint8_t* samples;  /* host capture (page-locked memory lets copies overlap) */
  size_t n;                /* samples */
  double sample_rate_mhz;
  cuvhs_output* out;       /* caller-owned, as for cuvhs_decode_capture */
  cuvhs_status status;     /* filled in per item */
} cuvhs_batch_item;

cuvhs_status cuvhs_batch_create(const cuvhs_batch_config* cfg, cuvhs_batch** out);
void cuvhs_batch_destroy(cuvhs_batch* b);
int cuvhs_batch_lanes(const cuvhs_batch* b);
/* Decode all items; returns CUVHS_OK when every item's status is CUVHS_OK,
 * else the first failing item's status (cuvhs_batch_last_error has its message). */
cuvhs_status cuvhs_batch_decode(cuvhs_batch* b, cuvhs_batch_item* items, int n_items);
const char* cuvhs_batch_last_error(const cuvhs_batch* b);
/* .tbc.json text of one decoded item (as cuvhs_json for a single capture). */
long long cuvhs_batch_json(const cuvhs_batch_item* item, char* dst, long long cap);
/* Field slots per round the batch uses for captures at this sample rate
 * (after the autotuner ran for it, or round_fields); 0 before first use. */
int cuvhs_batch_round_fields(const cuvhs_batch* b, double sample_rate_mhz);
/* Per-stage device times summed over the batch's contexts (as
 * cuvhs_stage_times), recorded while timing is on. */
void cuvhs_batch_set_timing(cuvhs_batch* b, int on);
int cuvhs_batch_stage_times(const cuvhs_batch* b, double* ms, long long* launches, int cap);

/* ------------------------------------------------------------- calibration
 * A differentiable decode model and its adjoint, for calibrating a tape's
 * decode parameters against a known test pattern.  No counterpart in the
 * reference, which has no gradients.  cuvhs_adjoint_create decodes the
 * capture's first `fields` fields with the normal decoder and keeps, on the
 * device, what the parameter-dependent part of the decode starts from: the
 * FM demod, the colour-under pre-band-pass, the refined line locations and
 * the chroma tracks.  The model then redoes, for parameters
 *   de-emphasis  H(z) = (n0 + n1 z^-1 + n2 z^-2) / (1 + m1 z^-1 + m2 z^-2),
 *                n0 = 1 + m1 + m2 - n1 - n2 (unit DC gain), times the
 *                decoder's 3 MHz super-Gaussian video low-pass,
 *   carrier_hz   FM carrier offset removed from the video,
 *   deviation    FM deviation scale,
 *   line_offset  per-line start offsets (samples) added to the line locations,
 *   chroma_phase per-line colour-under phase offsets (radians),
 * the video filter, the Catmull-Rom luma and chroma resampling, the
 * heterodyne, the 1024-point chroma line band-pass and the burst-driven ACC
 * gain (FP32 samples, FP64 positions), and
 *   L = mean (Y - Y*)^2 + mean (C - C*)^2
 * over lines 10..261, columns 80..893 (back porch with the burst, and the
 * active picture) of every field, in TBC units, against target planes.  cuvhs_adjoint_bwd returns dL/d every
 * parameter through hand-written adjoint kernels, recomputing the forward
 * quantities it needs instead of storing them. */
typedef struct cuvhs_adjoint cuvhs_adjoint;

#define CUVHS_ADJOINT_ROWS 264 /* line_offset entries per field (rows 0..263) */

typedef struct cuvhs_adjoint_params {
  double deemph[4];      /* n1, n2, m1, m2 */
  double carrier_hz;
  double deviation;
  double* line_offset;   /* [fields * CUVHS_ADJOINT_ROWS] */
  double* chroma_phase;  /* [fields * CUVHS_FIELD_HEIGHT] */
} cuvhs_adjoint_params;

cuvhs_status cuvhs_adjoint_create(const cuvhs_config* cfg, const uint8_t* samples, size_t n, int fields,
                                  cuvhs_adjoint** out);
void cuvhs_adjoint_destroy(cuvhs_adjoint* a);
int cuvhs_adjoint_fields(const cuvhs_adjoint* a); /* fields the model covers (<= requested) */
/* Nominal parameters (the decoder's own de-emphasis, no offsets); the caller
 * provides the per-line arrays, which are zeroed. */
cuvhs_status cuvhs_adjoint_default_params(const cuvhs_adjoint* a, cuvhs_adjoint_params* p);
/* Target planes [fields][263][910] in TBC units. */
cuvhs_status cuvhs_adjoint_set_target(cuvhs_adjoint* a, const float* luma, const float* chroma);
/* Forward: the loss (needs a target) and, optionally, the model's planes. */
cuvhs_status cuvhs_adjoint_fwd(cuvhs_adjoint* a, const cuvhs_adjoint_params* p, double* loss, float* luma,
                               float* chroma);
/* Backward: the loss and dL/dparameters into grad (whose arrays the caller provides). */
cuvhs_status cuvhs_adjoint_bwd(cuvhs_adjoint* a, const cuvhs_adjoint_params* p, double* loss,
                               cuvhs_adjoint_params* grad);
/* Model inputs and state for inspection: "linelocs" (f64, fields*525),
 * "gains" (f32, fields*263, the ACC gains of the last pass), "tracks" (i32,
 * fields), "demod" and "pre" (f32, fields*tile_stride).  Returns the element
 * count; copies at most cap. */
long long cuvhs_adjoint_array(const cuvhs_adjoint* a, const char* name, void* dst, long long cap);

#ifdef __cplusplus
}
#endif
#endif
