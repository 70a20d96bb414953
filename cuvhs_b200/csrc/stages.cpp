// Stage-level entry points (include/cuvhs.h): one stage of the decode on
// caller-owned buffers, each the counterpart of one stage function of the
// reference's Pipeline::process_chunk (src/pipeline/pipeline.cu:1557-2548).
// They run the same kernels and host helpers as Context::decode_chunk, on the
// context's stream and scratch, and share its carried state.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cuvhs.h"
#include "pipeline.h"

namespace {

using cuvhs::Context;

cuvhs_status bad(Context& c, const std::string& msg) {
  c.status = CUVHS_ERR_INVALID_ARGUMENT;
  c.err = msg;
  return c.status;
}

// Common entry: clears the status, selects the device and checks a field or
// tile count against the context's allocation.
bool enter(Context& c, int n, const char* what) {
  c.status = CUVHS_OK;
  c.err.clear();
  if (n < 1 || n > c.batch) {
    bad(c, std::string(what) + " must be in [1, batch_fields]");
    return false;
  }
  cudaSetDevice(c.device);
  return true;
}

}  // namespace

extern "C" {

double cuvhs_ire0_hz(const cuvhs_ctx* ctx) { return ctx ? ctx->c.fmt.ire0 : 0.0; }
double cuvhs_pulse_threshold_hz(const cuvhs_ctx* ctx) { return ctx ? ctx->c.fmt.pulse_threshold_hz : 0.0; }

// fm_demod (src/pipeline/fm_demod.cu:396-485): K1a and K1b over `tiles` slots.
cuvhs_status cuvhs_stage_fm_demod(cuvhs_ctx* ctx, const void* d_raw, size_t n_read, int tiles, float* d_video,
                                  float* d_sync, float* d_envelope) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  if (!d_raw || !d_video || !d_sync || !d_envelope) return bad(c, "null buffer");
  if (!enter(c, tiles, "tiles")) return c.status;
  const size_t total = (size_t)tiles * c.spp;
  n_read = std::min(n_read, total);
  cuvhs::DemodArgs da = c.demod_args(tiles);
  da.raw = static_cast<const uint8_t*>(d_raw);
  da.n_read = (int)n_read;
  da.env = d_envelope;
  da.video = d_video;
  da.sync = d_sync;
  cudaEvent_t ev;
  c.begin_stage(cuvhs::kStageK1a, ev);
  if (c.dc_correct) cuvhs::launch_dc_mean(da.raw, (int)n_read, c.in_fmt, c.d_dcsum, c.d_dc, c.stream);
  cuvhs::launch_k1a(da, 0, tiles, c.stream);
  c.end_stage(cuvhs::kStageK1a, ev, c.dc_correct ? 3 : 1);
  cudaMemsetAsync(c.d_guard_count, 0, sizeof(int), c.stream);
  c.begin_stage(cuvhs::kStageK1b, ev);
  cuvhs::launch_k1b(da, 0, tiles, c.stream);
  c.end_stage(cuvhs::kStageK1b, ev);
  c.begin_stage(cuvhs::kStageGuard, ev);
  cuvhs::launch_sync_guard(c.guard_args(da), c.stream);
  c.end_stage(cuvhs::kStageGuard, ev);
  cudaMemcpyAsync(c.hp_guard, c.d_guard_count, sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  if (!c.check_cuda("fm_demod") || !c.sync("fm_demod")) return c.status;
  if (!c.guard_ok(*c.hp_guard)) return c.status;
  return CUVHS_OK;
}

// discover_vsyncs (src/pipeline/vsync_discover.cu:5-72) and the clustering of
// its candidates into field windows (src/pipeline/pipeline.cu:1567-1651).
cuvhs_status cuvhs_stage_discover_vsyncs(cuvhs_ctx* ctx, const float* d_sync, int tiles, int max_fields,
                                         int64_t* field_offsets, int* n_fields, int64_t* next_offset) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  if (!d_sync || !field_offsets || !n_fields) return bad(c, "null buffer");
  if (!enter(c, tiles, "tiles")) return c.status;
  if (max_fields < 1) return bad(c, "max_fields must be positive");
  const long long total = (long long)tiles * c.spp;
  const int nf = std::min(max_fields, c.batch);
  if (!c.field_windows(d_sync, total, tiles, nf)) return c.status;
  *n_fields = c.hp_win->fields;
  for (int i = 0; i < c.hp_win->fields; i++) field_offsets[i] = (int64_t)c.hp_offs[i];
  if (next_offset) *next_offset = (int64_t)c.hp_win->next_rel;
  return CUVHS_OK;
}

namespace {

// The field windows of a stage call on the device: n windows at the given
// chunk offsets.
bool upload_windows(Context& c, const int64_t* field_offsets, int n) {
  cuvhs::WindowInfo w;
  w.fields = n;
  for (int f = 0; f < n; f++) c.hp_offs[f] = (long long)field_offsets[f];
  *c.hp_win = w;
  cudaMemcpyAsync(c.d_win, c.hp_win, sizeof(w), cudaMemcpyHostToDevice, c.stream);
  if (n) cudaMemcpyAsync(c.d_offs, c.hp_offs, (size_t)n * sizeof(long long), cudaMemcpyHostToDevice, c.stream);
  return c.check_cuda("window upload");
}

}  // namespace

// sync_pulses (src/pipeline/sync_pulses.cu:10-82) over per-field windows.
cuvhs_status cuvhs_stage_sync_pulses(cuvhs_ctx* ctx, const float* d_sync, int tiles, const int64_t* field_offsets,
                                     int n_fields, int32_t* starts, int32_t* lengths, int32_t* counts) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  if (!d_sync || !field_offsets || !starts || !lengths || !counts) return bad(c, "null buffer");
  if (!enter(c, tiles, "tiles")) return c.status;
  if (n_fields < 0 || n_fields > c.batch) return bad(c, "n_fields must be in [0, batch_fields]");
  const long long total = (long long)tiles * c.spp;
  for (int f = 0; f < n_fields; f++)
    if (field_offsets[f] < 0 || field_offsets[f] >= total) return bad(c, "field offset outside the chunk");
  if (n_fields == 0) return CUVHS_OK;
  if (!c.field_windows(d_sync, total, tiles, 1)) return c.status;  // the chunk's edge lists
  if (!upload_windows(c, field_offsets, n_fields)) return c.status;
  cuvhs::LineLocArgs la = c.lineloc_args(tiles, n_fields, 0);
  la.total = total;
  cuvhs::launch_field_pulses(la, c.stream);
  std::vector<int32_t> ps((size_t)n_fields * cuvhs::kMaxPulses), pl(ps.size());
  cudaMemcpyAsync(counts, c.d_pn, n_fields * sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(ps.data(), c.d_ps, ps.size() * sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(pl.data(), c.d_pl, pl.size() * sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  if (!c.check_cuda("sync_pulses") || !c.sync("sync_pulses")) return c.status;
  for (int f = 0; f < n_fields; f++) {
    const size_t o = (size_t)f * cuvhs::kMaxPulses;
    std::copy(ps.begin() + o, ps.begin() + o + counts[f], starts + o);
    std::copy(pl.begin() + o, pl.begin() + o + counts[f], lengths + o);
  }
  return CUVHS_OK;
}

// The host line locations of src/pipeline/pipeline.cu:1717-1778 ("K2b"), in
// field order with the carried field-order state; or, with the single-pass
// locator selected, src/pipeline/line_locs.cu:544-593 (no carried state).
cuvhs_status cuvhs_stage_line_locations(cuvhs_ctx* ctx, uint64_t raw_offset, const int64_t* field_offsets,
                                        int n_fields, const int32_t* starts, const int32_t* lengths,
                                        const int32_t* counts, double* linelocs, int32_t* is_first_field) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  if (!field_offsets || !starts || !lengths || !counts || !linelocs) return bad(c, "null buffer");
  c.status = CUVHS_OK;
  c.err.clear();
  if (n_fields < 0 || n_fields > c.batch) return bad(c, "n_fields must be in [0, batch_fields]");
  if (n_fields == 0) return CUVHS_OK;
  cudaSetDevice(c.device);
  const int LPF = c.fmt.lines_per_frame;
  c.single_pass = c.cfg.single_pass_lines != 0 || std::getenv("CUVHS_K2B_DISABLE") != nullptr;
  std::vector<int32_t> pn(n_fields);
  for (int f = 0; f < n_fields; f++) pn[f] = std::max(0, std::min<int>(counts[f], cuvhs::kMaxPulses));
  const size_t np = (size_t)n_fields * cuvhs::kMaxPulses;
  if (!upload_windows(c, field_offsets, n_fields)) return c.status;
  cudaMemcpyAsync(c.d_ps, starts, np * sizeof(int), cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_pl, lengths, np * sizeof(int), cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_pn, pn.data(), n_fields * sizeof(int), cudaMemcpyHostToDevice, c.stream);
  cuvhs::LineLocArgs la = c.lineloc_args(n_fields, n_fields, (long long)raw_offset);
  cuvhs::launch_line_locations(la, c.stream);
  std::vector<int32_t> first(n_fields);
  cudaMemcpyAsync(linelocs, c.d_ll, (size_t)n_fields * LPF * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(first.data(), c.d_is_first, n_fields * sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  if (!c.check_cuda("line_locations") || !c.sync("line_locations")) return c.status;
  if (is_first_field) std::copy(first.begin(), first.end(), is_first_field);
  return CUVHS_OK;
}

// hsync_refine (src/pipeline/hsync_refine.cu:21-271).
cuvhs_status cuvhs_stage_hsync_refine(cuvhs_ctx* ctx, const float* d_sync, int tiles, double* d_linelocs,
                                      int n_fields) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  if (!d_sync || !d_linelocs) return bad(c, "null buffer");
  if (!enter(c, n_fields, "n_fields")) return c.status;
  if (tiles < 1) return bad(c, "tiles must be positive");
  cuvhs::LineArgs la = c.line_args(n_fields);
  la.total = (long long)std::min(n_fields, tiles) * c.spp;  // every read stays inside d_sync
  la.sync = d_sync;
  la.ll = d_linelocs;
  cudaEvent_t ev;
  c.begin_stage(cuvhs::kStageHsync, ev);
  cuvhs::launch_hsync_refine(la, c.stream);
  c.end_stage(cuvhs::kStageHsync, ev);
  if (!c.check_cuda("hsync_refine") || !c.sync("hsync_refine")) return c.status;
  return CUVHS_OK;
}

// tbc_resample (src/pipeline/tbc_resample.cu:19-186).
cuvhs_status cuvhs_stage_tbc_resample(cuvhs_ctx* ctx, const float* d_video, int tiles, const double* d_linelocs,
                                      int n_fields, uint16_t* d_luma) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  if (!d_video || !d_linelocs || !d_luma) return bad(c, "null buffer");
  if (!enter(c, n_fields, "n_fields")) return c.status;
  if (tiles < 1) return bad(c, "tiles must be positive");
  cuvhs::LineArgs la = c.line_args(n_fields);
  la.total = (long long)std::min(n_fields, tiles) * c.spp;  // every read stays inside d_video
  la.video = d_video;
  la.ll = const_cast<double*>(d_linelocs);  // the resampler only reads it
  la.luma = d_luma;
  cudaEvent_t ev;
  c.begin_stage(cuvhs::kStageLuma, ev);
  cuvhs::launch_luma(la, c.stream);
  c.end_stage(cuvhs::kStageLuma, ev);
  if (!c.check_cuda("tbc_resample") || !c.sync("tbc_resample")) return c.status;
  return CUVHS_OK;
}

// chroma_decode (src/pipeline/chroma_decode.cu:526-1002): pre-band-pass of
// the raw chunk, then the line decode with the track and phase decisions.
cuvhs_status cuvhs_stage_chroma_decode(cuvhs_ctx* ctx, const void* d_raw, size_t n_read, const double* d_linelocs,
                                       int n_fields, uint16_t* d_chroma, int32_t* field_phase_ids) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  if (!d_raw || !d_linelocs || !d_chroma) return bad(c, "null buffer");
  if (!enter(c, n_fields, "n_fields")) return c.status;
  const size_t total = (size_t)n_fields * c.spp;
  n_read = std::min(n_read, total);
  const uint8_t* raw = static_cast<const uint8_t*>(d_raw);
  if (c.dc_correct) cuvhs::launch_dc_mean(raw, (int)n_read, c.in_fmt, c.d_dcsum, c.d_dc, c.stream);
  cuvhs::ChromaArgs ca = c.chroma_args(raw, (int)n_read, c.dc_correct ? c.d_dc : nullptr, n_fields);
  ca.ll = d_linelocs;
  ca.chroma = d_chroma;
  ca.total = (long long)total;
  cudaEvent_t ev;
  c.begin_stage(cuvhs::kStageChromaPre, ev);
  cuvhs::launch_chroma_prefilter(ca, c.stream);
  c.end_stage(cuvhs::kStageChromaPre, ev);
  if (!c.check_cuda("chroma prefilter")) return c.status;
  if (!c.chroma_fields(ca, n_fields)) return c.status;
  if (!c.check_cuda("chroma_decode") || !c.sync("chroma_decode")) return c.status;
  if (field_phase_ids)
    for (int f = 0; f < n_fields; f++) field_phase_ids[f] = c.h_phase[f];
  return CUVHS_OK;
}

}  // extern "C"
