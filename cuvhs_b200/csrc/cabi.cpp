// extern "C" entry points of libcuvhs (declared in include/cuvhs.h).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cuvhs.h"
#include "pipeline.h"

namespace {

using cuvhs::ChunkResult;
using cuvhs::Context;

cuvhs_status fail(Context& c, cuvhs_status s, const std::string& msg) {
  c.status = s;
  c.err = msg;
  return s;
}

// Copy one chunk's results to the caller's host buffers (appending).
cuvhs_status append_chunk(Context& c, const ChunkResult& r, cuvhs_output* out) {
  const size_t F = (size_t)c.fmt.output_line_len * c.fmt.output_field_lines;
  if (out->fields_out + (size_t)r.fields > out->max_fields)
    return fail(c, CUVHS_ERR_CAPACITY, "output field buffer too small");
  size_t need = 0;
  for (int i = 0; i < r.fields; i++) need += (size_t)r.field_info[i].dropout_count;
  if (out->dropouts_out + need > out->max_dropouts && need > 0)
    return fail(c, CUVHS_ERR_CAPACITY, "output dropout buffer too small");
  if (r.fields > 0 && !r.outputs_copied) {
    if (out->luma)
      cudaMemcpyAsync(out->luma + out->fields_out * F, c.d_luma, (size_t)r.fields * F * sizeof(uint16_t),
                      cudaMemcpyDeviceToHost, c.stream);
    if (out->chroma)
      cudaMemcpyAsync(out->chroma + out->fields_out * F, c.d_chroma, (size_t)r.fields * F * sizeof(uint16_t),
                      cudaMemcpyDeviceToHost, c.stream);
    if (!c.sync("output copy")) return c.status;
  }
  for (int i = 0; i < r.fields; i++) {
    cuvhs_field_info fi = r.field_info[i];
    fi.dropout_offset = (int32_t)out->dropouts_out;
    for (int d = 0; d < fi.dropout_count; d++) {
      const size_t k = (size_t)i * cuvhs::kMaxDropouts + d;
      if (out->dropout_line) out->dropout_line[out->dropouts_out] = c.hp_do_lines[k];
      if (out->dropout_startx) out->dropout_startx[out->dropouts_out] = c.hp_do_starts[k];
      if (out->dropout_endx) out->dropout_endx[out->dropouts_out] = c.hp_do_ends[k];
      out->dropouts_out++;
    }
    if (out->fields) out->fields[out->fields_out] = fi;
    out->fields_out++;
  }
  out->next_raw_offset = r.next_raw_offset;
  return CUVHS_OK;
}

bool page_locked(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

// Decode one chunk into `out`.  When the caller's planes are page-locked and
// have room for every field the chunk can produce, the decoder copies each
// plane there as soon as it is final (overlapping the rest of the decode);
// otherwise the planes are copied after the decode.
cuvhs_status decode_into(Context& c, const uint8_t* src, size_t n_avail, uint64_t raw_offset, int num_fields,
                         cuvhs_output* out, const uint8_t* cap_base = nullptr, size_t cap_n = 0,
                         bool async = false) {
  const size_t F = (size_t)c.fmt.output_line_len * c.fmt.output_field_lines;
  uint16_t *dl = nullptr, *dc = nullptr;
  // a chunk yields at most min(num_fields, n_avail / samples_per_field) fields
  const size_t most = std::min<size_t>((size_t)std::max(num_fields, 0), n_avail / (size_t)c.fmt.samples_per_field);
  if (out->fields_out + most <= out->max_fields) {
    if (page_locked(out->luma)) dl = out->luma + out->fields_out * F;
    if (page_locked(out->chroma)) dc = out->chroma + out->fields_out * F;
    if ((out->luma && !dl) || (out->chroma && !dc)) dl = dc = nullptr;  // both or neither
  }
  ChunkResult r;
  // a chunk of a whole page-locked capture prefetches the next chunk's window
  // and, with page-locked planes, defers its plane copies (the capture loop
  // drains them); so does an asynchronous chunk call (cuvhs_flush drains them)
  if (cap_base && !page_locked(cap_base)) cap_base = nullptr;
  const bool defer = (cap_base != nullptr || async) && (dl || dc);
  if (!c.decode_chunk(src, false, n_avail, raw_offset, num_fields, r, dl, dc, cap_base, cap_n, defer))
    return c.status;
  return append_chunk(c, r, out);
}

template <typename T>
long long copy_out(const std::vector<T>& v, void* dst, long long cap) {
  if (dst && cap > 0) std::memcpy(dst, v.data(), sizeof(T) * (size_t)std::min<long long>(cap, (long long)v.size()));
  return (long long)v.size();
}

template <typename T>
long long copy_ptr(const T* p, size_t n, void* dst, long long cap) {
  if (dst && cap > 0 && p) std::memcpy(dst, p, sizeof(T) * (size_t)std::min<long long>(cap, (long long)n));
  return (long long)n;
}

}  // namespace

namespace cuvhs {

cuvhs_status create_context(const cuvhs_config& cfg, cuvhs_ctx** out) {
  *out = nullptr;
  cuvhs_ctx* h = new (std::nothrow) cuvhs_ctx();
  if (!h) return CUVHS_ERR_OUT_OF_MEMORY;
  if (!h->c.init(cfg)) {
    cuvhs_status s = h->c.status != CUVHS_OK ? h->c.status : CUVHS_ERR_CUDA;
    fprintf(stderr, "cuvhs_create: %s\n", h->c.err.c_str());
    delete h;
    return s;
  }
  *out = h;
  return CUVHS_OK;
}

}  // namespace cuvhs

extern "C" {

void cuvhs_default_config(cuvhs_config* cfg) {
  if (!cfg) return;
  cfg->system = 0;
  cfg->sample_rate_mhz = 28.0;
  cfg->device = 0;
  cfg->batch_fields = 0;
  cfg->stream_mode = 0;
  cfg->input_format = 0;
  cfg->dc_correct = 0;
  cfg->single_pass_lines = 0;
  cfg->guard_band_hz = 0.0;
  cfg->device_memory_limit_mb = 0.0;
}

const char* cuvhs_status_string(cuvhs_status s) {
  switch (s) {
    case CUVHS_OK: return "ok";
    case CUVHS_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CUVHS_ERR_CUDA: return "CUDA error";
    case CUVHS_ERR_OUT_OF_MEMORY: return "out of device memory";
    case CUVHS_ERR_IO: return "I/O error";
    case CUVHS_ERR_CAPACITY: return "capacity exceeded";
    case CUVHS_ERR_UNSUPPORTED: return "unsupported";
    case CUVHS_ERR_EXISTS: return "output exists";
  }
  return "unknown status";
}

cuvhs_status cuvhs_create(const cuvhs_config* cfg, cuvhs_ctx** out) {
  if (!cfg || !out) return CUVHS_ERR_INVALID_ARGUMENT;
  return cuvhs::create_context(*cfg, out);
}

void cuvhs_destroy(cuvhs_ctx* ctx) { delete ctx; }

const char* cuvhs_last_error(const cuvhs_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }
int cuvhs_batch_fields(const cuvhs_ctx* ctx) { return ctx ? ctx->c.batch : 0; }
int cuvhs_field_width(const cuvhs_ctx* ctx) { return ctx ? ctx->c.fmt.output_line_len : 0; }
int cuvhs_field_height(const cuvhs_ctx* ctx) { return ctx ? ctx->c.fmt.output_field_lines : 0; }
int cuvhs_lines_per_frame(const cuvhs_ctx* ctx) { return ctx ? ctx->c.fmt.lines_per_frame : 0; }
size_t cuvhs_samples_per_field(const cuvhs_ctx* ctx) { return ctx ? (size_t)ctx->c.fmt.samples_per_field : 0; }
size_t cuvhs_tile_stride(const cuvhs_ctx* ctx) { return ctx ? (size_t)ctx->c.spp : 0; }
void cuvhs_reset(cuvhs_ctx* ctx) {
  if (ctx) ctx->c.reset_state();
}

cuvhs_status cuvhs_get_state(const cuvhs_ctx* ctx, cuvhs_state* s) {
  if (!ctx || !s) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = const_cast<cuvhs_ctx*>(ctx)->c;  // reading the device state changes nothing
  cudaSetDevice(c.device);
  cuvhs::LineLocState lls;
  if (!c.read_lls(lls)) return c.status;
  *s = cuvhs_state();
  s->last_parity = c.last_parity ? 1 : 0;
  s->prev_first_field = lls.prev_first_field;
  s->prev_progressive_field = lls.prev_progressive_field;
  s->prev_first_hsync_readloc = lls.prev_first_hsync_readloc;
  s->prev_first_hsync_loc = lls.prev_first_hsync_loc;
  s->prev_first_hsync_diff = lls.prev_first_hsync_diff;
  s->chroma_valid = c.chroma_valid ? 1 : 0;
  s->chroma_track = c.chroma_track;
  s->chroma_threshold = c.chroma_threshold;
  s->chroma_cycle_start = c.chroma_cycle_start;
  return CUVHS_OK;
}

cuvhs_status cuvhs_set_state(cuvhs_ctx* ctx, const cuvhs_state* s) {
  if (!ctx || !s) return CUVHS_ERR_INVALID_ARGUMENT;
  if (s->chroma_track < 0 || s->chroma_track > 1 || s->chroma_cycle_start < 0 || s->chroma_cycle_start > 7 ||
      s->prev_first_field < -1 || s->prev_first_field > 1)
    return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  cudaSetDevice(c.device);
  cuvhs::LineLocState lls;
  lls.prev_first_field = s->prev_first_field;
  lls.prev_progressive_field = s->prev_progressive_field;
  lls.prev_first_hsync_readloc = s->prev_first_hsync_readloc;
  lls.prev_first_hsync_loc = s->prev_first_hsync_loc;
  lls.prev_first_hsync_diff = s->prev_first_hsync_diff;
  if (!c.write_lls(lls)) return c.status;
  c.last_parity = s->last_parity != 0;
  c.chroma_valid = s->chroma_valid != 0;
  c.chroma_track = s->chroma_track;
  c.chroma_threshold = s->chroma_threshold;
  c.chroma_cycle_start = s->chroma_cycle_start;
  return CUVHS_OK;
}
void cuvhs_set_debug(cuvhs_ctx* ctx, int on) {
  if (ctx) ctx->c.debug = on != 0;
}

cuvhs_status cuvhs_decode_chunk(cuvhs_ctx* ctx, const uint8_t* samples, size_t n_avail, uint64_t raw_offset,
                                int num_fields, cuvhs_output* out) {
  if (!ctx || !samples || !out) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  c.status = CUVHS_OK;
  return decode_into(c, samples, n_avail, raw_offset, num_fields, out);
}

cuvhs_status cuvhs_decode_chunk_async(cuvhs_ctx* ctx, const uint8_t* samples, size_t n_avail, uint64_t raw_offset,
                                      int num_fields, cuvhs_output* out) {
  if (!ctx || !samples || !out) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  c.status = CUVHS_OK;
  return decode_into(c, samples, n_avail, raw_offset, num_fields, out, nullptr, 0, true);
}

cuvhs_status cuvhs_flush(cuvhs_ctx* ctx) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  c.status = CUVHS_OK;
  cudaSetDevice(c.device);
  if (!c.drain_copies()) return c.status;
  return CUVHS_OK;
}

cuvhs_status cuvhs_decode_chunk_device(cuvhs_ctx* ctx, const uint8_t* d_samples, size_t n_avail,
                                       uint64_t raw_offset, int num_fields, int* fields_out,
                                       uint64_t* next_raw_offset) {
  if (!ctx || !d_samples) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  c.status = CUVHS_OK;
  ChunkResult r;
  if (!c.decode_chunk(d_samples, true, n_avail, raw_offset, num_fields, r)) return c.status;
  if (fields_out) *fields_out = r.fields;
  if (next_raw_offset) *next_raw_offset = r.next_raw_offset;
  return CUVHS_OK;
}

cuvhs_status cuvhs_device_outputs(const cuvhs_ctx* ctx, const uint16_t** d_luma, const uint16_t** d_chroma) {
  if (!ctx) return CUVHS_ERR_INVALID_ARGUMENT;
  if (d_luma) *d_luma = ctx->c.d_luma;
  if (d_chroma) *d_chroma = ctx->c.d_chroma;
  return CUVHS_OK;
}

// Pipeline::run's loop over an in-memory capture (src/pipeline/pipeline.cu:2650-2665).
cuvhs_status cuvhs_decode_capture(cuvhs_ctx* ctx, const uint8_t* samples, size_t n, cuvhs_output* out) {
  if (!ctx || !samples || !out) return CUVHS_ERR_INVALID_ARGUMENT;
  Context& c = ctx->c;
  c.status = CUVHS_OK;
  const size_t spf = (size_t)c.fmt.samples_per_field;
  uint64_t raw_offset = 0;
  while (raw_offset < n) {
    const int remaining_fields = (int)((n - raw_offset) / spf);
    if (remaining_fields <= 0) break;
    const int nf = std::min(c.batch, remaining_fields);
    const size_t before = out->fields_out;
    const uint64_t prev_next = out->next_raw_offset;
    cuvhs_status s = decode_into(c, samples + raw_offset * c.bps, n - raw_offset, raw_offset, nf, out, samples, n);
    if (s != CUVHS_OK) {
      c.drain_copies();
      return s;
    }
    if (out->fields_out == before) {
      out->next_raw_offset = prev_next;
      break;
    }
    raw_offset = out->next_raw_offset;
  }
  if (!c.drain_copies()) return c.status;
  return CUVHS_OK;
}

long long cuvhs_json(const cuvhs_ctx* ctx, const cuvhs_output* out, char* dst, long long cap) {
  if (!ctx || !out) return -1;
  std::string s = cuvhs::tbc_json(ctx->c.fmt, out->fields, out->fields_out, out->dropout_line, out->dropout_startx,
                                  out->dropout_endx);
  if (dst && cap > 0) {
    const size_t n = std::min<size_t>((size_t)cap - 1, s.size());
    std::memcpy(dst, s.data(), n);
    dst[n] = 0;
  }
  return (long long)s.size();
}

void* cuvhs_stream(const cuvhs_ctx* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

void cuvhs_set_timing_mask(cuvhs_ctx* ctx, unsigned mask) {
  if (ctx) ctx->c.timing_mask = mask;
}

void cuvhs_set_timing(cuvhs_ctx* ctx, int on) {
  if (ctx) ctx->c.timing = on != 0;
}

int cuvhs_stage_count(void) { return cuvhs::kNumStages; }

const char* cuvhs_stage_name(int i) { return (i >= 0 && i < cuvhs::kNumStages) ? cuvhs::kStageNames[i] : ""; }

int cuvhs_stage_times(const cuvhs_ctx* ctx, double* ms, long long* launches, int cap) {
  if (!ctx) return 0;
  const int n = std::min(cap, (int)cuvhs::kNumStages);
  for (int i = 0; i < n; i++) {
    if (ms) ms[i] = ctx->c.stage_ms[i];
    if (launches) launches[i] = ctx->c.stage_launches[i];
  }
  return cuvhs::kNumStages;
}

int cuvhs_stage_timeline(const cuvhs_ctx* ctx, int* stage, double* start_ms, double* end_ms, int cap) {
  if (!ctx) return 0;
  const auto& t = ctx->c.timeline;
  const int n = std::min(cap, (int)t.size());
  for (int i = 0; i < n; i++) {
    if (stage) stage[i] = t[i].stage;
    if (start_ms) start_ms[i] = t[i].start;
    if (end_ms) end_ms[i] = t[i].end;
  }
  return (int)t.size();
}

void cuvhs_reset_stage_times(cuvhs_ctx* ctx) {
  if (!ctx) return;
  for (int i = 0; i < cuvhs::kNumStages; i++) {
    ctx->c.stage_ms[i] = 0.0;
    ctx->c.stage_launches[i] = 0;
  }
  ctx->c.launches = 0;
}

long long cuvhs_launch_count(const cuvhs_ctx* ctx) { return ctx ? ctx->c.launches : 0; }

long long cuvhs_debug_array(const cuvhs_ctx* ctx, const char* name, void* dst, long long cap) {
  if (!ctx || !name) return -1;
  const Context& c = ctx->c;
  const std::string s(name);
  if (s == "meta") return copy_out(c.dbg_meta, dst, cap);
  if (s == "vsync_candidates") return copy_out(c.dbg_vsync, dst, cap);
  if (s == "field_offsets") return copy_out(c.dbg_offs, dst, cap);
  if (s == "k2_pulse_count") return copy_out(c.dbg_k2c, dst, cap);
  if (s == "k2_pulse_starts") return copy_out(c.dbg_k2s, dst, cap);
  if (s == "k2_pulse_lengths") return copy_out(c.dbg_k2l, dst, cap);
  if (s == "k2b_pulse_count") return copy_out(c.dbg_k2bc, dst, cap);
  if (s == "k2b_pulse_starts") return copy_out(c.dbg_k2bs, dst, cap);
  if (s == "k2b_pulse_lengths") return copy_out(c.dbg_k2bl, dst, cap);
  if (s == "k2b_pulse_types") return copy_out(c.dbg_k2bt, dst, cap);
  if (s == "is_first") return copy_out(c.dbg_is_first, dst, cap);
  const size_t P = (size_t)c.last_fields;
  if (s == "do_count") return copy_ptr(c.hp_do_count, P, dst, cap);
  if (s == "do_lines") return copy_ptr(c.hp_do_lines, P * cuvhs::kMaxDropouts, dst, cap);
  if (s == "do_starts") return copy_ptr(c.hp_do_starts, P * cuvhs::kMaxDropouts, dst, cap);
  if (s == "do_ends") return copy_ptr(c.hp_do_ends, P * cuvhs::kMaxDropouts, dst, cap);
  if (s == "guard_positions") return copy_out(c.dbg_guard_pos, dst, cap);
  if (s == "guard_values") return copy_out(c.dbg_guard_vals, dst, cap);
  if (s == "linelocs_coarse") return copy_out(c.dbg_ll_coarse, dst, cap);
  if (s == "lineloc_clocks") return copy_out(c.dbg_clk_ll, dst, cap);
  if (s == "guard_clocks") return copy_out(c.dbg_clk_guard, dst, cap);
  if (s == "linelocs") return copy_out(c.dbg_ll, dst, cap);
  if (s == "demod") return copy_out(c.dbg_demod, dst, cap);
  if (s == "video") return copy_out(c.dbg_video, dst, cap);
  if (s == "sync") return copy_out(c.dbg_sync, dst, cap);
  if (s == "envelope") return copy_out(c.dbg_env, dst, cap);
  if (s == "chroma_prefilt") return copy_out(c.dbg_pre, dst, cap);
  return -1;
}

// ------------------------------------------------------------------ file path
// main + RawReader + TBCWriter + Pipeline::run (src/main.cpp:97-165,
// src/io/raw_reader.cpp:128-151, src/io/tbc_writer.cpp:10-175,
// src/pipeline/pipeline.cu:2626-2713).
cuvhs_status cuvhs_decode_file(const cuvhs_config* cfg, const char* in_path, const char* out_base, int overwrite) {
  if (!cfg || !in_path || !out_base) return CUVHS_ERR_INVALID_ARGUMENT;
  const std::string base(out_base);
  const std::string luma_path = base + ".tbc", chroma_path = base + "_chroma.tbc", json_path = base + ".tbc.json";
  if (!overwrite) {
    struct stat st;
    for (const std::string* p : {&luma_path, &chroma_path, &json_path}) {
      if (stat(p->c_str(), &st) == 0) {
        fprintf(stderr, "Output exists: %s (use --overwrite)\n", p->c_str());
        return CUVHS_ERR_EXISTS;
      }
    }
  }
  const bool is_stdin = std::strcmp(in_path, "-") == 0;
  int fd = is_stdin ? STDIN_FILENO : ::open(in_path, O_RDONLY);
  if (fd < 0) {
    perror(in_path);
    return CUVHS_ERR_IO;
  }
  struct stat st;
  bool streaming = is_stdin;
  size_t file_size = 0;
  if (!is_stdin) {
    if (fstat(fd, &st) < 0) {
      perror("fstat");
      ::close(fd);
      return CUVHS_ERR_IO;
    }
    if (S_ISFIFO(st.st_mode) || S_ISCHR(st.st_mode)) streaming = true;
    else file_size = (size_t)st.st_size / (cfg->input_format == 0 ? 1 : 2);  // samples
  }
  cuvhs_config c2 = *cfg;
  if (streaming) c2.stream_mode = 1;
  cuvhs_ctx* ctx = nullptr;
  cuvhs_status s = cuvhs_create(&c2, &ctx);
  if (s != CUVHS_OK) {
    if (!is_stdin) ::close(fd);
    return s;
  }
  Context& c = ctx->c;
  FILE* fl = fopen(luma_path.c_str(), "wb");
  FILE* fc = fl ? fopen(chroma_path.c_str(), "wb") : nullptr;
  if (!fl || !fc) {
    perror(!fl ? luma_path.c_str() : chroma_path.c_str());
    if (fl) fclose(fl);
    if (!is_stdin) ::close(fd);
    cuvhs_destroy(ctx);
    return CUVHS_ERR_IO;
  }
  const size_t spf = (size_t)c.fmt.samples_per_field, spp = (size_t)c.spp;
  const size_t F = (size_t)c.fmt.output_line_len * c.fmt.output_field_lines;
  const size_t bps = (size_t)c.bps;  // bytes per sample; offsets and counts below are in samples
  std::vector<uint16_t> luma((size_t)c.batch * F), chroma((size_t)c.batch * F);
  std::vector<int32_t> dl, ds, de;
  std::vector<cuvhs_field_info> all;
  std::vector<int32_t> all_dl, all_ds, all_de;
  std::vector<uint8_t> buf;
  // stream mode keeps the samples from buf_origin on, reading forward as needed
  uint64_t buf_origin = 0;
  bool eof = false;
  auto buffered = [&]() { return (uint64_t)(buf.size() / bps); };
  auto fill_stream = [&](uint64_t upto) {
    while (!eof && buf_origin + buffered() < upto) {
      const size_t want = (size_t)(upto - (buf_origin + buffered())) * bps;
      const size_t old = buf.size();
      buf.resize(old + want);
      size_t got = 0;
      while (got < want) {
        ssize_t r = ::read(fd, buf.data() + old + got, want - got);
        if (r > 0) got += (size_t)r;
        else if (r == 0) { eof = true; break; }
        else if (errno == EINTR) continue;
        else { eof = true; break; }
      }
      buf.resize(old + got);
    }
  };
  auto write_json = [&]() -> bool {
    const std::string text = cuvhs::tbc_json(c.fmt, all.data(), all.size(), all_dl.data(), all_ds.data(), all_de.data());
    const std::string tmp = json_path + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) {
      perror(tmp.c_str());
      return false;
    }
    fwrite(text.data(), 1, text.size(), f);
    fclose(f);
    if (rename(tmp.c_str(), json_path.c_str()) != 0) {
      perror("rename .tbc.json");
      return false;
    }
    return true;
  };
  uint64_t raw_offset = 0;
  s = CUVHS_OK;
  while (true) {
    int nf = c.batch;
    if (!streaming) {
      if (raw_offset >= file_size) break;
      const int remaining_fields = (int)((file_size - raw_offset) / spf);
      if (remaining_fields <= 0) break;
      nf = std::min(c.batch, remaining_fields);
    }
    const size_t want = (size_t)nf * spp;
    size_t n_avail = 0;
    const uint8_t* src = nullptr;
    if (!streaming) {
      const size_t n = std::min(want, file_size - (size_t)raw_offset) * bps;
      buf.resize(n);
      size_t got = 0;
      while (got < n) {
        ssize_t r = pread(fd, buf.data() + got, n - got, (off_t)(raw_offset * bps + got));
        if (r > 0) got += (size_t)r;
        else if (r < 0 && errno == EINTR) continue;
        else break;
      }
      n_avail = got / bps;
      src = buf.data();
    } else {
      if (raw_offset > buf_origin) {
        const size_t drop = std::min((size_t)(raw_offset - buf_origin), (size_t)buffered());
        buf.erase(buf.begin(), buf.begin() + drop * bps);
        buf_origin += drop;
      }
      fill_stream(raw_offset + want);
      n_avail = buf_origin + buffered() > raw_offset ? (size_t)(buf_origin + buffered() - raw_offset) : 0;
      src = buf.data() + (raw_offset - buf_origin) * bps;
    }
    if (n_avail < spf) break;
    cuvhs_output out;
    std::memset(&out, 0, sizeof(out));
    dl.assign((size_t)nf * cuvhs::kMaxDropouts, 0);
    ds.assign(dl.size(), 0);
    de.assign(dl.size(), 0);
    std::vector<cuvhs_field_info> fields(nf);
    out.luma = luma.data();
    out.chroma = chroma.data();
    out.fields = fields.data();
    out.dropout_line = dl.data();
    out.dropout_startx = ds.data();
    out.dropout_endx = de.data();
    out.max_fields = (size_t)nf;
    out.max_dropouts = dl.size();
    s = cuvhs_decode_chunk(ctx, src, n_avail, raw_offset, nf, &out);
    if (s != CUVHS_OK) {
      fprintf(stderr, "decode failed: %s\n", cuvhs_last_error(ctx));
      break;
    }
    if (out.fields_out == 0) break;
    if (fwrite(luma.data(), sizeof(uint16_t), out.fields_out * F, fl) != out.fields_out * F ||
        fwrite(chroma.data(), sizeof(uint16_t), out.fields_out * F, fc) != out.fields_out * F) {
      s = CUVHS_ERR_IO;
      break;
    }
    for (size_t i = 0; i < out.fields_out; i++) {
      cuvhs_field_info fi = fields[i];
      const int32_t o = fi.dropout_offset;
      fi.dropout_offset = (int32_t)all_dl.size();
      for (int d = 0; d < fi.dropout_count; d++) {
        all_dl.push_back(dl[o + d]);
        all_ds.push_back(ds[o + d]);
        all_de.push_back(de[o + d]);
      }
      all.push_back(fi);
    }
    raw_offset = out.next_raw_offset;
    if (!write_json()) {
      s = CUVHS_ERR_IO;
      break;
    }
  }
  fflush(fl);
  fflush(fc);
  fclose(fl);
  fclose(fc);
  if (s == CUVHS_OK && !write_json()) s = CUVHS_ERR_IO;
  if (s == CUVHS_OK) fprintf(stderr, "\nWrote %s (%d fields)\n", json_path.c_str(), (int)all.size());
  if (!is_stdin) ::close(fd);
  cuvhs_destroy(ctx);
  return s;
}

}  // extern "C"
