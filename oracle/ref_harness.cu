// Test harness around the UNMODIFIED reference decoder (hunterschuler/cuVHS).
//
// This file is test infrastructure: it is compiled by oracle/Makefile together
// with the reference's own sources, read in place from the reference tree, into
// oracle/_ref/ref_harness (never into the product).  It runs the reference's
// Pipeline chunk loop exactly as Pipeline::run does (src/pipeline/pipeline.cu:2626-2713)
// and, after every chunk, copies out the intermediates the CLI never writes:
// VSYNC candidates, raw and validated sync pulses, coarse and refined line
// locations, field parity, dropouts, chroma state and a few tiles of the FP64
// demod / sync / envelope / chroma-prefiltered signals.  With --time it runs the
// same loop without dumps and prints the decode throughput as one JSON line.
//
// Pipeline's members are private; the harness reaches them by compiling the
// reference header with `private` defined as `public` (member order, and hence
// layout, is unchanged).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <strings.h>
#include <vector>

#include <cuda_runtime.h>
#include <cufft.h>

#define private public
#include "pipeline/pipeline.h"
#undef private
#include "pipeline/sync_pulses.h"
#include "pipeline/dropout_detect.h"

namespace {

struct Dumper {
  std::string dir;
  FILE* manifest = nullptr;
  bool open(const std::string& d) {
    dir = d;
    std::string cmd = "mkdir -p '" + d + "'";
    if (system(cmd.c_str()) != 0) return false;
    manifest = fopen((dir + "/manifest.txt").c_str(), "w");
    return manifest != nullptr;
  }
  void write(const std::string& name, const char* dtype, const void* data, size_t count, size_t elem) {
    std::string path = dir + "/" + name + ".bin";
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return;
    if (count) fwrite(data, elem, count, f);
    fclose(f);
    fprintf(manifest, "%s %s %zu\n", name.c_str(), dtype, count);
    fflush(manifest);
  }
  template <typename T>
  void dev(const std::string& name, const char* dtype, const void* dptr, size_t count) {
    std::vector<T> h(count);
    if (count) cudaMemcpy(h.data(), dptr, count * sizeof(T), cudaMemcpyDeviceToHost);
    write(name, dtype, h.data(), count, sizeof(T));
  }
  void dev_f64_as_f32(const std::string& name, const void* dptr, size_t count) {
    std::vector<double> h(count);
    if (count) cudaMemcpy(h.data(), dptr, count * sizeof(double), cudaMemcpyDeviceToHost);
    std::vector<float> g(count);
    for (size_t i = 0; i < count; i++) g[i] = (float)h[i];
    write(name, "f32", g.data(), count, sizeof(float));
  }
  void dev_f64(const std::string& name, const void* dptr, size_t count) {
    dev<double>(name, "f64", dptr, count);
  }
};

}  // namespace

int main(int argc, char** argv) {
  double mhz = 28.0;
  bool pal = false;
  long long reserve_mb = 0;
  std::string in, out, dump_dir;
  bool time_only = false;
  int dump_tiles = 2;
  int pos = 0;
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "-f") && i + 1 < argc) mhz = atof(argv[++i]);
    else if (!strcmp(argv[i], "--system") && i + 1 < argc) pal = !strcasecmp(argv[++i], "PAL");
    else if (!strcmp(argv[i], "--reserve-mb") && i + 1 < argc) reserve_mb = atoll(argv[++i]);
    else if (!strcmp(argv[i], "--dump") && i + 1 < argc) dump_dir = argv[++i];
    else if (!strcmp(argv[i], "--dump-tiles") && i + 1 < argc) dump_tiles = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--time")) time_only = true;
    else if (pos == 0) { in = argv[i]; pos++; }
    else if (pos == 1) { out = argv[i]; pos++; }
  }
  if (pos < 2) {
    fprintf(stderr, "usage: ref_harness [-f MHz] [--system NTSC|PAL] [--reserve-mb N] [--dump DIR] [--dump-tiles N] "
                    "[--time] in.u8 out_base\n");
    return 2;
  }

  GPUDevice gpu;
  if (!gpu.init(0)) return 1;
  VideoFormat fmt(pal ? VideoSystem::PAL : VideoSystem::NTSC, mhz);
  RawReader reader;
  if (!reader.open(in, InputFormat::U8)) return 1;
  TBCWriter writer;
  if (!writer.open(out, fmt, true)) return 1;
  Pipeline pl(gpu, fmt, reader, writer);
  // --reserve-mb: device memory held while the reference sizes its buffers
  // (from the free memory) and released afterwards, for kernels that need
  // local memory beyond what its default allocation leaves
  void* reserve = nullptr;
  if (reserve_mb > 0 && cudaMalloc(&reserve, (size_t)reserve_mb << 20) != cudaSuccess) return 1;
  if (!pl.allocate_buffers()) return 1;
  if (reserve) cudaFree(reserve);

  Dumper dump;
  bool dumping = !dump_dir.empty() && !time_only;
  if (dumping && !dump.open(dump_dir)) return 1;

  const size_t spf = fmt.samples_per_field;
  const size_t spp = spf + 20 * (size_t)fmt.samples_per_line;
  size_t total_samples = reader.total_samples();
  size_t raw_offset = 0;
  int total_fields = 0;
  int chunk = 0;
  cudaDeviceSynchronize();
  auto t0 = std::chrono::steady_clock::now();
  while (true) {
    size_t remaining_samples = total_samples - raw_offset;
    int remaining_fields = (int)(remaining_samples / fmt.samples_per_field);
    if (remaining_fields <= 0) break;
    int fields_this_chunk = std::min(pl.batch_size, remaining_fields);
    size_t next_raw_offset = 0;
    int processed = pl.process_chunk(raw_offset, fields_this_chunk, next_raw_offset);
    {
      const cudaError_t e = cudaGetLastError();  // the reference does not check its launches
      if (e != cudaSuccess) fprintf(stderr, "ref_harness: CUDA error after chunk %d: %s\n", chunk, cudaGetErrorString(e));
    }
    if (processed == 0) break;
    if (dumping) {
      cudaDeviceSynchronize();
      char pre[64];
      snprintf(pre, sizeof(pre), "c%d_", chunk);
      std::string p(pre);
      size_t n_read = std::min((size_t)fields_this_chunk * spp, total_samples - raw_offset);
      int tiles = (int)std::min(n_read / spf, (size_t)fields_this_chunk);
      long long meta[8] = {(long long)raw_offset, (long long)processed, (long long)spp,
                           (long long)tiles, (long long)fields_this_chunk,
                           (long long)next_raw_offset, (long long)pl.batch_size, 0};
      dump.write(p + "meta", "i64", meta, 8, sizeof(long long));
      int ncand = 0;
      cudaMemcpy(&ncand, pl.d_candidate_count, sizeof(int), cudaMemcpyDeviceToHost);
      int nstored = std::min(ncand, tiles * 20);
      dump.dev<int>(p + "vsync_candidates", "i32", pl.d_candidate_indices, (size_t)std::max(0, nstored));
      dump.dev<int>(p + "k2b_pulse_count", "i32", pl.d_pulse_count, processed);
      dump.dev<int>(p + "k2b_pulse_starts", "i32", pl.d_pulse_starts, (size_t)processed * MAX_PULSES);
      dump.dev<int>(p + "k2b_pulse_lengths", "i32", pl.d_pulse_lengths, (size_t)processed * MAX_PULSES);
      dump.dev<int>(p + "k2b_pulse_types", "i32", pl.d_pulse_types, (size_t)processed * MAX_PULSES);
      dump.dev_f64(p + "linelocs_coarse", pl.d_linelocs_coarse, (size_t)processed * fmt.lines_per_frame);
      dump.dev_f64(p + "linelocs", pl.d_linelocs, (size_t)processed * fmt.lines_per_frame);
      dump.dev<int>(p + "is_first", "i32", pl.d_is_first_field, processed);
      dump.dev<int>(p + "do_count", "i32", pl.d_do_count, processed);
      dump.dev<int>(p + "do_lines", "i32", pl.d_do_lines, (size_t)processed * MAX_DROPOUTS_PER_FIELD);
      dump.dev<int>(p + "do_starts", "i32", pl.d_do_starts, (size_t)processed * MAX_DROPOUTS_PER_FIELD);
      dump.dev<int>(p + "do_ends", "i32", pl.d_do_ends, (size_t)processed * MAX_DROPOUTS_PER_FIELD);
      double cs[4] = {pl.chroma_state.valid ? 1.0 : 0.0, (double)pl.chroma_state.current_track,
                      pl.chroma_state.good_metric_threshold, (double)pl.chroma_state.cycle_start};
      dump.write(p + "chroma_state", "f64", cs, 4, sizeof(double));
      double k2b[5] = {(double)pl.k2b_prev_first_field, (double)pl.k2b_prev_progressive_field,
                       (double)pl.k2b_prev_first_hsync_readloc, pl.k2b_prev_first_hsync_loc,
                       pl.k2b_prev_first_hsync_diff};
      dump.write(p + "k2b_state", "f64", k2b, 5, sizeof(double));
      // Field offsets of this chunk, recovered from the writer's fileLoc entries.
      std::vector<size_t> offs(processed);
      for (int i = 0; i < processed; i++)
        offs[i] = writer.field_meta[(size_t)total_fields + i].file_loc - raw_offset;
      std::vector<long long> offs_ll(offs.begin(), offs.end());
      dump.write(p + "field_offsets", "i64", offs_ll.data(), offs_ll.size(), sizeof(long long));
      // Re-run the reference's K2 pulse finder on the same offsets to recover
      // its raw output (K2b overwrote the device arrays with validated pulses).
      size_t* d_offs = nullptr;
      cudaMalloc(&d_offs, processed * sizeof(size_t));
      cudaMemcpy(d_offs, offs.data(), processed * sizeof(size_t), cudaMemcpyHostToDevice);
      int* d_ps = nullptr; int* d_pl = nullptr; int* d_pc = nullptr;
      cudaMalloc(&d_ps, (size_t)processed * MAX_PULSES * sizeof(int));
      cudaMalloc(&d_pl, (size_t)processed * MAX_PULSES * sizeof(int));
      cudaMalloc(&d_pc, processed * sizeof(int));
      if (d_offs && d_ps && d_pl && d_pc) {
        sync_pulses(static_cast<double*>(pl.d_demod_05), d_ps, d_pl, d_pc, d_offs, processed, spp, fmt);
        cudaDeviceSynchronize();
        dump.dev<int>(p + "k2_pulse_count", "i32", d_pc, processed);
        dump.dev<int>(p + "k2_pulse_starts", "i32", d_ps, (size_t)processed * MAX_PULSES);
        dump.dev<int>(p + "k2_pulse_lengths", "i32", d_pl, (size_t)processed * MAX_PULSES);
      }
      if (d_offs) cudaFree(d_offs);
      if (d_ps) cudaFree(d_ps);
      if (d_pl) cudaFree(d_pl);
      if (d_pc) cudaFree(d_pc);
      size_t nt = (size_t)std::min(dump_tiles, tiles) * spp;
      dump.dev_f64_as_f32(p + "demod05_f32", pl.d_demod_05, nt);
      dump.dev_f64_as_f32(p + "envelope_f32", pl.d_envelope, nt);
      dump.dev_f64_as_f32(p + "chroma_prefilt_f32", pl.d_demod, nt);
      // d_demod now holds the chroma pre-filtered raw; recompute the video demod
      // (deterministic cuFFT plans) to dump it too.
      fm_demod(pl.demod_state, static_cast<double*>(pl.d_raw), static_cast<double*>(pl.d_demod),
               static_cast<double*>(pl.d_demod_05), static_cast<double*>(pl.d_envelope), tiles, spp, fmt);
      cudaDeviceSynchronize();
      dump.dev_f64_as_f32(p + "demod_f32", pl.d_demod, nt);
      // Full-precision sync demod near the first few lines of each field, for
      // threshold-exactness checks: 40 lines from each field offset.
      std::vector<double> win;
      size_t wl = 40 * (size_t)fmt.samples_per_line;
      for (int i = 0; i < processed && i < 4; i++) {
        std::vector<double> h(wl);
        size_t o = offs[i];
        if (o + wl <= (size_t)tiles * spp) {
          cudaMemcpy(h.data(), static_cast<double*>(pl.d_demod_05) + o, wl * sizeof(double), cudaMemcpyDeviceToHost);
          win.insert(win.end(), h.begin(), h.end());
        }
      }
      dump.write(p + "demod05_head_f64", "f64", win.data(), win.size(), sizeof(double));
    }
    raw_offset = next_raw_offset;
    total_fields += processed;
    writer.write_json();
    chunk++;
  }
  cudaDeviceSynchronize();
  auto t1 = std::chrono::steady_clock::now();
  double secs = std::chrono::duration<double>(t1 - t0).count();
  writer.finalize();
  printf("{\"fields\": %d, \"seconds\": %.6f, \"fields_per_s\": %.3f, \"batch_size\": %d, \"chunks\": %d}\n",
         total_fields, secs, total_fields / secs, pl.batch_size, chunk);
  return 0;
}
