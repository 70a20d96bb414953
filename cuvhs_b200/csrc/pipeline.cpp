// Chunk decode orchestration (host side of libcuvhs).
//
// Mirrors the reference's per-chunk flow (src/pipeline/pipeline.cu:1525-2624):
// demod the chunk's tiles, find VSYNC candidates and cluster them into field
// windows, find each window's sync pulses, derive line locations, refine them,
// resample luma and chroma, detect dropouts, then assign field parity.  The
// sample-rate work runs in the kernels; the per-field pulse logic (a few
// hundred pulses per field) and the chroma track decisions run here on the
// host, exactly as the reference does them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cuvhs.h"
#include "cuvhs_internal.h"
#include "pipeline.h"

namespace cuvhs {

namespace {

template <typename T>
T* dalloc(size_t n, std::string& err, bool& ok) {
  if (!ok) return nullptr;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) {
    ok = false;
    err = std::string("cudaMalloc failed: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return nullptr;
  }
  return static_cast<T*>(p);
}

template <typename T>
void upload(T* d, const std::vector<T>& h, cudaStream_t st) {
  if (!h.empty()) cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

}  // namespace

const int kPhaseCycle[8] = {3, 2, 1, 4, 3, 2, 1, 4};

// NTSC field phase table keyed by (first field, burst quadrant), no phase
// delta known (src/pipeline/chroma_decode.cu:337-377: the decoder always looks
// up the first field of a run with delta -1).
int phase_id_for(int is_first, int quadrant) {
  static const int first_q[4] = {3, 1, 3, 1};   // quadrant -> id for first fields
  static const int second_q[4] = {4, 2, 4, 2};  // quadrant -> id for second fields
  if (quadrant < 0 || quadrant > 3) return 1;
  return is_first ? first_q[quadrant] : second_q[quadrant];
}

const char* const kStageNames[kNumStages] = {"k1a_demod",      "k1b_video_sync", "sync_edges",
                                             "hsync_refine",   "luma_resample",  "chroma_prefilter",
                                             "chroma_lines",   "burst_metric",   "dropouts",
                                             "sync_guard",     "field_windows",  "line_locations",
                                             "host_windows_wait", "host_chroma_wait", "host_final_wait"};

double Context::host_clock() const {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

Context::~Context() { release(); }

cudaEvent_t Context::next_event() {
  if (pool_used == event_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    event_pool.push_back(e);
  }
  return event_pool[pool_used++];
}

void Context::begin_stage_on(int stage, cudaEvent_t& a, cudaStream_t st) {
  a = nullptr;
  if (!timing || !((timing_mask >> stage) & 1u)) return;
  a = next_event();
  cudaEventRecord(a, st);
  if (t0_pending) {
    ev_t0 = a;
    t0_pending = false;
    timeline.clear();
  }
}

void Context::end_stage_on(int stage, cudaEvent_t a, cudaStream_t st, int kernels) {
  stage_launches[stage] += kernels;
  launches += kernels;
  if (!timing || !a) return;
  cudaEvent_t b = next_event();
  cudaEventRecord(b, st);
  marks.push_back({stage, a, b});
}

// Called after a stream synchronisation: every recorded pair has completed.
void Context::collect_stage_times() {
  for (const Mark& m : marks) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, m.a, m.b) == cudaSuccess) stage_ms[m.stage] += ms;
    float s0 = 0.0f;
    if (ev_t0 && cudaEventElapsedTime(&s0, ev_t0, m.a) == cudaSuccess) timeline.push_back({m.stage, s0, s0 + ms});
  }
  marks.clear();
  // events stay recorded until the chunk's timeline is complete
  if (!ev_t0) pool_used = 0;
}

void Context::release() {
  if (device >= 0) cudaSetDevice(device);
  for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
  event_pool.clear();
  marks.clear();
  pool_used = 0;
  for (void* p : allocations) cudaFree(p);
  allocations.clear();
  for (void* p : host_allocations) cudaFreeHost(p);
  host_allocations.clear();
  hp_round_burst = nullptr;
  if (ev_host) cudaEventDestroy(ev_host);
  ev_host = nullptr;
  for (cudaEvent_t& e : ev_piece) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  if (ev_luma) cudaEventDestroy(ev_luma);
  ev_luma = nullptr;
  if (ev_edges) cudaEventDestroy(ev_edges);
  ev_edges = nullptr;
  for (cudaEvent_t* e : {&ev_prefetch, &ev_small, &ev_chroma, &ev_out_done[0], &ev_out_done[1]}) {
    if (*e) cudaEventDestroy(*e);
    *e = nullptr;
  }
  if (hstream) cudaStreamDestroy(hstream);
  hstream = nullptr;
  if (pstream) cudaStreamDestroy(pstream);
  pstream = nullptr;
  for (cudaEvent_t* e : {&ev_ll, &ev_win, &ev_winhost, &ev_k1b, &ev_pre, &ev_guard, &ev_hs, &ev_trial, &ev_trialh, &ev_cpass}) {
    if (*e) cudaEventDestroy(*e);
    *e = nullptr;
  }
  if (gstream) cudaStreamDestroy(gstream);
  gstream = nullptr;
  if (lstream) cudaStreamDestroy(lstream);
  lstream = nullptr;
  pf = Prefetch();
  if (xstream) cudaStreamDestroy(xstream);
  xstream = nullptr;
  if (ostream) cudaStreamDestroy(ostream);
  ostream = nullptr;
  if (stream) cudaStreamDestroy(stream);
  stream = nullptr;
}

// Device and page-locked host buffers for `batch` fields.
bool Context::alloc_buffers() {
  bool ok = true;
  const size_t S = (size_t)batch * spp;
  auto A = [&](auto* tag, size_t n) {
    using T = std::remove_pointer_t<decltype(tag)>;
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    if (ok && dev_limit > 0 && dev_used + bytes > dev_limit) {
      ok = false;
      err = "device memory limit reached";
    }
    T* p = dalloc<T>(n, err, ok);
    if (p) {
      allocations.push_back(p);
      dev_used += bytes;
    }
    return p;
  };
  env_blocks = (spp + des.a_out - 1) / des.a_out;
  d_raw_set[0] = A((uint8_t*)nullptr, S * bps + 64);
  d_raw_set[1] = A((uint8_t*)nullptr, S * bps + 64);
  d_dc = A((float*)nullptr, 1);
  d_dcsum = A((unsigned long long*)nullptr, 1);
  d_raw = d_raw_set[0];
  d_dem = A((float*)nullptr, S);
  d_env = A((float*)nullptr, S);
  d_video = A((float*)nullptr, S);
  d_sync = A((float*)nullptr, S);
  d_env_part = A((double*)nullptr, (size_t)batch * env_blocks);
  edge_cap = (int)std::min<size_t>(S / 4 + 4096, (size_t)INT_MAX / 2);
  const size_t edge_alloc = std::max((size_t)edge_cap, (size_t)batch * kEdgesPerSlot(spp));
  d_fall = A((unsigned*)nullptr, edge_alloc);
  d_rise = A((unsigned*)nullptr, edge_alloc);
  d_counts = A((int*)nullptr, 4 * kMaxPortions);
  d_edge_blk = A((int2*)nullptr, std::max((size_t)edge_blocks((long long)batch * spp) + 1,
                                          (size_t)batch * kEdgeBlocksPerSlot(spp)));
  d_edge_mask = A((unsigned*)nullptr, edge_mask_words((long long)batch * spp));
  d_ll = A((double*)nullptr, (size_t)batch * fmt.lines_per_frame);
  const size_t F = (size_t)fmt.output_line_len * fmt.output_field_lines;
  for (int k = 0; k < 2; k++) {
    d_luma_set[k] = A((uint16_t*)nullptr, (size_t)batch * F);
    d_chroma_set[k] = A((uint16_t*)nullptr, (size_t)batch * F);
  }
  d_luma = d_luma_set[0];
  d_chroma = d_chroma_set[0];
  d_burst = A((float*)nullptr, (size_t)batch * fmt.output_field_lines * fmt.burst_len);
  d_track = A((int*)nullptr, batch);
  d_trial = A((int*)nullptr, 2);
  d_burst_trial = A((float*)nullptr, (size_t)2 * fmt.output_field_lines * fmt.burst_len);
  d_pick = A((int*)nullptr, 1);
  d_do_count = A((int*)nullptr, batch);
  d_do_lines = A((int*)nullptr, (size_t)batch * kMaxDropouts);
  d_do_starts = A((int*)nullptr, (size_t)batch * kMaxDropouts);
  d_do_ends = A((int*)nullptr, (size_t)batch * kMaxDropouts);
  d_do_cls = A((unsigned char*)nullptr, (size_t)batch * dropout_class_bytes_per_field(spp));
  d_ga = A((float2*)nullptr, des.ga.size());
  d_gb = A((float2*)nullptr, des.gb.size());
  d_gc = A((float*)nullptr, des.gc.size());
  d_twa = A((float2*)nullptr, des.tw_a.size());
  d_twb = A((float2*)nullptr, des.tw_b.size());
  d_twc = A((float2*)nullptr, des.tw_c.size());
  d_twl = A((float2*)nullptr, des.tw_line.size());
  d_twa_inv = A((float2*)nullptr, des.tw_a.size());
  d_twb_inv = A((float2*)nullptr, des.tw_b.size());
  d_twc_inv = A((float2*)nullptr, des.tw_c.size());
  d_twl_inv = A((float2*)nullptr, des.tw_line.size());
  d_win = A((WindowInfo*)nullptr, kMaxPortions);
  d_offs = A((long long*)nullptr, (size_t)batch + 1);
  d_cand = A((int*)nullptr, edge_alloc);
  d_ps = A((int*)nullptr, (size_t)batch * kMaxPulses);
  d_pl = A((int*)nullptr, (size_t)batch * kMaxPulses);
  d_pn = A((int*)nullptr, batch);
  d_vs = A((int*)nullptr, (size_t)batch * kMaxValid);
  d_vl = A((int*)nullptr, (size_t)batch * kMaxValid);
  d_vt = A((unsigned char*)nullptr, (size_t)batch * kMaxValid);
  d_vd = A((double*)nullptr, (size_t)batch * kMaxValid);
  d_vn = A((int*)nullptr, batch);
  d_prep = A((FieldPrep*)nullptr, batch);
  d_lls = A((LineLocState*)nullptr, kMaxPortions);
  d_lls_save = A((LineLocState*)nullptr, kMaxPortions);
  d_pulse_bits = A((unsigned*)nullptr, std::max(pulse_bit_words((long long)batch * spp),
                                                (size_t)batch * kBitWordsPerSlot(spp)));
  d_guard_flips = A((int*)nullptr, kMaxPortions);
  d_is_first = A((int*)nullptr, batch);
  d_dbg_vs = A((int*)nullptr, (size_t)batch * kMaxPulses);
  d_dbg_vl = A((int*)nullptr, (size_t)batch * kMaxPulses);
  d_dbg_vt = A((int*)nullptr, (size_t)batch * kMaxPulses);
  d_dbg_vn = A((int*)nullptr, batch);
  d_dbg_clk_ll = A((long long*)nullptr, (size_t)batch * kPhaseSlots);
  d_dbg_clk_guard = A((long long*)nullptr, (size_t)kGuardClockSamples * kPhaseSlots);
  d_col_frac = A((double*)nullptr, (size_t)fmt.output_line_len);
  d_guard_g = A((double2*)nullptr, (size_t)Design::kGuardN);
  d_guard_tw = A((double2*)nullptr, (size_t)Design::kGuardN);
  d_hs64 = A((double*)nullptr, des.hs64.size());
  const size_t guard_alloc = std::max((size_t)kGuardCap, (size_t)batch * kGuardPerSlot);
  d_guard_list = A((unsigned*)nullptr, guard_alloc);
  d_guard_count = A((int*)nullptr, kMaxPortions);
  d_guard_vals = A((double*)nullptr, guard_alloc);
  if (ok && !guard_supported(des.ga64_half, des.hs64_half)) {
    err = "sync guard support too long";
    ok = false;
  }
  if (!ok) return false;
  // pinned host staging for the per-chunk round trips
  auto H = [&](auto* tag, size_t n) {
    using T = std::remove_pointer_t<decltype(tag)>;
    void* p = nullptr;
    if (!ok) return (T*)nullptr;
    if (cudaHostAlloc(&p, std::max<size_t>(n, 1) * sizeof(T), cudaHostAllocDefault) != cudaSuccess) {
      ok = false;
      err = "cudaHostAlloc failed";
      cudaGetLastError();
      return (T*)nullptr;
    }
    host_allocations.push_back(p);
    return static_cast<T*>(p);
  };
  hp_counts = H((int*)nullptr, 4);
  hp_win = H((WindowInfo*)nullptr, kMaxPortions);
  hp_lls = H((LineLocState*)nullptr, kMaxPortions);
  hp_offs = H((long long*)nullptr, (size_t)batch + 1);
  hp_is_first = H((int*)nullptr, batch);
  hp_guard = H((int*)nullptr, 2 * kMaxPortions);
  hp_track = H((int*)nullptr, batch);
  hp_trial = H((int*)nullptr, 2);
  hp_pick = H((int*)nullptr, 1);
  hp_burst = H((float*)nullptr, (size_t)2 * fmt.output_field_lines * fmt.burst_len);
  {
    void* p = nullptr;
    if (cudaHostAlloc(&p, std::max(batch, 1) * sizeof(double), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&dp_metric, p, 0) != cudaSuccess) {
      if (p) cudaFreeHost(p);
      err = "cudaHostAlloc (mapped) failed";
      ok = false;
    } else {
      host_allocations.push_back(p);
      hp_metric = static_cast<double*>(p);
    }
  }
  hp_do_count = H((int*)nullptr, batch);
  hp_do_lines = H((int*)nullptr, (size_t)batch * kMaxDropouts);
  hp_do_starts = H((int*)nullptr, (size_t)batch * kMaxDropouts);
  hp_do_ends = H((int*)nullptr, (size_t)batch * kMaxDropouts);
  if (!ok) return false;
  return true;
}

void Context::free_buffers() {
  if (device >= 0) cudaSetDevice(device);
  for (void* p : allocations) cudaFree(p);
  allocations.clear();
  for (void* p : host_allocations) cudaFreeHost(p);
  host_allocations.clear();
  hp_round_burst = nullptr;
  dev_used = 0;
  cudaGetLastError();
}

bool Context::init(const cuvhs_config& c) {
  cfg = c;
  if (!(c.sample_rate_mhz >= 8.0 && c.sample_rate_mhz <= 100.0)) {
    err = "sample rate out of range (8-100 MHz)";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  if (c.system != kNtsc && c.system != kPal) {
    err = "system must be 0 (NTSC) or 1 (PAL)";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  if (!(c.guard_band_hz >= 0.0 && c.guard_band_hz <= 1.0e6)) {
    err = "guard_band_hz must be in [0, 1e6]";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  if (c.input_format < 0 || c.input_format > 2) {
    err = "input_format must be 0 (u8), 1 (s16) or 2 (u16)";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    err = "no CUDA device";
    status = CUVHS_ERR_CUDA;
    return false;
  }
  device = c.device;
  if (device < 0) {
    size_t best = 0;
    for (int i = 0; i < ndev; i++) {
      cudaDeviceProp p;
      cudaGetDeviceProperties(&p, i);
      if (p.totalGlobalMem > best) {
        best = p.totalGlobalMem;
        device = i;
      }
    }
  }
  if (device >= ndev) {
    err = "GPU " + std::to_string(device) + " not found";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  cudaSetDevice(device);
  in_fmt = c.input_format;
  bps = in_fmt == 0 ? 1 : 2;
  dc_correct = c.dc_correct != 0;
  fmt.init(c.sample_rate_mhz, c.system);
  des.build_cached(fmt);
  spp = fmt.spp;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t field_px = (size_t)fmt.output_line_len * fmt.output_field_lines;
  const size_t per_field = (size_t)spp * (2 * bps + 4 * 5) + (size_t)spp / 4 + field_px * 8 +
                           (size_t)fmt.output_field_lines * kMaxBurstLen * 4 + 65536 + dropout_class_bytes_per_field(spp) +
                           (size_t)kMaxValid * 17 + (size_t)kMaxPulses * 20 + sizeof(FieldPrep);
  int b = c.batch_fields;
  if (b <= 0) {
    b = (int)std::min<size_t>((size_t)(free_b * 0.5) / per_field, 2048);
    if (b < 1) b = 1;
  }
  if (c.stream_mode && b > 64) b = 64;
  // 32-bit sample indices inside a chunk
  const int cap_fields = (int)std::min<long long>(INT_MAX / 2 / (long long)spp, 1 << 20);
  if (b > cap_fields) b = cap_fields;
  batch = b;
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&xstream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ostream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&hstream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithPriority(&lstream, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
      cudaStreamCreateWithPriority(&pstream, cudaStreamNonBlocking, (prio_low + prio_high) / 2) != cudaSuccess ||
      cudaStreamCreateWithPriority(&gstream, cudaStreamNonBlocking, prio_high) != cudaSuccess) {
    err = "cudaStreamCreate failed";
    status = CUVHS_ERR_CUDA;
    return false;
  }
  // Buffers for `batch` fields; a sized-from-free-memory batch backs off by
  // halves when an allocation fails (the reference retries at smaller VRAM
  // fractions, src/pipeline/pipeline.cu:1384-1475).  An explicit batch_fields
  // is kept or the context fails, since the batch sets the chunking.
  dev_limit = (size_t)std::max(0.0, c.device_memory_limit_mb) * (1u << 20);
  for (;;) {
    batch = b;
    if (alloc_buffers()) break;
    free_buffers();
    if (c.batch_fields > 0 || b <= 1) {
      status = CUVHS_ERR_OUT_OF_MEMORY;
      release();
      return false;
    }
    b = std::max(1, b / 2);
  }
  hp_trial[0] = 0;
  hp_trial[1] = 1;
  if (cudaMemcpy(d_trial, hp_trial, 2 * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
    err = "trial track upload failed";
    status = CUVHS_ERR_CUDA;
    release();
    return false;
  }
  bool ev_ok = cudaEventCreateWithFlags(&ev_host, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_luma, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_edges, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_ll, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_win, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_winhost, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_k1b, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_pre, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_hs, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_trial, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_trialh, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_cpass, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev_guard, cudaEventDisableTiming) == cudaSuccess;
  for (cudaEvent_t* e : {&ev_prefetch, &ev_small, &ev_chroma, &ev_out_done[0], &ev_out_done[1]})
    ev_ok = ev_ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
  for (cudaEvent_t& e : ev_piece) ev_ok = ev_ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
  if (!ev_ok) {
    err = "cudaEventCreate failed";
    status = CUVHS_ERR_CUDA;
    return false;
  }
  upload(d_ga, des.ga, stream);
  upload(d_gb, des.gb, stream);
  upload(d_gc, des.gc, stream);
  upload(d_twa, des.tw_a, stream);
  upload(d_twb, des.tw_b, stream);
  upload(d_twc, des.tw_c, stream);
  upload(d_twl, des.tw_line, stream);
  upload(d_twa_inv, des.tw_a, stream);
  upload(d_twb_inv, des.tw_b, stream);
  upload(d_twc_inv, des.tw_c, stream);
  upload(d_twl_inv, des.tw_line, stream);
  cudaMemcpyAsync(d_guard_g, des.guard_g.data(), des.guard_g.size() * sizeof(double), cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(d_guard_tw, des.guard_tw.data(), des.guard_tw.size() * sizeof(double), cudaMemcpyHostToDevice,
                  stream);
  upload(d_hs64, des.hs64, stream);
  cudaMemsetAsync(d_guard_count, 0, sizeof(int), stream);
  {
    const LineLocState fresh;
    cudaMemcpy(d_lls, &fresh, sizeof(fresh), cudaMemcpyHostToDevice);
  }
  std::vector<double> col_frac(fmt.output_line_len);
  for (int c = 0; c < fmt.output_line_len; c++) col_frac[c] = (double)c / (double)fmt.output_line_len;
  upload(d_col_frac, col_frac, stream);
  if (cudaStreamSynchronize(stream) != cudaSuccess) {
    err = std::string("upload failed: ") + cudaGetErrorString(cudaGetLastError());
    status = CUVHS_ERR_CUDA;
    return false;
  }
  return true;
}

bool Context::check_cuda(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string(where) + ": " + cudaGetErrorString(e);
    status = CUVHS_ERR_CUDA;
    return false;
  }
  return true;
}

bool Context::sync(const char* where) {
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(xstream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ostream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(hstream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lstream);
  if (e != cudaSuccess) {
    err = std::string(where) + ": " + cudaGetErrorString(e);
    status = CUVHS_ERR_CUDA;
    return false;
  }
  collect_stage_times();
  return check_cuda(where);
}

// Wait for the work recorded before ev_host (the host reads results it
// copied); later work on the stream keeps running.
bool Context::drain_copies() {
  cudaError_t e = cudaStreamSynchronize(xstream);
  const cudaError_t e0 = cudaStreamSynchronize(ostream);
  if (e == cudaSuccess) e = e0;
  const cudaError_t e2 = cudaStreamSynchronize(hstream);
  pf.valid = false;
  rpf.valid = false;
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) {
    err = std::string("output copies: ") + cudaGetErrorString(e);
    status = CUVHS_ERR_CUDA;
    return false;
  }
  return true;
}

bool Context::wait_host_event(const char* where) {
  cudaError_t e = cudaEventSynchronize(ev_host);
  if (e != cudaSuccess) {
    err = std::string(where) + ": " + cudaGetErrorString(e);
    status = CUVHS_ERR_CUDA;
    return false;
  }
  return check_cuda(where);
}

void Context::reset_state() {
  if (d_lls) write_lls(LineLocState());
  chroma_valid = false;
  chroma_track = 0;
  chroma_threshold = 0.0;
  chroma_cycle_start = 0;
  last_parity = true;
}

// Host burst-cancellation metric over one field's burst windows (lines 16..245
// in pairs), as the track detector measures it (chroma_decode.cu:383-411).
double host_burst_metric(const float* b, int H, int bl) {
  const int skip = 16;
  double total = 0.0;
  int count = 0;
  for (int line = skip; line < H - skip - 1; line += 2) {
    const float* x = b + (size_t)line * bl;
    const float* y = x + bl;
    double s = 0.0;
    for (int i = 0; i < bl; i++) s += std::fabs((double)x[i] + (double)y[i]);
    total += s / bl;
    count++;
  }
  return count > 0 ? total / count : 1e9;
}

// Burst phase in degrees by I/Q product detection over lines 16..246
// (chroma_decode.cu:415-450).
double host_burst_phase(const float* b, int H, const Format& fmt) {
  const int skip = 16;
  const double PI = 3.14159265358979323846;
  double It = 0.0, Qt = 0.0;
  for (int line = skip; line < H - skip; line++) {
    const float* x = b + (size_t)line * fmt.burst_len;
    double I = 0.0, Q = 0.0;
    for (int i = 0; i < fmt.burst_len; i++) {
      const double v = x[i];
      const double t = 2.0 * PI * fmt.fsc / fmt.output_rate * (double)(fmt.burst_start + i);
      I += v * std::cos(t);
      Q += v * std::sin(t);
    }
    const double m = std::sqrt(I * I + Q * Q);
    if (m > 0.0) {
      It += I / m;
      Qt += Q / m;
    }
  }
  return std::fmod(std::atan2(Qt, It) * 180.0 / PI + 360.0, 360.0);
}

DemodArgs Context::demod_args(int T) const {
  DemodArgs da;
  da.raw = d_raw;
  da.in_fmt = in_fmt;
  da.n_read = cur_n_read;
  da.dc = dc_correct ? d_dc : nullptr;
  da.total = (long long)T * spp;
  da.tiles = T;
  da.spp = spp;
  da.tile = des.tile;
  da.ga = d_ga;
  da.gb = d_gb;
  da.tw_a = d_twa;
  da.tw_b = d_twb;
  da.tw_a_inv = d_twa_inv;
  da.tw_b_inv = d_twb_inv;
  da.a_pos = des.a_pos;
  da.a_out = des.a_out;
  da.b_pos = des.b_pos;
  da.b_out = des.b_out;
  da.rot_re = des.rot_re;
  da.rot_im = des.rot_im;
  da.d0 = (float)des.d0;
  da.demod_scale = des.demod_scale;
  da.demod_offset = des.demod_offset;
  da.corr_video = des.corr_video;
  da.corr_sync = des.corr_sync;
  da.dem = d_dem;
  da.env = d_env;
  da.env_part = d_env_part;
  da.env_blocks = env_blocks;
  da.video = d_video;
  da.sync = d_sync;
  da.pulse_bits = d_pulse_bits;
  da.thr_rel = (float)(fmt.pulse_threshold_hz - fmt.ire0);
  da.guard_hz = cfg.guard_band_hz > 0.0 ? (float)cfg.guard_band_hz : kGuardHz;
  da.guard_list = d_guard_list;
  da.guard_count = d_guard_count;
  da.guard_cap = kGuardCap;
  return da;
}

GuardArgs Context::guard_args(const DemodArgs& da) const {
  GuardArgs g;
  g.raw = da.raw;
  g.in_fmt = da.in_fmt;
  g.n_read = da.n_read;
  g.dc = da.dc;
  g.total = da.total;
  g.spp = spp;
  g.tile = des.tile;
  g.gfft = d_guard_g;
  g.tw = d_guard_tw;
  g.ha = des.ga64_half;
  g.hs64 = d_hs64;
  g.hb = des.hs64_half;
  g.scale = fmt.fs_hz / (2.0 * 3.14159265358979323846);
  g.ire0 = fmt.ire0;
  g.thr_hz = fmt.pulse_threshold_hz;
  g.thr_rel = da.thr_rel;
  g.sync = da.sync;
  g.list = d_guard_list;
  g.count = d_guard_count;
  g.cap = kGuardCap;
  g.values = d_guard_vals;
  g.flips = d_guard_flips;
  if (debug) g.dbg_clk = d_dbg_clk_guard;
  return g;
}

ChromaArgs Context::chroma_args(const uint8_t* raw, int n_read, const float* dc, int T) const {
  ChromaArgs ca;
  ca.raw = raw;
  ca.in_fmt = in_fmt;
  ca.n_read = n_read;
  ca.dc = dc;
  ca.pre = d_dem;  // the raw demod is no longer needed after K1b
  ca.fields = T;
  ca.spp = spp;
  ca.ctile = des.ctile;
  ca.c_half = des.c_half;
  ca.c_out = des.c_out;
  ca.gc = d_gc;
  ca.tw_c = d_twc;
  ca.tw_line = d_twl;
  ca.tw_c_inv = d_twc_inv;
  ca.tw_line_inv = d_twl_inv;
  ca.ll = d_ll;
  ca.total = 0;
  ca.track = d_track;
  ca.het_scale = des.het_scale;
  ca.fsc_bin = des.fsc_bin;
  ca.bw_bins = des.bw_bins;
  ca.burst_start = fmt.burst_start;
  ca.burst_len = fmt.burst_len;
  ca.line_fft = fmt.line_fft;
  ca.out_w = fmt.output_line_len;
  ca.out_h = fmt.output_field_lines;
  ca.lines_per_frame = fmt.lines_per_frame;
  ca.burst_abs_ref = (float)fmt.burst_abs_ref;
  ca.chroma = d_chroma;
  ca.burst = d_burst;
  ca.metric = dp_metric;
  ca.col_frac = d_col_frac;
  return ca;
}

LineArgs Context::line_args(int P) const {
  LineArgs la;
  la.video = d_video;
  la.sync = d_sync;
  la.ll = d_ll;
  la.fields = P;
  la.total = (long long)P * spp;
  la.lines_per_frame = fmt.lines_per_frame;
  la.active_line_start = fmt.active_line_start;
  la.thr_rel = (float)(fmt.pulse_threshold_hz - fmt.ire0);
  la.one_us = 1.0e-6 * fmt.fs_hz;
  la.hsync_width = fmt.hsync_width;
  la.right_edge_offset = 2.25 * ((fmt.fs_hz / 1.0e6) / 40.0);
  la.luma = d_luma;
  la.out_w = fmt.output_line_len;
  la.out_h = fmt.output_field_lines;
  la.luma_gain = (float)(fmt.output_scale / fmt.hz_ire);
  la.luma_offset = (float)(-fmt.vsync_ire * fmt.output_scale + fmt.output_zero);
  la.col_frac = d_col_frac;
  la.oob_value = (uint16_t)fmt.output_zero;
  return la;
}

DropoutArgs Context::dropout_args(int P) const {
  DropoutArgs dd;
  dd.env = d_env;
  dd.env_part = d_env_part;
  dd.env_blocks = env_blocks;
  dd.ll = d_ll;
  dd.fields = P;
  dd.spp = spp;
  dd.lines_per_frame = fmt.lines_per_frame;
  dd.active_line_start = fmt.active_line_start;
  dd.out_w = fmt.output_line_len;
  dd.out_h = fmt.output_field_lines;
  dd.luma = d_luma;
  dd.chroma = d_chroma;
  dd.do_count = d_do_count;
  dd.do_lines = d_do_lines;
  dd.do_starts = d_do_starts;
  dd.do_ends = d_do_ends;
  dd.cls = d_do_cls;
  dd.max_blocks = (int)dropout_class_bytes_per_field(spp);
  return dd;
}

bool Context::guard_ok(int listed) {
  if (listed <= kGuardCap) return true;
  err = "more than " + std::to_string(kGuardCap) + " sync samples near the pulse threshold in one chunk (" +
        std::to_string(listed) + "); decode shorter chunks";
  status = CUVHS_ERR_CAPACITY;
  return false;
}

bool Context::field_windows(const float* sync, long long total, int tiles, int num_fields) {
  const float thr_rel = (float)(fmt.pulse_threshold_hz - fmt.ire0);
  cudaMemsetAsync(d_counts, 0, 4 * sizeof(int), stream);
  {
    cudaEvent_t ev_;
    begin_stage(kStageEdges, ev_);
    launch_edges(sync, total, thr_rel, d_fall, d_rise, d_counts, edge_cap, d_edge_blk, d_edge_mask, stream);
    end_stage(kStageEdges, ev_, 3);
  }
  LineLocArgs la = lineloc_args(tiles, num_fields, 0);
  la.total = total;
  launch_field_windows(la, stream);
  cudaMemcpyAsync(hp_win, d_win, sizeof(WindowInfo), cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(hp_offs, d_offs, (size_t)num_fields * sizeof(long long), cudaMemcpyDeviceToHost, stream);
  if (!check_cuda("field windows") || !this->sync("field windows")) return false;
  if (hp_win->err) {
    err = "sync edge list overflow";
    status = CUVHS_ERR_CAPACITY;
    return false;
  }
  return true;
}

LineLocArgs Context::lineloc_args(int tiles, int num_fields, long long raw_offset) const {
  LineLocArgs a;
  a.fmt = fmt;
  a.fall = d_fall;
  a.rise = d_rise;
  a.counts = d_counts;
  a.edge_cap = edge_cap;
  a.total = (long long)tiles * spp;
  a.tiles = tiles;
  a.num_fields = num_fields;
  a.minw = (int)(20.0e-6 * fmt.fs_hz);
  a.maxw = (int)(35.0e-6 * fmt.fs_hz);
  a.win = d_win;
  a.offs = d_offs;
  a.cand = d_cand;
  a.cand_cap = edge_cap;
  a.ps = d_ps;
  a.pl = d_pl;
  a.pn = d_pn;
  a.vs = d_vs;
  a.vl = d_vl;
  a.vt = d_vt;
  a.vd = d_vd;
  a.vn = d_vn;
  a.prep = d_prep;
  a.state = d_lls;
  a.ll = d_ll;
  a.is_first = d_is_first;
  a.raw_offset = raw_offset;
  a.single_pass = single_pass ? 1 : 0;
  if (debug) {
    a.dbg_vs = d_dbg_vs;
    a.dbg_vl = d_dbg_vl;
    a.dbg_vt = d_dbg_vt;
    a.dbg_vn = d_dbg_vn;
    a.dbg_clk = d_dbg_clk_ll;
  }
  return a;
}

bool Context::read_lls(LineLocState& st) {
  if (cudaStreamSynchronize(stream) != cudaSuccess || cudaStreamSynchronize(lstream) != cudaSuccess ||
      cudaMemcpy(&st, d_lls, sizeof(LineLocState), cudaMemcpyDeviceToHost) != cudaSuccess)
    return check_cuda("line-location state");
  return true;
}

bool Context::write_lls(const LineLocState& st) {
  if (cudaStreamSynchronize(stream) != cudaSuccess || cudaStreamSynchronize(lstream) != cudaSuccess ||
      cudaMemcpy(d_lls, &st, sizeof(LineLocState), cudaMemcpyHostToDevice) != cudaSuccess)
    return check_cuda("line-location state");
  return true;
}

// Chroma of fields [0, P) with the track and phase decisions of
// chroma_decode.cu:640-1001: on the first chunk the track and burst phase come
// from two trial passes over field 0; then every field is computed with the
// alternating track assignment and the reference's per-15-field flip-and-retry
// passes are replayed on the host.  Sets h_phase and the carried chroma state.
bool Context::chroma_fields(ChromaArgs& ca, int P, const DropoutArgs* conceal, uint16_t* dst_chroma,
                            bool trial_on_device, cudaStream_t chroma_stream) {
  // the chroma passes run on cs; the concealment (which needs the dropout
  // lists of the decode stream) follows each pass on the decode stream
  cudaStream_t cs = chroma_stream ? chroma_stream : stream;
  const int H = fmt.output_field_lines;
  const size_t F = (size_t)fmt.output_line_len * H;
  double t_host = 0.0;
  // Fields [f0, f0 + nf) are decoded as the host's decision will most likely
  // leave them: conceal and send them now; a retry pass that rewrites fields
  // repeats this for them (concealment only ever runs on freshly decoded lines).
  auto finish = [&](int f0, int nf) {
    if (cs != stream) cudaStreamWaitEvent(stream, ev_cpass, 0);  // the pass's lines (not its metric)
    if (conceal) {
      cudaEvent_t ev_;
      begin_stage(kStageDropouts, ev_);
      launch_dropout_conceal_chroma(*conceal, f0, nf, stream);
      end_stage(kStageDropouts, ev_);
    }
    if (dst_chroma) {
      cudaEventRecord(ev_chroma, stream);
      cudaStreamWaitEvent(ostream, ev_chroma, 0);
      cudaMemcpyAsync(dst_chroma + (size_t)f0 * F, ca.chroma + (size_t)f0 * F, (size_t)nf * F * sizeof(uint16_t),
                      cudaMemcpyDeviceToHost, ostream);
    }
  };
  auto chroma_pass = [&](int f0, int nf, bool write) {
    cudaEvent_t ev_;
    begin_stage_on(kStageChromaLines, ev_, cs);
    launch_chroma_lines(ca, f0, nf, write, cs);
    end_stage_on(kStageChromaLines, ev_, cs);
    cudaEventRecord(ev_cpass, cs);  // the concealment needs the lines, not the metric
    if (write) {
      begin_stage_on(kStageBurstMetric, ev_, cs);
      launch_burst_metric(ca, f0, nf, cs);  // writes hp_metric through its mapping
      end_stage_on(kStageBurstMetric, ev_, cs);
    }
  };
  int det_track, cycle_start;
  double thr;
  const bool on_device = trial_on_device && !chroma_valid;
  const size_t nb_ = (size_t)H * fmt.burst_len;
  auto detect = [&](int& det, double& th, int& cyc) {
    const double m0 = host_burst_metric(hp_burst, H, fmt.burst_len),
                 m1 = host_burst_metric(hp_burst + nb_, H, fmt.burst_len);
    det = (m1 < m0) ? 1 : 0;
    th = (det ? m1 : m0) * 4.0;
    const double ph = host_burst_phase(hp_burst + det * nb_, H, fmt);
    const int quadrant = ((int)(ph / 90.0 + 0.5)) % 4;
    const int pid = phase_id_for(1, quadrant);
    cyc = 0;
    for (int i = 0; i < 8; i += 2)
      if (kPhaseCycle[i] == pid) {
        cyc = i;
        break;
      }
  };
  if (chroma_valid) {
    det_track = chroma_track;
    thr = chroma_threshold;
    cycle_start = chroma_cycle_start;
  } else if (on_device) {
    // the trials and the device pick ran beside luma and dropouts; the pass
    // over every field follows the pick without a host round trip, and the
    // host's own decision from the same windows is taken after it (fields
    // computed on another track are recomputed below)
    cudaStreamWaitEvent(cs, ev_trial, 0);
    det_track = cycle_start = 0;
    thr = 0.0;
  } else {
    // Track and burst phase from field 0 (chroma_decode.cu:684-743): both
    // trial tracks in one round trip; the detected track's burst windows are
    // the ones the phase measurement reads.
    const size_t nb = (size_t)H * fmt.burst_len;
    for (int t = 0; t < 2; t++) {
      cudaMemcpyAsync(d_track, hp_trial + t, sizeof(int), cudaMemcpyHostToDevice, cs);
      chroma_pass(0, 1, false);
      cudaMemcpyAsync(hp_burst + t * nb, d_burst, nb * sizeof(float), cudaMemcpyDeviceToHost, cs);
    }
    cudaEventRecord(ev_host, cs);
    t_host = host_clock();
    if (!wait_host_event("chroma track detect")) return false;
    host_phase(kHostChromaWait, t_host);
    detect(det_track, thr, cycle_start);
  }
  // Every field's chroma depends only on its own track, so all fields are
  // computed in one pass with the initial assignment; the reference's
  // 15-field chunks with up to three flip-and-retry passes each
  // (chroma_decode.cu:782-981) are then replayed on the host, recomputing
  // only fields whose track a flip changed.
  if (!on_device) {
    for (int f = 0; f < P; f++) hp_track[f] = (f & 1) ? (1 - det_track) : det_track;
    cudaMemcpyAsync(d_track, hp_track, P * sizeof(int), cudaMemcpyHostToDevice, cs);
  }
  chroma_pass(0, P, true);
  cudaEventRecord(ev_host, cs);
  finish(0, P);
  t_host = host_clock();
  if (!wait_host_event("chroma lines")) return false;
  host_phase(kHostChromaWait, t_host);
  computed_track.resize(P);
  if (on_device) {
    // the trial windows and the device's pick (copied after the pick)
    const cudaError_t e = cudaEventSynchronize(ev_trialh);
    if (e != cudaSuccess) {
      err = std::string("chroma track windows: ") + cudaGetErrorString(e);
      status = CUVHS_ERR_CUDA;
      return false;
    }
    detect(det_track, thr, cycle_start);
    const int dev = *hp_pick;
    for (int f = 0; f < P; f++) computed_track[f] = (f & 1) ? (1 - dev) : dev;
  }
  int cur = det_track;
  h_phase.assign(P, 0);
  for (int f = 0; f < P; f++) {
    hp_track[f] = (f & 1) ? (1 - cur) : cur;
    h_phase[f] = kPhaseCycle[(cycle_start + f) % 8];
    if (!on_device) computed_track[f] = hp_track[f];
  }
  const int fpc = std::max(1, std::min((4096 / H), P));
  for (int f0 = 0; f0 < P; f0 += fpc) {
    const int nf = std::min(fpc, P - f0);
    int retries = 3;
    bool ok = false;
    while (!ok && retries-- > 0) {
      bool stale = false;
      for (int f = f0; f < f0 + nf; f++) stale = stale || computed_track[f] != hp_track[f];
      if (stale) {
        cudaMemcpyAsync(d_track + f0, hp_track + f0, nf * sizeof(int), cudaMemcpyHostToDevice, cs);
        chroma_pass(f0, nf, true);
        cudaEventRecord(ev_host, cs);
        finish(f0, nf);
        if (!wait_host_event("chroma retry")) return false;
        for (int f = f0; f < f0 + nf; f++) computed_track[f] = hp_track[f];
      }
      int first_bad = INT_MAX;
      for (int f = 0; f < nf; f++)
        if (hp_metric[f0 + f] > thr) {
          first_bad = f;
          break;
        }
      if (first_bad == INT_MAX) {
        ok = true;
      } else {
        cur = 1 - cur;
        for (int ff = f0 + first_bad; ff < P; ff++) hp_track[ff] = (ff & 1) ? (1 - cur) : cur;
      }
    }
  }
  chroma_valid = true;
  chroma_track = (P & 1) ? (1 - cur) : cur;
  chroma_threshold = thr;
  chroma_cycle_start = (cycle_start + P) % 8;
  return true;
}

// Decode one chunk.  `src` is host memory unless `src_on_device`.
bool Context::decode_chunk(const uint8_t* src, bool src_on_device, size_t n_avail, uint64_t raw_offset,
                           int num_fields, ChunkResult& res, uint16_t* dst_luma, uint16_t* dst_chroma,
                           const uint8_t* cap_base, size_t cap_n, bool defer) {
  res = ChunkResult();
  // the reference reads its switch on every chunk (pipeline.cu:1694)
  single_pass = cfg.single_pass_lines != 0 || std::getenv("CUVHS_K2B_DISABLE") != nullptr;
  if (timing) {  // a new timeline (an earlier chunk that failed left its marks behind)
    marks.clear();
    pool_used = 0;
    ev_t0 = nullptr;
    t0_pending = true;
  }
  // Unless the caller defers them and the chunk succeeded, no copy into
  // caller memory or pinned staging is still in flight when this returns.
  struct CopyDrain {
    Context* c;
    bool keep = false;
    ~CopyDrain() {
      if (keep) return;
      cudaStreamSynchronize(c->xstream);
      cudaStreamSynchronize(c->ostream);
      cudaStreamSynchronize(c->hstream);
      cudaStreamSynchronize(c->pstream);  // after an error, nothing of the chunk is left running
      cudaStreamSynchronize(c->lstream);
      cudaStreamSynchronize(c->gstream);
      c->pf.valid = false;
    }
  } drain{this};
  if (num_fields < 1 || num_fields > batch) {
    err = "num_fields must be in [1, batch_fields]";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  cudaSetDevice(device);
  const size_t spf = (size_t)fmt.samples_per_field;
  const size_t total_samples = (size_t)num_fields * spp;
  const size_t n_read = std::min(total_samples, n_avail);
  if (n_read < spf) return true;  // no field: end of capture
  const int T = (int)std::min(n_read / spf, (size_t)num_fields);
  // ---- buffer sets: planes alternate between two sets when they are copied
  // out asynchronously; the input window may already be on the device
  const bool pipelined = dst_luma != nullptr || dst_chroma != nullptr;
  const int oset = pipelined ? out_set : 0;
  d_luma = d_luma_set[oset];
  d_chroma = d_chroma_set[oset];
  cudaStreamWaitEvent(stream, ev_out_done[oset], 0);  // an earlier chunk's copies out of this set
  const bool prefetched = !src_on_device && pf.valid && pf.raw_offset == raw_offset && pf.n_read == n_read &&
                          pf.total == total_samples;
  const int rset = prefetched ? pf.set : raw_set;
  pf.valid = false;
  d_raw = d_raw_set[rset];
  raw_set = rset;
  cur_n_read = (int)n_read;
  // ---- K1: FM demod over T tiles
  DemodArgs da = demod_args(T);
  cudaMemsetAsync(d_guard_count, 0, sizeof(int), stream);  // K1b lists near-threshold sync samples
  cudaMemsetAsync(d_pulse_bits, 0, pulse_bit_words((long long)T * spp) * sizeof(unsigned), stream);
  // ---- input: the chunk window (bps bytes per sample); positions past the
  // samples read count as 0 in every kernel, the reference's zero fill.  Host
  // input arrives in pieces on the copy stream; K1a of tiles [fa, fb) reads
  // chunk samples up to (fb-1)*spp - kOverlap + tile, so it starts as soon as
  // the piece reaching that far has landed.  With DC correction the chunk
  // mean is needed first, so K1a waits for the whole window.
  const int dc_kernels = dc_correct ? 2 : 0;
  auto k1a_range = [&](int f0, int nf) {
    cudaEvent_t ev_;
    begin_stage(kStageK1a, ev_);
    launch_k1a(da, f0, nf, stream);
    end_stage(kStageK1a, ev_);
  };
  auto k1b_range = [&](int f0, int nf) {
    cudaEvent_t ev_;
    begin_stage(kStageK1b, ev_);
    launch_k1b(da, f0, nf, stream);
    end_stage(kStageK1b, ev_);
  };
  auto dc_mean = [&] {
    if (!dc_correct) return;
    cudaEvent_t ev_;
    begin_stage(kStageK1a, ev_);
    launch_dc_mean(da.raw, (int)n_read, in_fmt, d_dcsum, d_dc, stream);
    end_stage(kStageK1a, ev_, dc_kernels);
  };
  if (src_on_device || prefetched) {
    // read in place (no kernel reads at or past n_read, so a short window
    // needs no copy), or the window prefetched during the previous chunk
    if (src_on_device) da.raw = src;
    else cudaStreamWaitEvent(stream, ev_prefetch, 0);
    dc_mean();
    k1a_range(0, T);
    k1b_range(0, T);
  } else {
    // host input in pieces: each tile range is demodulated (K1a) as soon as
    // its samples have landed, and filtered (K1b) one tile behind: K1b's
    // window for tile f reaches 2048 samples into tile f - 1 and a few hundred
    // into tile f + 1
    // pieces of at least ~10 tiles: smaller launches leave SMs idle (a 5-tile
    // K1a or K1b grid fills under half the GPU), which costs more than the
    // earlier start gains
    const int pieces = dc_correct ? 1 : std::max(1, std::min(kInputPieces, T / 10));
    size_t have = 0;
    int k1b_next = 0;
    for (int i = 0; i < pieces; i++) {
      const int fa = (int)((long long)T * i / pieces), fb = (int)((long long)T * (i + 1) / pieces);
      size_t need = (size_t)(fb - 1) * spp + (size_t)des.tile - kOverlap;
      if (i == pieces - 1 || need > n_read) need = n_read;
      if (need > have) {
        cudaMemcpyAsync(d_raw + have * bps, src + have * bps, (need - have) * bps, cudaMemcpyHostToDevice, hstream);
        have = need;
      }
      cudaEventRecord(ev_piece[i], hstream);
      cudaStreamWaitEvent(stream, ev_piece[i], 0);
      dc_mean();
      k1a_range(fa, fb - fa);
      const int ready = i == pieces - 1 ? T : fb - 1;  // tiles whose right neighbour is demodulated
      if (ready > k1b_next) {
        k1b_range(k1b_next, ready - k1b_next);
        k1b_next = ready;
      }
    }
  }
  // ---- the colour-under pre-band-pass needs only the raw samples, and its
  // output takes the demod buffer's place once K1b has read it: on its own
  // stream it runs beside the line locations (short, latency-bound kernels),
  // launched below.  It covers all T demodulated slots; the detected fields
  // are a prefix.
  ChromaArgs ca = chroma_args(da.raw, (int)n_read, da.dc, T);
  if (debug) {
    dbg_demod.resize(std::min<size_t>((size_t)T * spp, (size_t)debug_tiles * spp));
    cudaMemcpyAsync(dbg_demod.data(), d_dem, dbg_demod.size() * sizeof(float), cudaMemcpyDeviceToHost, stream);
  }
  cudaEventRecord(ev_k1b, stream);
  if (!check_cuda("demod")) return false;
  // ---- sync edges over the demodulated range, the field windows clustered
  // from their VSYNC runs, and the line locations: all on the device.  The
  // host reads back only the field count, offsets and next chunk start (a
  // few bytes) while the chroma pre-band-pass and the line locations run.
  // They first run on K1b's FP32 in-pulse bits, beside the guard; if the
  // guard flips a decision they run again on the corrected sync.
  const long long total_chunk = (long long)T * spp;
  LineLocArgs lla = lineloc_args(T, num_fields, (long long)raw_offset);
  // the whole chain on the high-priority line stream: its kernels are short
  // and latency bound, and the pre-band-pass (low priority) fills the SMs
  // they leave
  cudaStreamWaitEvent(lstream, ev_k1b, 0);
  if (debug) cudaMemsetAsync(d_dbg_clk_ll, 0, (size_t)batch * kPhaseSlots * sizeof(long long), lstream);
  auto windows_and_lines = [&](bool from_bits) {
    cudaMemsetAsync(d_counts, 0, 4 * sizeof(int), lstream);
    {
      cudaEvent_t ev_;
      begin_stage_on(kStageEdges, ev_, lstream);
      if (from_bits) {
        launch_edges_bits(d_pulse_bits, total_chunk, d_fall, d_rise, d_counts, edge_cap, d_edge_blk, lstream);
      } else {
        const float thr_rel = (float)(fmt.pulse_threshold_hz - fmt.ire0);
        launch_edges(d_sync, total_chunk, thr_rel, d_fall, d_rise, d_counts, edge_cap, d_edge_blk, d_edge_mask,
                     lstream);
      }
      end_stage_on(kStageEdges, ev_, lstream, 3);
    }
    cudaEventRecord(ev_edges, lstream);
    {
      cudaEvent_t ev_;
      begin_stage_on(kStageWindows, ev_, lstream);
      launch_field_windows(lla, lstream);
      end_stage_on(kStageWindows, ev_, lstream);
    }
    cudaEventRecord(ev_win, lstream);
    // the window record and offsets come back on the copy stream
    cudaStreamWaitEvent(xstream, ev_win, 0);
    cudaMemcpyAsync(hp_win, d_win, sizeof(WindowInfo), cudaMemcpyDeviceToHost, xstream);
    cudaMemcpyAsync(hp_offs, d_offs, (size_t)num_fields * sizeof(long long), cudaMemcpyDeviceToHost, xstream);
    cudaEventRecord(ev_winhost, xstream);
    // the carried line-location state is kept for a second run
    cudaMemcpyAsync(from_bits ? d_lls_save : d_lls, from_bits ? d_lls : d_lls_save, sizeof(LineLocState),
                    cudaMemcpyDeviceToDevice, lstream);
    {
      cudaEvent_t ev_;
      begin_stage_on(kStageLines, ev_, lstream);
      launch_field_pulses(lla, lstream);
      launch_line_locations(lla, lstream);
      end_stage_on(kStageLines, ev_, lstream, single_pass ? 2 : 3);
    }
    cudaEventRecord(ev_ll, lstream);
  };
  windows_and_lines(true);
  // The FP64 guard follows the edges (it needs only the raw capture and K1b's
  // list, and leaves the edge kernels the whole GPU); the colour-under
  // pre-band-pass, needed only by the chroma lines, follows the field windows
  // on the low-priority stream and fills the SMs the line locations leave.
  {
    cudaStreamWaitEvent(gstream, ev_edges, 0);
    cudaMemsetAsync(d_guard_flips, 0, sizeof(int), gstream);
    cudaEvent_t ev_;
    begin_stage_on(kStageGuard, ev_, gstream);
    launch_sync_guard(guard_args(da), gstream);
    end_stage_on(kStageGuard, ev_, gstream);
    cudaMemcpyAsync(hp_guard, d_guard_count, sizeof(int), cudaMemcpyDeviceToHost, gstream);
    cudaMemcpyAsync(hp_guard + 1, d_guard_flips, sizeof(int), cudaMemcpyDeviceToHost, gstream);
    cudaEventRecord(ev_guard, gstream);
  }
  cudaStreamWaitEvent(pstream, ev_edges, 0);
  {
    cudaEvent_t ev_;
    begin_stage_on(kStageChromaPre, ev_, pstream);
    launch_chroma_prefilter(ca, pstream);
    end_stage_on(kStageChromaPre, ev_, pstream);
  }
  cudaEventRecord(ev_pre, pstream);
  if (!check_cuda("guard and pre-band-pass")) return false;
  const int LPF = fmt.lines_per_frame;
  const int H = fmt.output_field_lines;
  if (!check_cuda("chroma prefilter")) return false;
  double t_host = host_clock();
  auto wait_event = [&](cudaEvent_t e, const char* what) {
    const cudaError_t r = cudaEventSynchronize(e);
    if (r != cudaSuccess) {
      err = std::string(what) + ": " + cudaGetErrorString(r);
      status = CUVHS_ERR_CUDA;
      return false;
    }
    return true;
  };
  if (!wait_event(ev_winhost, "field windows") || !wait_event(ev_guard, "sync guard")) return false;
  if (!guard_ok(hp_guard[0])) return false;
  if (hp_guard[1] > 0) {
    // a threshold decision flipped: edges, windows and line locations again
    // (after the speculative ones on the same stream) on the corrected sync
    cudaStreamWaitEvent(lstream, ev_guard, 0);
    windows_and_lines(false);
    if (!wait_event(ev_winhost, "field windows")) return false;
  }
  host_phase(kHostWindowsWait, t_host);
  if (hp_win->err) {
    err = "sync edge list overflow";
    status = CUVHS_ERR_CAPACITY;
    return false;
  }
  const int P = hp_win->fields;
  res.next_raw_offset = raw_offset + (uint64_t)hp_win->next_rel;
  // ---- the next chunk of a host capture starts at next_raw_offset: copy its
  // window into the other raw buffer now (the chunk loop's arithmetic, so the
  // next call finds it); the previous chunk that read that buffer has ended.
  if (cap_base && !src_on_device && res.next_raw_offset < cap_n) {
    const uint64_t nxt = res.next_raw_offset;
    const size_t rem_fields = (size_t)(cap_n - nxt) / spf;
    if (rem_fields > 0) {
      const int nf = (int)std::min<size_t>((size_t)batch, rem_fields);
      const size_t tot = (size_t)nf * spp, nr = std::min(tot, (size_t)(cap_n - nxt));
      if (nr >= spf) {
        const int ps = 1 - rset;
        cudaMemcpyAsync(d_raw_set[ps], cap_base + nxt * bps, nr * bps, cudaMemcpyHostToDevice, hstream);
        cudaEventRecord(ev_prefetch, hstream);
        pf.valid = true;
        pf.raw_offset = nxt;
        pf.n_read = nr;
        pf.total = tot;
        pf.set = ps;
      }
    }
  }
  if (debug) {
    // the chunk's intermediates as the reference keeps them: VSYNC
    // candidates, raw and validated pulses, coarse line locations
    if (cudaStreamSynchronize(lstream) != cudaSuccess || cudaStreamSynchronize(gstream) != cudaSuccess)
      return check_cuda("line locations");
    const int nc = std::min(hp_win->ncand, edge_cap);
    dbg_vsync.resize(nc);
    if (nc) cudaMemcpy(dbg_vsync.data(), d_cand, nc * sizeof(int), cudaMemcpyDeviceToHost);
    const size_t np = (size_t)P * kMaxPulses;
    dbg_k2c.assign(P, 0);
    dbg_k2s.assign(np, 0);
    dbg_k2l.assign(np, 0);
    dbg_k2bc.assign(P, 0);
    dbg_k2bs.assign(np, 0);
    dbg_k2bl.assign(np, 0);
    dbg_k2bt.assign(np, kHsync);
    if (P) {
      cudaMemcpy(dbg_k2c.data(), d_pn, P * sizeof(int), cudaMemcpyDeviceToHost);
      cudaMemcpy(dbg_k2bc.data(), d_dbg_vn, P * sizeof(int), cudaMemcpyDeviceToHost);
      std::vector<int> tmp(np);
      auto rows = [&](const int* d, std::vector<int>& out, const std::vector<int>& cnt) {
        cudaMemcpy(tmp.data(), d, np * sizeof(int), cudaMemcpyDeviceToHost);
        for (int f = 0; f < P; f++)
          std::copy(tmp.begin() + (size_t)f * kMaxPulses, tmp.begin() + (size_t)f * kMaxPulses + cnt[f],
                    out.begin() + (size_t)f * kMaxPulses);
      };
      rows(d_ps, dbg_k2s, dbg_k2c);
      rows(d_pl, dbg_k2l, dbg_k2c);
      rows(d_dbg_vs, dbg_k2bs, dbg_k2bc);
      rows(d_dbg_vl, dbg_k2bl, dbg_k2bc);
      rows(d_dbg_vt, dbg_k2bt, dbg_k2bc);
    }
    dbg_offs.assign(hp_offs, hp_offs + P);
    dbg_ll_coarse.resize((size_t)P * LPF);
    if (P) cudaMemcpy(dbg_ll_coarse.data(), d_ll, dbg_ll_coarse.size() * sizeof(double), cudaMemcpyDeviceToHost);
    dbg_meta = {T, P, spp};
    const int ng = std::min(hp_guard[0], kGuardCap);
    std::vector<unsigned> pos(ng);
    dbg_guard_vals.resize(ng);
    if (ng) {
      cudaMemcpy(pos.data(), d_guard_list, ng * sizeof(unsigned), cudaMemcpyDeviceToHost);
      cudaMemcpy(dbg_guard_vals.data(), d_guard_vals, ng * sizeof(double), cudaMemcpyDeviceToHost);
    }
    dbg_guard_pos.assign(pos.begin(), pos.end());
    dbg_clk_ll.resize((size_t)P * kPhaseSlots);
    if (P) cudaMemcpy(dbg_clk_ll.data(), d_dbg_clk_ll, dbg_clk_ll.size() * sizeof(long long), cudaMemcpyDeviceToHost);
    dbg_clk_guard.resize((size_t)std::min(ng, kGuardClockSamples) * kPhaseSlots);
    if (!dbg_clk_guard.empty())
      cudaMemcpy(dbg_clk_guard.data(), d_dbg_clk_guard, dbg_clk_guard.size() * sizeof(long long),
                 cudaMemcpyDeviceToHost);
  }
  if (P == 0) {
    // no field window (the reference returns 0 fields): drain and report none
    if (!sync("empty chunk")) return false;
    res.fields = 0;
    return true;
  }
  // ---- K4 hsync refinement on the line stream after the line locations (it
  // gates the chroma, so it runs at the highest priority), then K5 luma
  cudaStreamWaitEvent(lstream, ev_guard, 0);
  LineArgs la = line_args(P);
  {
    cudaEvent_t ev_;
    begin_stage_on(kStageHsync, ev_, lstream);
    launch_hsync_refine(la, lstream);
    end_stage_on(kStageHsync, ev_, lstream);
  }
  // ---- chroma track detection of a chunk without carried chroma state
  // (chroma_decode.cu:684-743): both trial passes over field 0 in one launch
  // and the device pick, on the pre-band-pass stream (they need its output
  // and field 0's refined line starts), beside luma and dropouts
  // (the chroma passes follow on the same stream, after the refinement)
  cudaEventRecord(ev_hs, lstream);
  cudaStreamWaitEvent(stream, ev_hs, 0);
  cudaStreamWaitEvent(pstream, ev_hs, 0);
  const bool trial_on_device = !chroma_valid;
  if (trial_on_device) {
    const size_t nb = (size_t)H * fmt.burst_len;
    ArgsMany<ChromaArgs> tm;
    for (int t = 0; t < 2; t++) {
      tm.a[t] = ca;
      tm.a[t].fields = 1;
      tm.a[t].total = (long long)P * spp;  // the full pass's signal range
      tm.a[t].track = d_trial + t;
      tm.a[t].burst = d_burst_trial + t * nb;
    }
    cudaEvent_t ev_;
    begin_stage_on(kStageChromaLines, ev_, pstream);
    launch_chroma_lines_many(tm, 2, -1, 1, false, pstream);
    end_stage_on(kStageChromaLines, ev_, pstream);
    TrackPickArgs tp;
    tp.burst0 = d_burst_trial;
    tp.burst1 = d_burst_trial + nb;
    tp.out_h = H;
    tp.burst_len = fmt.burst_len;
    tp.fields = P;
    tp.track = d_track;
    tp.pick = d_pick;
    launch_track_pick(tp, pstream);
    cudaEventRecord(ev_trial, pstream);
    // the windows and the pick go to the host on the copy stream, so that
    // the chroma pass follows the pick directly
    cudaStreamWaitEvent(xstream, ev_trial, 0);
    cudaMemcpyAsync(hp_burst, d_burst_trial, 2 * nb * sizeof(float), cudaMemcpyDeviceToHost, xstream);
    cudaMemcpyAsync(hp_pick, d_pick, sizeof(int), cudaMemcpyDeviceToHost, xstream);
    cudaEventRecord(ev_trialh, xstream);
  }
  {
    cudaEvent_t ev_;
    begin_stage(kStageLuma, ev_);
    launch_luma(la, stream);
    end_stage(kStageLuma, ev_);
  }
  if (!check_cuda("lines")) return false;
  // ---- K7 dropouts: detection, mapping and luma concealment (luma is final
  // now, so it leaves the device on the copy stream while chroma decodes)
  DropoutArgs dd = dropout_args(P);
  {
    cudaEvent_t ev_;
    begin_stage(kStageDropouts, ev_);
    launch_dropouts_two_pass(dd, stream);
    end_stage(kStageDropouts, ev_, 2);
  }
  if (!check_cuda("dropouts")) return false;
  // the copy stream takes the finished luma and the dropout lists (read by the
  // host after the final synchronisation)
  const size_t F = (size_t)fmt.output_line_len * H;
  cudaEventRecord(ev_luma, stream);
  cudaStreamWaitEvent(xstream, ev_luma, 0);
  cudaMemcpyAsync(hp_do_count, d_do_count, P * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  cudaMemcpyAsync(hp_is_first, d_is_first, P * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  const size_t ndo = (size_t)P * kMaxDropouts;
  cudaMemcpyAsync(hp_do_lines, d_do_lines, ndo * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  cudaMemcpyAsync(hp_do_starts, d_do_starts, ndo * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  cudaMemcpyAsync(hp_do_ends, d_do_ends, ndo * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  cudaEventRecord(ev_small, xstream);
  if (dst_luma) {
    cudaStreamWaitEvent(ostream, ev_luma, 0);
    cudaMemcpyAsync(dst_luma, d_luma, (size_t)P * F * sizeof(uint16_t), cudaMemcpyDeviceToHost, ostream);
  }
  // ---- K6 chroma on the P detected fields
  ca.fields = P;
  ca.total = (long long)P * spp;
  // the chroma lines run on the pre-band-pass stream beside luma and
  // dropouts; each pass is concealed and sent as it is decoded (chroma_fields)
  if (!chroma_fields(ca, P, &dd, dst_chroma, trial_on_device, pstream)) return false;
  if (!check_cuda("chroma concealment")) return false;
  cudaEventRecord(ev_out_done[oset], ostream);
  if (debug) {
    dbg_ll.resize((size_t)P * LPF);
    cudaMemcpyAsync(dbg_ll.data(), d_ll, dbg_ll.size() * sizeof(double), cudaMemcpyDeviceToHost, stream);
    const size_t nt = std::min<size_t>((size_t)T * spp, (size_t)debug_tiles * spp);
    dbg_video.resize(nt);
    dbg_sync.resize(nt);
    dbg_env.resize(nt);
    dbg_pre.resize(std::min<size_t>((size_t)P * spp, nt));
    cudaMemcpyAsync(dbg_video.data(), d_video, nt * sizeof(float), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(dbg_sync.data(), d_sync, nt * sizeof(float), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(dbg_env.data(), d_env, nt * sizeof(float), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(dbg_pre.data(), d_dem, dbg_pre.size() * sizeof(float), cudaMemcpyDeviceToHost, stream);
  }
  t_host = host_clock();
  {
    // the decode stream and the dropout lists; the plane copies may continue
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(ev_small);
    if (e != cudaSuccess) {
      err = std::string("decode: ") + cudaGetErrorString(e);
      status = CUVHS_ERR_CUDA;
      return false;
    }
    collect_stage_times();
    ev_t0 = nullptr;  // the chunk's timeline is complete: its events may be reused
    pool_used = 0;
    if (!check_cuda("decode")) return false;
  }
  host_phase(kHostFinalWait, t_host);
  if (pipelined) out_set = 1 - oset;
  drain.keep = defer;
  last_fields = P;
  res.outputs_copied = dst_luma != nullptr || dst_chroma != nullptr;
  // ---- field metadata: parity alternation (pipeline.cu:2575-2610)
  res.fields = P;
  res.field_info.resize(P);
  for (int i = 0; i < P; i++) {
    cuvhs_field_info& fi = res.field_info[i];
    fi.file_loc = raw_offset + (uint64_t)hp_offs[i];
    bool first;
    if (hp_is_first[i] >= 0 && (hp_is_first[i] == 1) != last_parity) first = (hp_is_first[i] == 1);
    else first = !last_parity;
    last_parity = first;
    fi.is_first_field = first ? 1 : 0;
    fi.field_phase_id = h_phase[i] > 0 ? h_phase[i] : 0;
    fi.dropout_count = std::max(0, std::min(hp_do_count[i], kMaxDropouts));
    fi.dropout_offset = 0;
  }
  if (debug) dbg_is_first.assign(hp_is_first, hp_is_first + P);
  return true;
}

}  // namespace cuvhs
