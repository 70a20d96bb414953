// Batched rounds: the next chunk of up to kMaxPortions captures of one sample
// rate decoded together, each stage one launch over all of them.
//
// The reference decodes one capture per process (src/main.cpp:97-165), each
// as a chain of chunks (src/pipeline/pipeline.cu:2626-2713).  A round places
// each capture's chunk in its own run of field slots of the context's
// buffers -- raw window, demod, video, sync, envelope, planes, line tables,
// edge and guard lists at the slot's offset -- and launches every kernel once
// over all captures (grid.z picks the capture; each capture's kernel
// arguments are those of its chunk alone).  Every capture is therefore decoded
// exactly as cuvhs_decode_capture decodes it with the same chunk size: the
// same arithmetic on the same samples, with its own carried state (parity,
// line-location history, chroma track and phase cycle).  The host's
// decisions (field counts, the chroma track detection and retries) are taken
// per capture after one wait for all of them.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "pipeline.h"

namespace cuvhs {

bool Context::decode_round(std::vector<Portion>& ps, const RoundPlan& next_plan) {
  cudaSetDevice(device);
  const int K = (int)ps.size();
  if (K < 1 || K > kMaxPortions) {
    err = "a round holds 1 to " + std::to_string(kMaxPortions) + " captures";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  if (dc_correct || debug) {
    err = "batched rounds decode without DC correction or debug capture";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  single_pass = cfg.single_pass_lines != 0 || std::getenv("CUVHS_K2B_DISABLE") != nullptr;
  const size_t spf = (size_t)fmt.samples_per_field;
  int slots = 0;
  for (Portion& p : ps) {
    p.res = ChunkResult();
    if (p.num_fields < 1 || p.slot0 != slots || p.st == nullptr) {
      err = "round portions must fill consecutive slots and carry a state";
      status = CUVHS_ERR_INVALID_ARGUMENT;
      return false;
    }
    slots += p.num_fields;
    const size_t total = (size_t)p.num_fields * spp;
    p.n_read = (int)std::min(total, p.n_avail);
    p.T = p.n_read < (int)spf ? 0 : (int)std::min((size_t)p.n_read / spf, (size_t)p.num_fields);
  }
  if (slots > batch) {
    err = "round exceeds the context's field slots";
    status = CUVHS_ERR_INVALID_ARGUMENT;
    return false;
  }
  // captures with a field to decode; the others end here (no field: end of capture)
  std::vector<int> live;
  for (int k = 0; k < K; k++)
    if (ps[k].T > 0) live.push_back(k);
  const int L = (int)live.size();
  if (L == 0) return true;
  // On return nothing of the round runs but its plane copies, which leave
  // from one of two plane sets while the next round runs (drain_copies waits
  // for them); after an error nothing of it runs at all.
  struct Drain {
    Context* c;
    bool keep_copies = false;
    ~Drain() {
      for (cudaStream_t st : {c->stream, c->pstream, c->lstream, c->gstream}) cudaStreamSynchronize(st);
      cudaStreamSynchronize(c->xstream);
      if (!keep_copies) {
        cudaStreamSynchronize(c->ostream);
        cudaStreamSynchronize(c->hstream);
        c->rpf.valid = false;
      }
      c->pf.valid = false;
    }
  } drain{this};
  // the round's input: prefetched by the round before, or copied now
  auto sig_of = [&](const std::vector<Portion>& v, const std::vector<int>& which) {
    std::vector<std::pair<const uint8_t*, long long>> sg;
    for (int k : which) sg.push_back({v[k].src, ((long long)v[k].n_read << 20) | v[k].slot0});
    return sg;
  };
  bool prefetched = false;
  {
    std::vector<int> all(L);
    for (int j = 0; j < L; j++) all[j] = live[j];
    if (rpf.valid && rpf.sig == sig_of(ps, all)) {
      prefetched = true;
      round_raw_set = rpf.set;
    }
    rpf.valid = false;
  }
  const size_t F = (size_t)fmt.output_line_len * fmt.output_field_lines;
  const int H = fmt.output_field_lines, LPF = fmt.lines_per_frame;
  const int oset = out_set;
  d_luma = d_luma_set[oset];
  d_chroma = d_chroma_set[oset];
  d_raw = d_raw_set[round_raw_set];
  cudaStreamWaitEvent(stream, ev_out_done[oset], 0);  // the copies of the round before last out of this set
  const size_t wps = kBitWordsPerSlot(spp), eps = kEdgesPerSlot(spp), bps_ = kEdgeBlocksPerSlot(spp);
  int max_T = 0, max_nf = 0;
  for (int j = 0; j < L; j++) {
    max_T = std::max(max_T, ps[live[j]].T);
    max_nf = std::max(max_nf, ps[live[j]].num_fields);
  }
  // ---- arguments of each live capture's chunk: the one-chunk arguments at its slots
  static thread_local ArgsMany<DemodArgs> dm;
  static thread_local ArgsMany<GuardArgs> gm;
  static thread_local ArgsMany<EdgeArgs> em;
  static thread_local ArgsMany<LineLocArgs> lm;
  static thread_local ArgsMany<ChromaArgs> cm;
  static thread_local ArgsMany<LineArgs> nm;
  static thread_local ArgsMany<DropoutArgs> om;
  for (int j = 0; j < L; j++) {
    Portion& p = ps[live[j]];
    const size_t s0 = (size_t)p.slot0;
    cur_n_read = p.n_read;
    DemodArgs da = demod_args(p.T);
    da.raw = d_raw + s0 * spp * bps;
    da.dem = d_dem + s0 * spp;
    da.env = d_env + s0 * spp;
    da.env_part = d_env_part + s0 * env_blocks;
    da.video = d_video + s0 * spp;
    da.sync = d_sync + s0 * spp;
    da.pulse_bits = d_pulse_bits + s0 * wps;
    da.guard_list = d_guard_list + s0 * kGuardPerSlot;
    da.guard_count = d_guard_count + j;
    da.guard_cap = p.num_fields * kGuardPerSlot;
    dm.a[j] = da;
    GuardArgs g = guard_args(da);
    g.list = da.guard_list;
    g.count = da.guard_count;
    g.cap = da.guard_cap;
    g.values = d_guard_vals + s0 * kGuardPerSlot;
    g.flips = d_guard_flips + j;
    g.dbg_clk = nullptr;
    gm.a[j] = g;
    EdgeArgs e;
    e.bits = da.pulse_bits;
    e.total = (long long)p.T * spp;
    e.blk = d_edge_blk + s0 * bps_;
    e.counts = d_counts + 4 * j;
    e.fall = d_fall + s0 * eps;
    e.rise = d_rise + s0 * eps;
    e.cap = (int)std::min<size_t>((size_t)p.num_fields * eps, INT_MAX / 2);
    em.a[j] = e;
    LineLocArgs la = lineloc_args(p.T, p.num_fields, (long long)p.raw_offset);
    la.fall = e.fall;
    la.rise = e.rise;
    la.counts = e.counts;
    la.edge_cap = e.cap;
    la.win = d_win + j;
    la.offs = d_offs + s0;
    la.cand = d_cand + s0 * eps;
    la.cand_cap = e.cap;
    la.ps = d_ps + s0 * kMaxPulses;
    la.pl = d_pl + s0 * kMaxPulses;
    la.pn = d_pn + s0;
    la.vs = d_vs + s0 * kMaxValid;
    la.vl = d_vl + s0 * kMaxValid;
    la.vt = d_vt + s0 * kMaxValid;
    la.vd = d_vd + s0 * kMaxValid;
    la.vn = d_vn + s0;
    la.prep = d_prep + s0;
    la.state = d_lls + j;
    la.ll = d_ll + s0 * LPF;
    la.is_first = d_is_first + s0;
    lm.a[j] = la;
    ChromaArgs ca = chroma_args(da.raw, p.n_read, da.dc, p.T);
    ca.pre = da.dem;
    ca.ll = la.ll;
    ca.track = d_track + s0;
    ca.chroma = d_chroma + s0 * F;
    ca.burst = d_burst + s0 * (size_t)H * fmt.burst_len;
    ca.metric = dp_metric + s0;
    cm.a[j] = ca;
    hp_lls[j] = p.st->lls;
  }
  // ---- input windows (one copy per capture, unless prefetched) and the
  // carried line-location states
  if (!prefetched)
    for (int j = 0; j < L; j++) {
      const Portion& p = ps[live[j]];
      cudaMemcpyAsync(d_raw + (size_t)p.slot0 * spp * bps, p.src, (size_t)p.n_read * bps, cudaMemcpyHostToDevice,
                      hstream);
    }
  cudaMemcpyAsync(d_lls, hp_lls, (size_t)L * sizeof(LineLocState), cudaMemcpyHostToDevice, hstream);
  cudaEventRecord(ev_piece[0], hstream);
  cudaStreamWaitEvent(stream, ev_piece[0], 0);
  cudaMemsetAsync(d_guard_count, 0, (size_t)L * sizeof(int), stream);
  for (int j = 0; j < L; j++)
    cudaMemsetAsync(dm.a[j].pulse_bits, 0, pulse_bit_words((long long)ps[live[j]].T * spp) * sizeof(unsigned),
                    stream);
  {
    cudaEvent_t ev_;
    begin_stage(kStageK1a, ev_);
    launch_k1a_many(dm, L, max_T, stream);
    end_stage(kStageK1a, ev_);
    begin_stage(kStageK1b, ev_);
    launch_k1b_many(dm, L, max_T, stream);
    end_stage(kStageK1b, ev_);
  }
  cudaEventRecord(ev_k1b, stream);
  if (!check_cuda("round demod")) return false;
  // ---- edges, field windows and line locations on the line stream; the
  // guard after the edges; the pre-band-pass after the windows
  cudaStreamWaitEvent(lstream, ev_k1b, 0);
  auto windows_and_lines = [&](bool from_bits) {
    cudaMemsetAsync(d_counts, 0, (size_t)4 * L * sizeof(int), lstream);
    cudaEvent_t ev_;
    begin_stage_on(kStageEdges, ev_, lstream);
    if (from_bits) {
      launch_edges_bits_many(em, L, (long long)max_T * spp, lstream);
    } else {
      const float thr_rel = (float)(fmt.pulse_threshold_hz - fmt.ire0);
      for (int j = 0; j < L; j++)
        launch_edges(dm.a[j].sync, em.a[j].total, thr_rel, em.a[j].fall, em.a[j].rise, em.a[j].counts, em.a[j].cap,
                     em.a[j].blk, d_edge_mask, lstream);
    }
    end_stage_on(kStageEdges, ev_, lstream, 3);
    cudaEventRecord(ev_edges, lstream);
    begin_stage_on(kStageWindows, ev_, lstream);
    launch_field_windows_many(lm, L, lstream);
    end_stage_on(kStageWindows, ev_, lstream);
    cudaEventRecord(ev_win, lstream);
    cudaStreamWaitEvent(xstream, ev_win, 0);
    cudaMemcpyAsync(hp_win, d_win, (size_t)L * sizeof(WindowInfo), cudaMemcpyDeviceToHost, xstream);
    cudaMemcpyAsync(hp_offs, d_offs, (size_t)slots * sizeof(long long), cudaMemcpyDeviceToHost, xstream);
    cudaEventRecord(ev_winhost, xstream);
    cudaMemcpyAsync(from_bits ? d_lls_save : d_lls, from_bits ? d_lls : d_lls_save, (size_t)L * sizeof(LineLocState),
                    cudaMemcpyDeviceToDevice, lstream);
    begin_stage_on(kStageLines, ev_, lstream);
    launch_field_pulses_many(lm, L, max_nf, lstream);
    launch_line_locations_many(lm, L, max_nf, lstream);
    end_stage_on(kStageLines, ev_, lstream, single_pass ? 2 : 3);
    cudaEventRecord(ev_ll, lstream);
  };
  windows_and_lines(true);
  {
    cudaStreamWaitEvent(gstream, ev_edges, 0);
    cudaMemsetAsync(d_guard_flips, 0, (size_t)L * sizeof(int), gstream);
    cudaEvent_t ev_;
    begin_stage_on(kStageGuard, ev_, gstream);
    launch_sync_guard_many(gm, L, gstream);
    end_stage_on(kStageGuard, ev_, gstream);
    cudaMemcpyAsync(hp_guard, d_guard_count, (size_t)L * sizeof(int), cudaMemcpyDeviceToHost, gstream);
    cudaMemcpyAsync(hp_guard + kMaxPortions, d_guard_flips, (size_t)L * sizeof(int), cudaMemcpyDeviceToHost,
                    gstream);
    cudaEventRecord(ev_guard, gstream);
  }
  cudaStreamWaitEvent(pstream, ev_win, 0);
  {
    cudaEvent_t ev_;
    begin_stage_on(kStageChromaPre, ev_, pstream);
    launch_chroma_prefilter_many(cm, L, max_T, pstream);
    end_stage_on(kStageChromaPre, ev_, pstream);
  }
  cudaEventRecord(ev_pre, pstream);
  if (!check_cuda("round line locations")) return false;
  double t_host = host_clock();
  if (cudaEventSynchronize(ev_winhost) != cudaSuccess || cudaEventSynchronize(ev_guard) != cudaSuccess)
    return check_cuda("round windows");
  int flips = 0;
  for (int j = 0; j < L; j++) {
    if (hp_guard[j] > gm.a[j].cap) {
      err = "more than " + std::to_string(gm.a[j].cap) + " sync samples near the pulse threshold in one chunk (" +
            std::to_string(hp_guard[j]) + "); decode shorter chunks";
      status = CUVHS_ERR_CAPACITY;
      return false;
    }
    flips += hp_guard[kMaxPortions + j];
  }
  if (flips > 0) {
    cudaStreamWaitEvent(lstream, ev_guard, 0);
    windows_and_lines(false);
    if (cudaEventSynchronize(ev_winhost) != cudaSuccess) return check_cuda("round windows");
  }
  host_phase(kHostWindowsWait, t_host);
  int max_P = 0;
  for (int j = 0; j < L; j++) {
    Portion& p = ps[live[j]];
    if (hp_win[j].err) {
      err = "sync edge list overflow";
      status = CUVHS_ERR_CAPACITY;
      return false;
    }
    p.res.fields = hp_win[j].fields;
    p.res.next_raw_offset = p.raw_offset + (uint64_t)hp_win[j].next_rel;
    max_P = std::max(max_P, p.res.fields);
  }
  // ---- the next round's input windows, into the other raw buffer
  if (next_plan) {
    std::vector<Portion> next;
    next_plan(ps, next);
    std::vector<int> nlive;
    const int other = 1 - round_raw_set;
    for (int k = 0; k < (int)next.size(); k++) {
      Portion& q = next[k];
      const size_t total = (size_t)q.num_fields * spp;
      q.n_read = (int)std::min(total, q.n_avail);
      if (q.n_read < (int)spf) continue;  // no field: not decoded
      nlive.push_back(k);
      cudaMemcpyAsync(d_raw_set[other] + (size_t)q.slot0 * spp * bps, q.src, (size_t)q.n_read * bps,
                      cudaMemcpyHostToDevice, hstream);
    }
    if (!nlive.empty()) {
      rpf.valid = true;
      rpf.set = other;
      rpf.sig = sig_of(next, nlive);
    }
  }
  if (max_P == 0) {
    if (!sync("empty round")) return false;
    return true;
  }
  cudaStreamWaitEvent(stream, ev_ll, 0);
  cudaStreamWaitEvent(stream, ev_guard, 0);
  // ---- hsync, luma, dropouts over every capture's detected fields
  for (int j = 0; j < L; j++) {
    const Portion& p = ps[live[j]];
    const size_t s0 = (size_t)p.slot0;
    LineArgs la = line_args(p.res.fields);
    la.video = dm.a[j].video;
    la.sync = dm.a[j].sync;
    la.ll = lm.a[j].ll;
    la.luma = d_luma + s0 * F;
    nm.a[j] = la;
    DropoutArgs dd = dropout_args(p.res.fields);
    dd.env = dm.a[j].env;
    dd.env_part = dm.a[j].env_part;
    dd.ll = lm.a[j].ll;
    dd.luma = la.luma;
    dd.chroma = cm.a[j].chroma;
    dd.do_count = d_do_count + s0;
    dd.do_lines = d_do_lines + s0 * kMaxDropouts;
    dd.do_starts = d_do_starts + s0 * kMaxDropouts;
    dd.do_ends = d_do_ends + s0 * kMaxDropouts;
    dd.cls = d_do_cls + s0 * (size_t)dd.max_blocks;
    om.a[j] = dd;
    cm.a[j].fields = p.res.fields;
    cm.a[j].total = (long long)p.res.fields * spp;
  }
  {
    cudaEvent_t ev_;
    begin_stage(kStageHsync, ev_);
    launch_hsync_refine_many(nm, L, max_P, stream);
    end_stage(kStageHsync, ev_);
    begin_stage(kStageLuma, ev_);
    launch_luma_many(nm, L, max_P, stream);
    end_stage(kStageLuma, ev_);
    begin_stage(kStageDropouts, ev_);
    launch_dropouts_two_pass_many(om, L, max_P, stream);
    end_stage(kStageDropouts, ev_, 2);
  }
  if (!check_cuda("round lines")) return false;
  // luma and the small per-field results leave on the copy stream
  cudaEventRecord(ev_luma, stream);
  cudaStreamWaitEvent(xstream, ev_luma, 0);
  cudaMemcpyAsync(hp_do_count, d_do_count, (size_t)slots * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  cudaMemcpyAsync(hp_is_first, d_is_first, (size_t)slots * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  const size_t ndo = (size_t)slots * kMaxDropouts;
  cudaMemcpyAsync(hp_do_lines, d_do_lines, ndo * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  cudaMemcpyAsync(hp_do_starts, d_do_starts, ndo * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  cudaMemcpyAsync(hp_do_ends, d_do_ends, ndo * sizeof(int), cudaMemcpyDeviceToHost, xstream);
  cudaEventRecord(ev_small, xstream);
  cudaStreamWaitEvent(ostream, ev_luma, 0);
  for (int j = 0; j < L; j++) {
    const Portion& p = ps[live[j]];
    if (p.dst_luma && p.res.fields > 0)
      cudaMemcpyAsync(p.dst_luma, nm.a[j].luma, (size_t)p.res.fields * F * sizeof(uint16_t), cudaMemcpyDeviceToHost,
                      ostream);
  }
  // ---- chroma: track and phase for captures without carried chroma state
  // (two trial passes over field 0 of every capture), then every field, then
  // the per-capture flip-and-retry replay (chroma_decode.cu:640-1001)
  cudaStreamWaitEvent(stream, ev_pre, 0);
  const size_t nb = (size_t)H * fmt.burst_len;
  std::vector<int> det(L), cyc(L), cur(L);
  std::vector<double> thr(L);
  bool any_detect = false;
  for (int j = 0; j < L; j++) any_detect = any_detect || !ps[live[j]].st->chroma_valid;
  if (any_detect) {
    if (!hp_round_burst) {
      void* q = nullptr;
      if (cudaHostAlloc(&q, (size_t)2 * kMaxPortions * nb * sizeof(float), cudaHostAllocDefault) != cudaSuccess)
        return check_cuda("round burst staging");
      host_allocations.push_back(q);
      hp_round_burst = static_cast<float*>(q);
    }
    // the trial passes read field 0 of the captures that detect (and have a
    // field); both trials go out before one wait, as in chroma_fields
    for (int j = 0; j < L; j++)
      cm.a[j].fields = (!ps[live[j]].st->chroma_valid && ps[live[j]].res.fields > 0) ? 1 : 0;
    for (int t = 0; t < 2; t++) {
      for (int j = 0; j < L; j++)
        cudaMemcpyAsync(d_track + ps[live[j]].slot0, hp_trial + t, sizeof(int), cudaMemcpyHostToDevice, stream);
      cudaEvent_t ev_;
      begin_stage(kStageChromaLines, ev_);
      launch_chroma_lines_many(cm, L, -1, 1, false, stream);
      end_stage(kStageChromaLines, ev_);
      for (int j = 0; j < L; j++)
        if (cm.a[j].fields > 0)
          cudaMemcpyAsync(hp_round_burst + ((size_t)2 * j + t) * nb, cm.a[j].burst, nb * sizeof(float),
                          cudaMemcpyDeviceToHost, stream);
    }
    cudaEventRecord(ev_host, stream);
    t_host = host_clock();
    if (!wait_host_event("round chroma track detect")) return false;
    host_phase(kHostChromaWait, t_host);
    for (int j = 0; j < L; j++) cm.a[j].fields = ps[live[j]].res.fields;
  }
  for (int j = 0; j < L; j++) {
    const PortionState& st = *ps[live[j]].st;
    if (st.chroma_valid) {
      det[j] = st.chroma_track;
      thr[j] = st.chroma_threshold;
      cyc[j] = st.chroma_cycle_start;
    } else {
      const float* b0 = hp_round_burst + (size_t)2 * j * nb;
      const double m0 = host_burst_metric(b0, H, fmt.burst_len), m1 = host_burst_metric(b0 + nb, H, fmt.burst_len);
      det[j] = (m1 < m0) ? 1 : 0;
      thr[j] = (det[j] ? m1 : m0) * 4.0;
      const double ph = host_burst_phase(b0 + det[j] * nb, H, fmt);
      const int quadrant = ((int)(ph / 90.0 + 0.5)) % 4;
      const int pid = phase_id_for(1, quadrant);
      cyc[j] = 0;
      for (int i = 0; i < 8; i += 2)
        if (kPhaseCycle[i] == pid) {
          cyc[j] = i;
          break;
        }
    }
    cur[j] = det[j];
    const Portion& p = ps[live[j]];
    for (int f = 0; f < p.res.fields; f++) hp_track[p.slot0 + f] = (f & 1) ? (1 - cur[j]) : cur[j];
  }
  cudaMemcpyAsync(d_track, hp_track, (size_t)slots * sizeof(int), cudaMemcpyHostToDevice, stream);
  {
    cudaEvent_t ev_;
    begin_stage(kStageChromaLines, ev_);
    launch_chroma_lines_many(cm, L, -1, max_P, true, stream);
    end_stage(kStageChromaLines, ev_);
    begin_stage(kStageBurstMetric, ev_);
    launch_burst_metric_many(cm, L, max_P, stream);
    end_stage(kStageBurstMetric, ev_);
    begin_stage(kStageDropouts, ev_);
    launch_dropout_conceal_chroma_many(om, L, max_P, stream);
    end_stage(kStageDropouts, ev_);
  }
  cudaEventRecord(ev_host, stream);
  t_host = host_clock();
  if (!wait_host_event("round chroma lines")) return false;
  host_phase(kHostChromaWait, t_host);
  // Per capture, the reference's 15-field groups with up to three retries
  // each (chroma_decode.cu:782-981), recomputing only fields a flip changed.
  // The captures advance in lockstep: each runs its host decisions until it
  // needs a group recomputed, then one launch set over all captures waiting
  // on a recompute (each on a view of its group's fields) and one wait serve
  // them together.
  const int fpc_cap = std::max(1, 4096 / H);
  struct Replay {
    int P = 0, fpc = 1, g = 0, it = 0;  // group, iteration within it
    bool done = true;
    std::vector<int> computed;
  };
  std::vector<Replay> rp(L);
  for (int j = 0; j < L; j++) {
    const Portion& p = ps[live[j]];
    Replay& r = rp[j];
    r.P = p.res.fields;
    r.done = r.P == 0;
    r.fpc = std::max(1, std::min(fpc_cap, std::max(r.P, 1)));
    r.computed.assign(hp_track + p.slot0, hp_track + p.slot0 + r.P);
  }
  std::vector<int> need;
  for (;;) {
    need.clear();
    for (int j = 0; j < L; j++) {
      Replay& r = rp[j];
      const Portion& p = ps[live[j]];
      int* track = hp_track + p.slot0;
      const double* metric = hp_metric + p.slot0;
      while (!r.done) {
        const int f0 = r.g * r.fpc, nf = std::min(r.fpc, r.P - f0);
        bool stale = false;
        for (int f = f0; f < f0 + nf; f++) stale = stale || r.computed[f] != track[f];
        if (stale) {
          need.push_back(j);  // recompute, then decide on the new metrics
          break;
        }
        int first_bad = INT_MAX;
        for (int f = 0; f < nf; f++)
          if (metric[f0 + f] > thr[j]) {
            first_bad = f;
            break;
          }
        bool next_group = first_bad == INT_MAX;
        if (!next_group) {
          cur[j] = 1 - cur[j];
          for (int ff = f0 + first_bad; ff < r.P; ff++) track[ff] = (ff & 1) ? (1 - cur[j]) : cur[j];
          next_group = ++r.it == 3;
        }
        if (next_group) {
          r.g++;
          r.it = 0;
          if (r.g * r.fpc >= r.P) r.done = true;
        }
      }
    }
    if (need.empty()) break;
    static thread_local ArgsMany<ChromaArgs> cv;
    static thread_local ArgsMany<DropoutArgs> ov;
    int max_nf = 0;
    for (size_t q = 0; q < need.size(); q++) {
      const int j = need[q];
      const Replay& r = rp[j];
      const int f0 = r.g * r.fpc, nf = std::min(r.fpc, r.P - f0);
      max_nf = std::max(max_nf, nf);
      const int s0 = ps[live[j]].slot0;
      cudaMemcpyAsync(d_track + s0 + f0, hp_track + s0 + f0, nf * sizeof(int), cudaMemcpyHostToDevice, stream);
      // the capture's fields [f0, f0 + nf) as a capture of nf fields
      ChromaArgs c = cm.a[j];
      c.ll += (size_t)f0 * LPF;
      c.track += f0;
      c.chroma += (size_t)f0 * F;
      c.burst += (size_t)f0 * H * fmt.burst_len;
      c.metric += f0;
      c.fields = nf;
      cv.a[q] = c;
      DropoutArgs o = om.a[j];
      o.ll += (size_t)f0 * LPF;
      o.luma += (size_t)f0 * F;
      o.chroma += (size_t)f0 * F;
      o.do_count += f0;
      o.do_lines += (size_t)f0 * kMaxDropouts;
      o.do_starts += (size_t)f0 * kMaxDropouts;
      o.do_ends += (size_t)f0 * kMaxDropouts;
      o.cls += (size_t)f0 * o.max_blocks;
      o.fields = nf;
      ov.a[q] = o;
    }
    const int nq = (int)need.size();
    cudaEvent_t ev_;
    begin_stage(kStageChromaLines, ev_);
    launch_chroma_lines_many(cv, nq, -1, max_nf, true, stream);
    end_stage(kStageChromaLines, ev_);
    begin_stage(kStageBurstMetric, ev_);
    launch_burst_metric_many(cv, nq, max_nf, stream);
    end_stage(kStageBurstMetric, ev_);
    begin_stage(kStageDropouts, ev_);
    launch_dropout_conceal_chroma_many(ov, nq, max_nf, stream);
    end_stage(kStageDropouts, ev_);
    cudaEventRecord(ev_host, stream);
    if (!wait_host_event("round chroma retry")) return false;
    for (int j : need) {
      Replay& r = rp[j];
      const int f0 = r.g * r.fpc, nf = std::min(r.fpc, r.P - f0);
      const int* track = hp_track + ps[live[j]].slot0;
      for (int f = f0; f < f0 + nf; f++) r.computed[f] = track[f];
    }
  }
  // chroma planes out
  cudaEventRecord(ev_chroma, stream);
  cudaStreamWaitEvent(ostream, ev_chroma, 0);
  for (int j = 0; j < L; j++) {
    const Portion& p = ps[live[j]];
    if (p.dst_chroma && p.res.fields > 0)
      cudaMemcpyAsync(p.dst_chroma, cm.a[j].chroma, (size_t)p.res.fields * F * sizeof(uint16_t),
                      cudaMemcpyDeviceToHost, ostream);
  }
  cudaEventRecord(ev_out_done[oset], ostream);
  // carried line-location states back
  cudaMemcpyAsync(hp_lls, d_lls, (size_t)L * sizeof(LineLocState), cudaMemcpyDeviceToHost, stream);
  t_host = host_clock();
  if (cudaStreamSynchronize(stream) != cudaSuccess || cudaEventSynchronize(ev_small) != cudaSuccess)
    return check_cuda("round decode");
  out_set = 1 - oset;
  drain.keep_copies = true;
  collect_stage_times();
  ev_t0 = nullptr;
  pool_used = 0;
  if (!check_cuda("round decode")) return false;
  host_phase(kHostFinalWait, t_host);
  // ---- per capture: carried state and field metadata (parity alternation,
  // pipeline.cu:2575-2610)
  for (int j = 0; j < L; j++) {
    Portion& p = ps[live[j]];
    PortionState& st = *p.st;
    const int P = p.res.fields;
    st.lls = hp_lls[j];
    if (P > 0) {
      st.chroma_valid = true;
      st.chroma_track = (P & 1) ? (1 - cur[j]) : cur[j];
      st.chroma_threshold = thr[j];
      st.chroma_cycle_start = (cyc[j] + P) % 8;
    }
    p.res.field_info.resize(P);
    p.res.outputs_copied = p.dst_luma != nullptr || p.dst_chroma != nullptr;
    for (int i = 0; i < P; i++) {
      cuvhs_field_info& fi = p.res.field_info[i];
      const int s = p.slot0 + i;
      fi.file_loc = p.raw_offset + (uint64_t)hp_offs[s];
      bool first;
      if (hp_is_first[s] >= 0 && (hp_is_first[s] == 1) != st.last_parity) first = (hp_is_first[s] == 1);
      else first = !st.last_parity;
      st.last_parity = first;
      fi.is_first_field = first ? 1 : 0;
      fi.field_phase_id = kPhaseCycle[(cyc[j] + i) % 8];
      fi.dropout_count = std::max(0, std::min(hp_do_count[s], kMaxDropouts));
      fi.dropout_offset = 0;
    }
  }
  return true;
}

}  // namespace cuvhs
