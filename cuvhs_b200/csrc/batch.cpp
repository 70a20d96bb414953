// Batched decoding of many independent captures (extern "C" cuvhs_batch_*).
//
// The reference decodes one capture per process (src/main.cpp:97-165).  Here
// the captures of one sample rate are decoded in rounds (Context::decode_round,
// round.cpp): each round takes the next chunk of up to kMaxPortions captures,
// chunk size max_fields as a single-capture decode would use, and runs every
// stage once over all of them.  `lanes` host threads each drive rounds on
// their own contexts (one per sample rate, kept between calls) over their share
// of the captures, so one lane's host decisions overlap another's kernels.
// The field slots of a round come from an online autotuner: a rate's first
// rounds run at max_fields slots and double while the time per decoded field
// falls by more than 5%; the fastest size is kept for the rest of the decode
// and later calls (round_fields fixes it instead).  Rounds of any size decode
// the same chunks, so tuning on the caller's captures changes no output.
// Each capture starts from a fresh state and keeps its own carried state
// between rounds, so its output is its single-capture decode's whatever the
// lanes, round size or item order.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cuvhs.h"
#include "pipeline.h"

// Round sizes the tuner tries: max_fields times 1, 2, 4 (the context holds the largest).
constexpr int kTuneMaxFactor = 4;

struct cuvhs_batch {
  cuvhs_batch_config cfg{};
  int device = 0;
  int lanes = 1;
  // lane -> (rate -> context); a context's field slots are the rate's round size
  std::vector<std::map<double, cuvhs_ctx*>> ctx;
  std::map<double, int> round_fields;  // per rate, tuned or given
  bool timing = false;                 // per-stage device times on every context
  std::mutex mu;
  std::string err;
  ~cuvhs_batch() {
    for (auto& m : ctx)
      for (auto& kv : m) cuvhs_destroy(kv.second);
  }
};

namespace cuvhs {
// Creates a decoder context (cabi.cpp).
cuvhs_status create_context(const cuvhs_config& cfg, cuvhs_ctx** out);
}  // namespace cuvhs

namespace {

using cuvhs::ChunkResult;
using cuvhs::Context;
using cuvhs::Portion;
using cuvhs::PortionState;

// Online round-size tuning of one lane: the current size, the best so far and
// its time per field, and whether the search has ended.
struct Tuner {
  int slots = 0, best = 0, cap = 0;
  double best_spf = 0.0;
  bool settled = false;
  // after a round of `fields` fields in `secs` seconds at `slots` slots
  void observe(int fields, double secs, int round_slots_used) {
    if (settled || fields <= 0) return;
    const double spf = secs / fields;
    if (best == 0 || spf < best_spf * 0.95) {
      best = slots;
      best_spf = spf;
      // grow only while rounds fill their slots (a partial round says nothing
      // about a larger one)
      if (slots * 2 <= cap && round_slots_used * 2 > slots) slots *= 2;
      else settled = true;
    } else {
      slots = best;
      settled = true;
    }
  }
};

// One capture being decoded: its item, carried state and position.
struct Capture {
  cuvhs_batch_item* item = nullptr;
  PortionState st;
  uint64_t raw = 0;
  bool done = false;
};

cuvhs_status make_context(cuvhs_batch* b, double mhz, int slots, cuvhs_ctx** out) {
  cuvhs_config cc;
  cuvhs_default_config(&cc);
  cc.sample_rate_mhz = mhz;
  cc.device = b->device;
  cc.batch_fields = slots;
  return cuvhs::create_context(cc, out);
}

void set_err(cuvhs_batch* b, const std::string& e) {
  std::lock_guard<std::mutex> g(b->mu);
  if (b->err.empty()) b->err = e;
}

// Appends one decoded chunk of a capture to its output (cabi.cpp's
// append_chunk for a round portion): planes already copied, dropout lists
// from the round's slots.
cuvhs_status append_portion(Context& c, const Portion& p, cuvhs_output* out, std::string& err) {
  const ChunkResult& r = p.res;
  size_t need = 0;
  for (int i = 0; i < r.fields; i++) need += (size_t)r.field_info[i].dropout_count;
  if (out->dropouts_out + need > out->max_dropouts && need > 0) {
    err = "output dropout buffer too small";
    return CUVHS_ERR_CAPACITY;
  }
  for (int i = 0; i < r.fields; i++) {
    cuvhs_field_info fi = r.field_info[i];
    fi.dropout_offset = (int32_t)out->dropouts_out;
    for (int d = 0; d < fi.dropout_count; d++) {
      const size_t k = ((size_t)p.slot0 + i) * cuvhs::kMaxDropouts + d;
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

// Where a capture stands between rounds: its next chunk's start, whether it
// has ended, and its output fields so far.
struct Stand {
  uint64_t raw;
  bool done;
  size_t fields_out;
};

// The next round from the captures' standings: in order, each capture's next
// chunk (max_fields fields or what remains) while the slots last.  Captures
// that have ended or whose output has no room are skipped (`full` lists the
// latter).  Pure: the same standings give the same round.
void plan_round(const std::vector<Capture>& caps, const std::vector<Stand>& st, int max_fields, int slots,
                size_t spf, size_t F, std::vector<Portion>& ps, std::vector<int>& idx, std::vector<int>* full) {
  ps.clear();
  idx.clear();
  int used = 0;
  for (int i = 0; i < (int)caps.size() && (int)ps.size() < cuvhs::kMaxPortions; i++) {
    if (st[i].done) continue;
    const cuvhs_batch_item& it = *caps[i].item;
    const size_t n = it.n;
    const uint64_t raw = st[i].raw;
    const int remaining = raw < n ? (int)((n - raw) / spf) : 0;
    if (remaining <= 0) continue;
    const int nf = std::min(max_fields, remaining);
    if (used + nf > slots) break;  // the round is full
    const cuvhs_output* out = it.out;
    const size_t most = std::min<size_t>((size_t)nf, (n - raw) / spf);
    if (st[i].fields_out + most > out->max_fields) {
      if (full) full->push_back(i);
      continue;
    }
    Portion p;
    p.src = it.samples + raw;
    p.n_avail = n - raw;
    p.raw_offset = raw;
    p.num_fields = nf;
    p.slot0 = used;
    p.st = const_cast<PortionState*>(&caps[i].st);
    p.dst_luma = out->luma ? out->luma + st[i].fields_out * F : nullptr;
    p.dst_chroma = out->chroma ? out->chroma + st[i].fields_out * F : nullptr;
    ps.push_back(p);
    idx.push_back(i);
    used += nf;
  }
}

// Decodes `caps` (one sample rate) in rounds on context `ctx`, chunk size
// max_fields, tune.slots field slots per round (the tuner may grow them).
// Once a round knows where its captures' next chunks start (after its field
// windows), the next round is planned from the standings it will leave and
// its input windows are copied in while the round finishes.
void run_rounds(cuvhs_batch* b, cuvhs_ctx* ctx, std::vector<Capture>& caps, int max_fields, Tuner& tune) {
  Context& c = ctx->c;
  const size_t spf = (size_t)c.fmt.samples_per_field;
  const size_t F = (size_t)c.fmt.output_line_len * c.fmt.output_field_lines;
  std::vector<Portion> ps;
  std::vector<int> idx, full;
  std::vector<Stand> st(caps.size());
  auto standings = [&]() {
    for (size_t i = 0; i < caps.size(); i++) st[i] = Stand{caps[i].raw, caps[i].done, caps[i].item->out->fields_out};
  };
  for (;;) {
    standings();
    full.clear();
    plan_round(caps, st, max_fields, tune.slots, spf, F, ps, idx, &full);
    for (int i : full) {
      caps[i].item->status = CUVHS_ERR_CAPACITY;
      set_err(b, "output field buffer too small");
      caps[i].done = true;
    }
    if (!full.empty()) continue;  // plan again without them
    for (Capture& cp : caps)
      if (!cp.done && (cp.raw >= cp.item->n || (cp.item->n - cp.raw) / spf == 0)) cp.done = true;
    const int used = ps.empty() ? 0 : ps.back().slot0 + ps.back().num_fields;
    if (ps.empty()) {
      c.drain_copies();  // the last rounds' planes are in the callers' buffers
      return;
    }
    c.status = CUVHS_OK;
    // the next round from the standings this one leaves (the tuner's size
    // after this round may differ: then the prefetch is not used)
    auto next_plan = [&](const std::vector<Portion>& cur, std::vector<Portion>& next) {
      std::vector<Stand> after = st;
      for (size_t j = 0; j < cur.size(); j++) {
        Stand& s2 = after[idx[j]];
        if (cur[j].res.fields == 0) s2.done = true;
        else {
          s2.raw = cur[j].res.next_raw_offset;
          s2.fields_out += (size_t)cur[j].res.fields;
        }
      }
      std::vector<int> nidx;
      plan_round(caps, after, max_fields, tune.slots, spf, F, next, nidx, nullptr);
    };
    const auto t0 = std::chrono::steady_clock::now();
    const bool ok = c.decode_round(ps, next_plan);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (ok) {
      int fields = 0;
      for (const Portion& p : ps) fields += p.res.fields;
      tune.observe(fields, secs, used);
    }
    if (!ok) {
      const cuvhs_status s = c.status != CUVHS_OK ? c.status : CUVHS_ERR_CUDA;
      set_err(b, c.err);
      for (int i : idx) {
        caps[i].item->status = s;
        caps[i].done = true;
      }
      continue;
    }
    for (size_t j = 0; j < ps.size(); j++) {
      Capture& cp = caps[idx[j]];
      const Portion& p = ps[j];
      if (p.res.fields == 0) {
        cp.done = true;  // the chunk held no field: end of capture
        continue;
      }
      std::string e;
      const cuvhs_status s = append_portion(c, p, cp.item->out, e);
      if (s != CUVHS_OK) {
        cp.item->status = s;
        set_err(b, e);
        cp.done = true;
        continue;
      }
      cp.raw = p.res.next_raw_offset;
    }
  }
}

}  // namespace

extern "C" {

cuvhs_status cuvhs_batch_create(const cuvhs_batch_config* cfg, cuvhs_batch** out) {
  if (!cfg || !out) return CUVHS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (cfg->lanes < 0 || cfg->max_fields < 0 || cfg->round_fields < 0) return CUVHS_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    fprintf(stderr, "cuvhs_batch_create: no CUDA device\n");
    return CUVHS_ERR_CUDA;
  }
  cuvhs_batch* b = new (std::nothrow) cuvhs_batch();
  if (!b) return CUVHS_ERR_OUT_OF_MEMORY;
  b->cfg = *cfg;
  if (b->cfg.max_fields == 0) b->cfg.max_fields = 256;
  if (b->cfg.round_fields > 0 && b->cfg.round_fields < b->cfg.max_fields) {
    delete b;
    return CUVHS_ERR_INVALID_ARGUMENT;
  }
  int dev = cfg->device;
  if (dev < 0) {
    size_t best = 0;
    dev = 0;
    for (int d = 0; d < ndev; d++) {
      cudaDeviceProp p;
      if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.totalGlobalMem > best) {
        best = p.totalGlobalMem;
        dev = d;
      }
    }
  }
  if (dev >= ndev) {
    delete b;
    return CUVHS_ERR_INVALID_ARGUMENT;
  }
  b->device = dev;
  b->lanes = cfg->lanes > 0 ? cfg->lanes : 4;
  b->ctx.resize(b->lanes);
  *out = b;
  return CUVHS_OK;
}

void cuvhs_batch_destroy(cuvhs_batch* b) { delete b; }

int cuvhs_batch_lanes(const cuvhs_batch* b) { return b ? b->lanes : 0; }

const char* cuvhs_batch_last_error(const cuvhs_batch* b) { return b ? b->err.c_str() : "null batch"; }

void cuvhs_batch_set_timing(cuvhs_batch* b, int on) {
  if (!b) return;
  b->timing = on != 0;
  for (auto& m : b->ctx)
    for (auto& kv : m) cuvhs_set_timing(kv.second, on);
}

int cuvhs_batch_stage_times(const cuvhs_batch* b, double* ms, long long* launches, int cap) {
  if (!b) return 0;
  const int n = std::min(cap, (int)cuvhs::kNumStages);
  for (int i = 0; i < n; i++) {
    if (ms) ms[i] = 0.0;
    if (launches) launches[i] = 0;
  }
  std::vector<double> t(cuvhs::kNumStages);
  std::vector<long long> l(cuvhs::kNumStages);
  for (auto& m : b->ctx)
    for (auto& kv : m) {
      cuvhs_stage_times(kv.second, t.data(), l.data(), cuvhs::kNumStages);
      for (int i = 0; i < n; i++) {
        if (ms) ms[i] += t[i];
        if (launches) launches[i] += l[i];
      }
    }
  return cuvhs::kNumStages;
}

int cuvhs_batch_round_fields(const cuvhs_batch* b, double sample_rate_mhz) {
  if (!b) return 0;
  auto it = b->round_fields.find(sample_rate_mhz);
  return it == b->round_fields.end() ? 0 : it->second;
}

long long cuvhs_batch_json(const cuvhs_batch_item* item, char* dst, long long cap) {
  if (!item || !item->out) return -1;
  cuvhs::Format fmt;
  fmt.init(item->sample_rate_mhz);
  const cuvhs_output* o = item->out;
  const std::string s = cuvhs::tbc_json(fmt, o->fields, o->fields_out, o->dropout_line, o->dropout_startx,
                                        o->dropout_endx);
  if (dst && cap > 0) {
    const size_t n = std::min<size_t>((size_t)cap - 1, s.size());
    std::memcpy(dst, s.data(), n);
    dst[n] = 0;
  }
  return (long long)s.size();
}

cuvhs_status cuvhs_batch_decode(cuvhs_batch* b, cuvhs_batch_item* items, int n_items) {
  if (!b || (!items && n_items > 0) || n_items < 0) return CUVHS_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < n_items; i++) {
    if (!items[i].samples || !items[i].out || !(items[i].sample_rate_mhz > 0.0)) return CUVHS_ERR_INVALID_ARGUMENT;
    items[i].status = CUVHS_OK;
  }
  b->err.clear();
  cudaSetDevice(b->device);
  const int max_fields = b->cfg.max_fields;
  // per rate: the captures, longest first, dealt to the lanes in turn
  std::map<double, std::vector<int>> by_rate;
  for (int i = 0; i < n_items; i++) by_rate[items[i].sample_rate_mhz].push_back(i);
  struct Job {
    double mhz;
    std::vector<int> items;
  };
  std::vector<std::vector<Job>> jobs(b->lanes);
  for (auto& kv : by_rate) {
    std::vector<int>& v = kv.second;
    std::stable_sort(v.begin(), v.end(), [&](int x, int y) { return items[x].n > items[y].n; });
    std::vector<Job> per(b->lanes);
    for (size_t k = 0; k < v.size(); k++) per[k % b->lanes].items.push_back(v[k]);
    for (int l = 0; l < b->lanes; l++)
      if (!per[l].items.empty()) jobs[l].push_back(Job{kv.first, per[l].items});
  }
  auto lane_fn = [&](int lane) {
    cudaSetDevice(b->device);
    for (Job& job : jobs[lane]) {
      // the round size: given, tuned by an earlier call, or tuned on these rounds
      Tuner tune;
      int known = 0;
      {
        std::lock_guard<std::mutex> g(b->mu);
        auto it = b->round_fields.find(job.mhz);
        if (it != b->round_fields.end()) known = it->second;
      }
      if (b->cfg.round_fields > 0) known = b->cfg.round_fields;
      // no round needs more slots than one chunk of every capture of the job
      cuvhs::Format fmt;
      fmt.init(job.mhz);
      long long need = 0;
      for (int i : job.items)
        need += std::min<long long>(max_fields, (long long)(items[i].n / (size_t)fmt.samples_per_field));
      const int cap = (int)std::max<long long>(
          max_fields, std::min<long long>(need, known > 0 ? known : (long long)max_fields * kTuneMaxFactor));
      cuvhs_ctx*& ctx = b->ctx[lane][job.mhz];
      if (ctx && cuvhs_batch_fields(ctx) < cap) {
        cuvhs_destroy(ctx);
        ctx = nullptr;
      }
      if (!ctx) {
        // a context too large for the free memory halves down to one chunk
        cuvhs_status s = CUVHS_ERR_OUT_OF_MEMORY;
        for (int sl = cap; sl >= max_fields; sl /= 2) {
          s = make_context(b, job.mhz, sl, &ctx);
          if (s == CUVHS_OK) break;
          ctx = nullptr;
          if (s != CUVHS_ERR_OUT_OF_MEMORY) break;
        }
        if (s != CUVHS_OK) {
          ctx = nullptr;
          for (int i : job.items) items[i].status = s;
          set_err(b, "context creation failed");
          continue;
        }
        cuvhs_set_timing(ctx, b->timing ? 1 : 0);
      }
      tune.cap = std::min(cap, cuvhs_batch_fields(ctx));
      if (known > 0) {
        tune.slots = tune.best = std::min(known, tune.cap);
        tune.settled = true;
      } else {
        tune.slots = max_fields;
      }
      std::vector<Capture> caps(job.items.size());
      for (size_t k = 0; k < job.items.size(); k++) {
        cuvhs_batch_item& it = items[job.items[k]];
        it.out->fields_out = 0;
        it.out->dropouts_out = 0;
        caps[k].item = &it;
      }
      run_rounds(b, ctx, caps, max_fields, tune);
      {
        std::lock_guard<std::mutex> g(b->mu);
        int& rf = b->round_fields[job.mhz];
        if (b->cfg.round_fields > 0) rf = b->cfg.round_fields;
        else if (tune.best > 0) rf = std::max(rf, tune.best);
      }
    }
  };
  std::vector<std::thread> th;
  for (int l = 1; l < b->lanes; l++) th.emplace_back(lane_fn, l);
  lane_fn(0);
  for (auto& t : th) t.join();
  for (int i = 0; i < n_items; i++)
    if (items[i].status != CUVHS_OK) return items[i].status;
  return CUVHS_OK;
}

}  // extern "C"
