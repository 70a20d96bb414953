// Batched decoding of many independent captures (extern "C" cuvhs_batch_*).
//
// The reference decodes one capture per process (src/main.cpp:97-165), so a
// set of captures runs back to back.  Here `lanes` host threads each own
// decoder contexts -- one per sample rate, created on first use and kept --
// and take captures from a shared queue, longest first.  Each lane's contexts
// have their own streams, so the GPU overlaps the kernels and copies of
// several captures while the lanes' host decisions (line locations, chroma
// track replay) run in parallel.  A capture is always decoded from a fresh
// state with a fixed chunk size, so its output is the single-capture decode's
// whatever the lane count or item order.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
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

struct cuvhs_batch {
  cuvhs_batch_config cfg{};
  int device = 0;
  int lanes = 1;
  // lane -> (rate -> context)
  std::vector<std::map<double, cuvhs_ctx*>> ctx;
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

extern "C" {

cuvhs_status cuvhs_batch_create(const cuvhs_batch_config* cfg, cuvhs_batch** out) {
  if (!cfg || !out) return CUVHS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (cfg->lanes < 0 || cfg->max_fields < 0) return CUVHS_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    fprintf(stderr, "cuvhs_batch_create: no CUDA device\n");
    return CUVHS_ERR_CUDA;
  }
  cuvhs_batch* b = new (std::nothrow) cuvhs_batch();
  if (!b) return CUVHS_ERR_OUT_OF_MEMORY;
  b->cfg = *cfg;
  if (b->cfg.max_fields == 0) b->cfg.max_fields = 256;
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
  const int hw = std::max(1, (int)std::thread::hardware_concurrency());
  b->lanes = cfg->lanes > 0 ? cfg->lanes : std::max(1, std::min(4, hw / 2));
  b->ctx.resize(b->lanes);
  *out = b;
  return CUVHS_OK;
}

void cuvhs_batch_destroy(cuvhs_batch* b) { delete b; }

int cuvhs_batch_lanes(const cuvhs_batch* b) { return b ? b->lanes : 0; }

const char* cuvhs_batch_last_error(const cuvhs_batch* b) { return b ? b->err.c_str() : "null batch"; }

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
    if (!items[i].samples || !items[i].out) return CUVHS_ERR_INVALID_ARGUMENT;
    items[i].status = CUVHS_OK;
  }
  // longest captures first, so the lanes finish together
  std::vector<int> order(n_items);
  for (int i = 0; i < n_items; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return items[x].n / items[x].sample_rate_mhz > items[y].n / items[y].sample_rate_mhz;
  });
  std::atomic<int> next{0};
  b->err.clear();
  auto lane_fn = [&](int lane) {
    cudaSetDevice(b->device);
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= n_items) break;
      cuvhs_batch_item& it = items[order[k]];
      cuvhs_ctx*& ctx = b->ctx[lane][it.sample_rate_mhz];
      if (!ctx) {
        cuvhs_config cc;
        cuvhs_default_config(&cc);
        cc.sample_rate_mhz = it.sample_rate_mhz;
        cc.device = b->device;
        cc.batch_fields = b->cfg.max_fields;
        cuvhs_status s = cuvhs::create_context(cc, &ctx);
        if (s != CUVHS_OK) {
          ctx = nullptr;
          it.status = s;
          std::lock_guard<std::mutex> g(b->mu);
          if (b->err.empty()) b->err = "context creation failed";
          continue;
        }
      }
      cuvhs_reset(ctx);
      it.out->fields_out = 0;
      it.out->dropouts_out = 0;
      it.status = cuvhs_decode_capture(ctx, it.samples, it.n, it.out);
      if (it.status != CUVHS_OK) {
        std::lock_guard<std::mutex> g(b->mu);
        if (b->err.empty()) b->err = cuvhs_last_error(ctx);
      }
    }
  };
  const int nl = std::min(b->lanes, std::max(1, n_items));
  std::vector<std::thread> th;
  for (int l = 1; l < nl; l++) th.emplace_back(lane_fn, l);
  lane_fn(0);
  for (auto& t : th) t.join();
  for (int i = 0; i < n_items; i++)
    if (items[i].status != CUVHS_OK) return items[i].status;
  return CUVHS_OK;
}

}  // extern "C"
