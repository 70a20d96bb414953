// Dropout detection and concealment on caller-owned device buffers, without
// allocating any device memory (cuvhs_dropouts_noalloc in include/cuvhs.h).
//
// Some callers cannot call cudaMalloc: code that runs while its stream is being
// captured into a CUDA graph (an allocation there is not part of the graph and
// breaks the capture), real-time capture loops that must never block inside
// the allocator, and hosts whose device memory is owned by another allocator.
// The decoder context allocates its scratch once at creation; this entry point
// instead keeps its only scratch -- per-block partial sums of the envelope,
// from which each field's tile mean (the dropout threshold) is formed -- in a
// file-scope device array of fixed size.  The detection and concealment kernel
// is the decoder's own (launch_dropouts).
//
// The partial sums are formed over the decoder's own K1a output blocks, in the
// order K1a forms them (each thread's samples in block order, a warp shuffle
// tree, then the warps in order), so the FP64 tile mean -- and every threshold
// decision that depends on it -- is bit-identical to the decoder's.  The block
// size follows from the capture rate, which is derived here from the NTSC tile
// stride (283 lines of round(fs / 15734.264) samples); for capture rates within
// one line-rate step of a K1a support boundary the derived block size can
// differ from the decoder's, and the mean can then differ in its last bit.
#include <cuda.h>  // CUcontext / CUresult for the driver entry points (no libcuda link)
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/cuvhs.h"
#include "cuvhs_internal.h"

namespace cuvhs {
namespace {

constexpr int kPartialThreads = Design::kNa / 16;  // K1a's CTA: 16 block positions per thread
constexpr int kNtscTileLines = 283;                // 263 field lines + 20 margin lines
constexpr double kNtscLineRate = 15734.264;
constexpr int kMaxDevices = 64;

// The scratch: every call on a device shares it and it keeps the last call's
// contents.  Each call writes every entry it reads before reading it, so
// nothing has to start at zero.  Calls that overlap on the GPU (two streams,
// or two host threads) race on it.
static __device__ __align__(256) double g_env_partials[CUVHS_NOALLOC_MAX_PARTIALS];

// Device address of the array, per device, with the id of the CUDA context it
// was looked up in: after cudaDeviceReset (or in another context) the module
// is loaded again and the array can move, so a new context id means a new
// lookup.  Context ids are unique for the life of the process.
struct Setup {
  unsigned long long ctx_id = 0;
  double* addr = nullptr;
};
std::mutex g_setup_mutex;
Setup g_setup[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the calling thread's current context (0 if there is none yet).
bool current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
  });
  if (!get_current || !get_id) return false;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return false;
  *id = 0;
  return !ctx || get_id(ctx, id) == CUDA_SUCCESS;
}

// Partial b of field f: the envelope of K1a block b of the field's slot,
// samples [b * a_out, b * a_out + nout), summed as K1a's emit step sums them.
__global__ void __launch_bounds__(kPartialThreads) env_partials_kernel(const float* __restrict__ env, int spp,
                                                                      int a_out, int a_lead, int per_tile,
                                                                      double* __restrict__ out) {
  __shared__ double red[kPartialThreads / 32];
  const int f = blockIdx.y, b = blockIdx.x, t = threadIdx.x;
  const float* e = env + ((long long)f * spp + (long long)b * a_out);
  const int nout = min(a_out, spp - b * a_out);
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < Design::kNa / kPartialThreads; q++) {
    const int i = t + kPartialThreads * q - a_lead;
    if (i >= 0 && i < nout) s += (double)__ldg(&e[i]);
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((t & 31) == 0) red[t >> 5] = s;
  __syncthreads();
  if (t == 0) {
    double acc = 0.0;
    for (int w = 0; w < kPartialThreads / 32; w++) acc += red[w];
    out[(size_t)f * per_tile + b] = acc;
  }
}

}  // namespace
}  // namespace cuvhs

extern "C" cuvhs_status cuvhs_dropouts_noalloc(const float* d_envelope, const double* d_linelocs, int fields,
                                               int tile_stride, uint16_t* d_luma, uint16_t* d_chroma,
                                               int32_t* d_count, int32_t* d_lines, int32_t* d_startx,
                                               int32_t* d_endx, void* stream) {
  using namespace cuvhs;
  if (!d_envelope || !d_linelocs || !d_luma || !d_chroma || !d_count || !d_lines || !d_startx || !d_endx ||
      fields < 1 || tile_stride < kNtscTileLines)
    return CUVHS_ERR_INVALID_ARGUMENT;
  // An error left by an earlier, unrelated call is the caller's: leave it
  // pending and do nothing.
  if (cudaPeekAtLastError() != cudaSuccess) {
    fprintf(stderr, "cuvhs_dropouts_noalloc: an earlier CUDA error is pending; nothing was launched\n");
    return CUVHS_ERR_CUDA;
  }
  if (dropout_class_bytes_per_field(tile_stride) > (size_t)kMaxClassBytes) {  // classes live in shared memory
    fprintf(stderr, "cuvhs_dropouts_noalloc: tile_stride %d is above the %d samples one call handles\n",
            tile_stride, kMaxClassBytes * 16);
    return CUVHS_ERR_CAPACITY;
  }
  // the decoder's K1a block geometry at the capture rate of this tile stride
  const double fs = (double)(tile_stride / kNtscTileLines) * kNtscLineRate;
  const int half = k1a_half_support(fs);
  const int a_out = Design::kNa - 2 * half - 1, a_lead = half + 1;
  const long long per_tile = ((long long)tile_stride + a_out - 1) / a_out;
  if ((long long)fields * per_tile > CUVHS_NOALLOC_MAX_PARTIALS) {
    fprintf(stderr,
            "cuvhs_dropouts_noalloc: %d fields of %d samples need %lld envelope partial sums; "
            "the fixed scratch holds %d (at most %lld fields of this size per call)\n",
            fields, tile_stride, (long long)fields * per_tile, CUVHS_NOALLOC_MAX_PARTIALS,
            CUVHS_NOALLOC_MAX_PARTIALS / per_tile);
    return CUVHS_ERR_CAPACITY;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return CUVHS_ERR_CUDA;
  }
  if (dev >= kMaxDevices) return CUVHS_ERR_UNSUPPORTED;
  double* partials = nullptr;
  {
    // Set-up, once per device and context, with that device current: the
    // array's name is a host-side stand-in, so look up its device address.
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long ctx = 0;
    const bool have_ctx = current_context_id(&ctx);
    Setup& s = g_setup[dev];
    if (!have_ctx || ctx == 0 || !s.addr || s.ctx_id != ctx) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_env_partials);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        fprintf(stderr, "cuvhs_dropouts_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        s = Setup();
        return CUVHS_ERR_CUDA;
      }
      // the lookup made the device's context current if there was none
      unsigned long long now = 0;
      s.addr = static_cast<double*>(p);
      s.ctx_id = current_context_id(&now) ? now : 0;  // 0: look it up again next call
    }
    partials = s.addr;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dim3 grid((unsigned)per_tile, (unsigned)fields);
  env_partials_kernel<<<grid, kPartialThreads, 0, st>>>(d_envelope, tile_stride, a_out, a_lead, (int)per_tile,
                                                         partials);
  cudaError_t e = cudaGetLastError();  // no earlier error was pending: this one is ours
  if (e == cudaSuccess) {
    DropoutArgs a;
    a.env = d_envelope;
    a.env_part = partials;
    a.env_blocks = (int)per_tile;
    a.ll = d_linelocs;
    a.fields = fields;
    a.spp = tile_stride;
    a.lines_per_frame = 525;
    a.active_line_start = 10;
    a.out_w = CUVHS_FIELD_WIDTH;
    a.out_h = CUVHS_FIELD_HEIGHT;
    a.luma = d_luma;
    a.chroma = d_chroma;
    a.do_count = d_count;
    a.do_lines = d_lines;
    a.do_starts = d_startx;
    a.do_ends = d_endx;
    a.max_blocks = (int)dropout_class_bytes_per_field(tile_stride);
    e = launch_dropouts(a, st);
    cudaGetLastError();  // the same error, returned above; clear it
  }
  if (e != cudaSuccess) {
    fprintf(stderr, "cuvhs_dropouts_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return CUVHS_ERR_CUDA;
  }
  return CUVHS_OK;
}
