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
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/cuvhs.h"
#include "cuvhs_internal.h"

namespace cuvhs {
namespace {

constexpr int kPartialSamples = 4096;  // envelope samples per partial sum
constexpr int kPartialThreads = 256;
constexpr int kMaxDevices = 64;

// The scratch: every call on a device shares it and it keeps the last call's
// contents.  Each call writes every entry it reads before reading it, so
// nothing has to start at zero.  Calls that overlap on the GPU (two streams,
// or two host threads) race on it.
static __device__ __align__(256) double g_env_partials[CUVHS_NOALLOC_MAX_PARTIALS];

std::mutex g_setup_mutex;
double* g_partials_addr[kMaxDevices] = {};  // device address of the array, per device

__global__ void __launch_bounds__(kPartialThreads) env_partials_kernel(const float* __restrict__ env, int spp,
                                                                      int per_tile, double* __restrict__ out) {
  __shared__ double red[kPartialThreads / 32];
  const int f = blockIdx.y, b = blockIdx.x;
  const long long start = (long long)f * spp + (long long)b * kPartialSamples;
  const long long end = min(start + kPartialSamples, (long long)(f + 1) * spp);
  double s = 0.0;
  for (long long i = start + threadIdx.x; i < end; i += kPartialThreads) s += (double)__ldg(&env[i]);
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kPartialThreads / 32; w++) t += red[w];
    out[(size_t)f * per_tile + b] = t;
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
      fields < 1 || tile_stride < 1)
    return CUVHS_ERR_INVALID_ARGUMENT;
  const long long per_tile = ((long long)tile_stride + kPartialSamples - 1) / kPartialSamples;
  if (dropout_class_bytes_per_field(tile_stride) > 200 * 1024) {  // the per-field classes live in shared memory
    fprintf(stderr, "cuvhs_dropouts_noalloc: tile_stride %d is above the %d samples one call handles\n",
            tile_stride, 200 * 1024 * 16);
    return CUVHS_ERR_CAPACITY;
  }
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
    // Set-up, once per device with that device current: the array's name is a
    // host-side stand-in, so look up its device address.
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_env_partials);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        fprintf(stderr, "cuvhs_dropouts_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return CUVHS_ERR_CUDA;
      }
      g_partials_addr[dev] = static_cast<double*>(p);
    }
    partials = g_partials_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dim3 grid((unsigned)per_tile, (unsigned)fields);
  env_partials_kernel<<<grid, kPartialThreads, 0, st>>>(d_envelope, tile_stride, (int)per_tile, partials);
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
  launch_dropouts(a, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "cuvhs_dropouts_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return CUVHS_ERR_CUDA;
  }
  return CUVHS_OK;
}
