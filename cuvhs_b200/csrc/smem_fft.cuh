// Shared-memory FP32 complex FFT for one CTA (sm_100a).
//
// Stockham auto-sort, radix-16 passes (plus one radix-2/4/8 pass for sizes that
// are not a power of 16).  Each thread holds its butterflies' inputs in
// registers, so one padded buffer serves as both source and destination of a
// pass (read all -> barrier -> write all -> barrier).  Index i lives at i + i/16
// so the stride-16 writes of the first pass do not collide on banks.
// Twiddles come from a per-pass table computed in FP64 on the host and
// rounded once to FP32: pass NS (>= 16) stores W_{NS*R}^{r*k} at
// (NS - 16) + (r - 1) * NS + k, so a warp's twiddle loads (consecutive k) are
// contiguous.  fft_twiddle_count(N) entries in all.
#pragma once
#include <cuda_runtime.h>

namespace cuvhs {

__host__ __device__ constexpr int fft_pad(int n) { return n + (n >> 4); }

// The thread index as a value the compiler cannot prove equal to its source.
// Two transforms in one kernel compute the same shared-memory and twiddle
// offsets; given the plain index the compiler keeps the first transform's
// offsets live until the second uses them, which spills the transforms' data.
__device__ __forceinline__ int opaque_index(int t) {
  int r;
  asm volatile("mov.u32 %0, %1;" : "=r"(r) : "r"(t));
  return r;
}

// Radix of the pass that starts at span NS in an N-point transform.
__host__ __device__ constexpr int fft_radix(int N, int NS) { return NS * 16 <= N ? 16 : N / NS; }
// Entries of the per-pass twiddle table of an N-point transform.
__host__ __device__ constexpr int fft_twiddle_count(int N) {
  int n = 0;
  for (int ns = 16; ns < N; ns *= 16) n += (fft_radix(N, ns) - 1) * ns;
  return n;
}
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }

template <bool INV>
__device__ __forceinline__ float2 cmul_tw(float2 a, float2 w) {
  // a * w (forward) or a * conj(w) (inverse)
  if (INV) return make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
  return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// multiply by -i (forward) / +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// e^{-+2 pi i m / 16} constants
struct Root16 {
  static constexpr float c[16] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
                                  0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f,
                                  -1.0f, -0.92387953251128674f, -0.70710678118654752f, -0.38268343236508977f,
                                  0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f};
  static constexpr float s[16] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f,
                                  1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
                                  0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f,
                                  -1.0f, -0.92387953251128674f, -0.70710678118654752f, -0.38268343236508977f};
};

// v * W_R^m with R | 16 (m in units of 1/R turn)
template <int R, int M, bool INV>
__device__ __forceinline__ float2 rot(float2 v) {
  constexpr int m16 = (M * (16 / R)) & 15;
  if (m16 == 0) return v;
  if (m16 == 4) return mul_mi<INV>(v);
  if (m16 == 8) return make_float2(-v.x, -v.y);
  if (m16 == 12) return mul_mi<!INV>(v);
  const float c = Root16::c[m16];
  const float s = INV ? Root16::s[m16] : -Root16::s[m16];
  return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
}

template <bool INV>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
  float2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_mi<INV>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

// In-register DFT of size R, in place.  Output bin r ends up in v[dft_slot<R>(r)]
// (a compile-time permutation, free once the loops are unrolled).
template <int R>
__host__ __device__ constexpr int dft_slot(int r) {
  return R == 16 ? 4 * (r & 3) + (r >> 2) : (R == 8 ? 2 * (r & 3) + (r >> 2) : r);
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 2) {
    dft2<INV>(v[0], v[1]);
  } else if constexpr (R == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    // 8 = 4 (n1) x 2 (n2): x[2 n1 + n2]; bin k1 + 4 k2 lands in v[2 k1 + k2]
    dft4<INV>(v[0], v[2], v[4], v[6]);
    dft4<INV>(v[1], v[3], v[5], v[7]);
    v[3] = rot<8, 1, INV>(v[3]);
    v[5] = rot<8, 2, INV>(v[5]);
    v[7] = rot<8, 3, INV>(v[7]);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) dft2<INV>(v[2 * k1], v[2 * k1 + 1]);
  } else if constexpr (R == 16) {
    // 16 = 4 (n1) x 4 (n2): x[4 n1 + n2]; A[n2][k1] in v[4 k1 + n2];
    // bin k1 + 4 k2 lands in v[4 k1 + k2]
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) dft4<INV>(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
    v[4 + 1] = rot<16, 1, INV>(v[4 + 1]);
    v[4 + 2] = rot<16, 2, INV>(v[4 + 2]);
    v[4 + 3] = rot<16, 3, INV>(v[4 + 3]);
    v[8 + 1] = rot<16, 2, INV>(v[8 + 1]);
    v[8 + 2] = rot<16, 4, INV>(v[8 + 2]);
    v[8 + 3] = rot<16, 6, INV>(v[8 + 3]);
    v[12 + 1] = rot<16, 3, INV>(v[12 + 1]);
    v[12 + 2] = rot<16, 6, INV>(v[12 + 2]);
    v[12 + 3] = rot<16, 9, INV>(v[12 + 3]);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) dft4<INV>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  }
}

template <int THREADS>
__device__ __forceinline__ void fft_sync() {
  if constexpr (THREADS == 32) {
    __syncwarp();
  } else if constexpr (THREADS == 64) {
    // two-warp transforms: threads [64 g, 64 g + 64) share barrier 1 + g.
    // Immediate barrier ids: with a register id the compiler reserves all 16
    // barriers per CTA, which caps residency at 4 CTAs per SM.
    const int g = threadIdx.x >> 6;
    if (g == 0) asm volatile("bar.sync 1, 64;" ::: "memory");
    else if (g == 1) asm volatile("bar.sync 2, 64;" ::: "memory");
    else if (g == 2) asm volatile("bar.sync 3, 64;" ::: "memory");
    else asm volatile("bar.sync 4, 64;" ::: "memory");
  } else {
    __syncthreads();
  }
}

// One Stockham pass of radix R on an N-point padded buffer, current span NS.
template <int N, int THREADS, int R, int NS, bool INV>
__device__ __forceinline__ void fft_pass(float2* s, const float2* __restrict__ tw, int tid) {
  constexpr int NB = N / R;
  constexpr int PER = (NB + THREADS - 1) / THREADS;
  float2 v[PER][R];
#pragma unroll
  for (int p = 0; p < PER; p++) {
    const int j = tid + p * THREADS;
    if ((NB % THREADS) == 0 || j < NB) {
#pragma unroll
      for (int r = 0; r < R; r++) v[p][r] = s[pidx(j + r * NB)];
      if constexpr (NS > 1) {
        const int k = j & (NS - 1);
        const float2* twp = tw + (NS - 16) + k;
#pragma unroll
        for (int r = 1; r < R; r++) v[p][r] = cmul_tw<INV>(v[p][r], __ldg(&twp[(r - 1) * NS]));
      }
      dft<R, INV>(v[p]);
    }
  }
  fft_sync<THREADS>();
#pragma unroll
  for (int p = 0; p < PER; p++) {
    const int j = tid + p * THREADS;
    if ((NB % THREADS) == 0 || j < NB) {
      const int k = j & (NS - 1);
      const int base = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) s[pidx(base + r * NS)] = v[p][dft_slot<R>(r)];
    }
  }
  fft_sync<THREADS>();
}

// Full N-point transform (N a power of two, 64 <= N <= 65536), natural order
// in and out, unnormalised.  THREADS is 32 (one warp), 64 (two warps of a
// CTA of up to 4 such groups, synchronised on named barriers) or the CTA.
// Caller must synchronise the transform's threads after filling s.  tid: this thread's index among the
// transform's THREADS threads (the lane for a one-warp transform).
template <int N, int THREADS, bool INV, int NS = 1>
__device__ __forceinline__ void smem_fft(float2* s, const float2* __restrict__ tw, int tid) {
  if constexpr (NS * 16 <= N) {
    fft_pass<N, THREADS, 16, NS, INV>(s, tw, tid);
    smem_fft<N, THREADS, INV, NS * 16>(s, tw, tid);
  } else if constexpr (NS < N) {
    constexpr int R = N / NS;  // 2, 4 or 8
    static_assert(R == 2 || R == 4 || R == 8, "N must be a power of two");
    fft_pass<N, THREADS, R, NS, INV>(s, tw, tid);
  }
}

}  // namespace cuvhs
