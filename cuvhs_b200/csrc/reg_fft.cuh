// Register-resident block FFT for one CTA of T = N/E threads (sm_100a), E = 16
// or 32 elements per thread.
//
// Thread t owns elements t + T*q, q = 0..E-1, of an N-point transform, both on
// entry (natural-order input) and on exit (natural-order output): Stockham
// passes of radix 16 (and one final radix 2/4/8 when N is not a power of 16)
// exchange data through a padded shared buffer between passes, but the first
// pass reads its inputs from registers and the last pass leaves its outputs in
// registers.  Since the output layout equals the input layout, a forward
// transform, a per-bin multiply and an inverse transform chain without any
// shared-memory round trip at the seams, and inputs/outputs move between HBM
// and registers with coalesced accesses (consecutive threads, consecutive
// elements).  Twiddles: the per-pass table of smem_fft.cuh (coalesced loads).
#pragma once
#include "smem_fft.cuh"

namespace cuvhs {

template <int N, int E = 16>
struct RegFFT {
  static_assert(E == 16 || E == 32, "16 or 32 elements per thread");
  static constexpr int T = N / E;
  static constexpr int G = E / 16;  // first-pass radix-16 butterflies per thread

  // One pass of radix R at span NS (> 1).  v holds the E values this thread
  // reads; LAST leaves the results in v in the t + T*q layout.
  template <int NS, bool INV, bool LAST>
  __device__ __forceinline__ static void pass(float2 (&v)[E], float2* s, const float2* __restrict__ tw, int t) {
    constexpr int R = fft_radix(N, NS);
    constexpr int B = E / R;  // butterflies per thread
    // inputs are twiddled as they are read, so only the E values stay live
    // across the barrier
    float2 w[B][R];
#pragma unroll
    for (int b = 0; b < B; b++) {
      const int j = t + T * b;
      const int k = j & (NS - 1);
      const float2* twp = tw + (NS - 16) + k;
      w[b][0] = s[pidx(j)];
#pragma unroll
      for (int r = 1; r < R; r++) w[b][r] = cmul_tw<INV>(s[pidx(j + r * (N / R))], __ldg(&twp[(r - 1) * NS]));
    }
    __syncthreads();  // every read done before this pass (or the caller) overwrites
#pragma unroll
    for (int b = 0; b < B; b++) dft<R, INV>(w[b]);
    if constexpr (LAST) {
#pragma unroll
      for (int b = 0; b < B; b++)
#pragma unroll
        for (int r = 0; r < R; r++) v[b + B * r] = w[b][dft_slot<R>(r)];
    } else {
#pragma unroll
      for (int b = 0; b < B; b++) {
        const int j = t + T * b;
        const int k = j & (NS - 1);
        const int base = (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) s[pidx(base + r * NS)] = w[b][dft_slot<R>(r)];
      }
      __syncthreads();
    }
  }

  template <int NS, bool INV>
  __device__ __forceinline__ static void rest(float2 (&v)[E], float2* s, const float2* __restrict__ tw, int t) {
    constexpr int R = fft_radix(N, NS);
    constexpr bool LAST = NS * R >= N;
    pass<NS, INV, LAST>(v, s, tw, t);
    if constexpr (!LAST) rest<NS * R, INV>(v, s, tw, t);
  }

  // Two independent transforms of the same direction in lockstep: v1 with
  // buffer s1, v2 with buffer s2.  Each pass loads a twiddle once for both,
  // waits on one barrier for both, and has twice the independent arithmetic;
  // every value is computed exactly as by two run() calls.
  template <int NS, bool INV, bool LAST>
  __device__ __forceinline__ static void pass2(float2 (&v1)[E], float2* s1, float2 (&v2)[E], float2* s2,
                                               const float2* __restrict__ tw, int t) {
    constexpr int R = fft_radix(N, NS);
    constexpr int B = E / R;
    float2 w1[B][R], w2[B][R];
#pragma unroll
    for (int b = 0; b < B; b++) {
      const int j = t + T * b;
      const int k = j & (NS - 1);
      const float2* twp = tw + (NS - 16) + k;
      w1[b][0] = s1[pidx(j)];
      w2[b][0] = s2[pidx(j)];
#pragma unroll
      for (int r = 1; r < R; r++) {
        const float2 c = __ldg(&twp[(r - 1) * NS]);
        w1[b][r] = cmul_tw<INV>(s1[pidx(j + r * (N / R))], c);
        w2[b][r] = cmul_tw<INV>(s2[pidx(j + r * (N / R))], c);
      }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; b++) {
      dft<R, INV>(w1[b]);
      dft<R, INV>(w2[b]);
    }
    if constexpr (LAST) {
#pragma unroll
      for (int b = 0; b < B; b++)
#pragma unroll
        for (int r = 0; r < R; r++) {
          v1[b + B * r] = w1[b][dft_slot<R>(r)];
          v2[b + B * r] = w2[b][dft_slot<R>(r)];
        }
    } else {
#pragma unroll
      for (int b = 0; b < B; b++) {
        const int j = t + T * b;
        const int k = j & (NS - 1);
        const int base = (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) {
          s1[pidx(base + r * NS)] = w1[b][dft_slot<R>(r)];
          s2[pidx(base + r * NS)] = w2[b][dft_slot<R>(r)];
        }
      }
      __syncthreads();
    }
  }

  template <int NS, bool INV>
  __device__ __forceinline__ static void rest2(float2 (&v1)[E], float2* s1, float2 (&v2)[E], float2* s2,
                                               const float2* __restrict__ tw, int t) {
    constexpr int R = fft_radix(N, NS);
    constexpr bool LAST = NS * R >= N;
    pass2<NS, INV, LAST>(v1, s1, v2, s2, tw, t);
    if constexpr (!LAST) rest2<NS * R, INV>(v1, s1, v2, s2, tw, t);
  }

  // run() on two transforms at once (see pass2); s1 and s2 may be in use by
  // the caller until this call.
  template <bool INV>
  __device__ __forceinline__ static void run2(float2 (&v1)[E], float2* s1, float2 (&v2)[E], float2* s2,
                                              const float2* __restrict__ tw, int t) {
    static_assert(N >= 256 && (N & (N - 1)) == 0, "power of two >= 256");
    float2 w1[G][16], w2[G][16];
#pragma unroll
    for (int g = 0; g < G; g++) {
#pragma unroll
      for (int r = 0; r < 16; r++) {
        w1[g][r] = v1[g + G * r];
        w2[g][r] = v2[g + G * r];
      }
      dft<16, INV>(w1[g]);
      dft<16, INV>(w2[g]);
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < G; g++)
#pragma unroll
      for (int r = 0; r < 16; r++) {
        s1[pidx(16 * (t + T * g) + r)] = w1[g][dft_slot<16>(r)];
        s2[pidx(16 * (t + T * g) + r)] = w2[g][dft_slot<16>(r)];
      }
    __syncthreads();
    rest2<16, INV>(v1, s1, v2, s2, tw, t);
  }

  // Transform v in place.  The buffer s (fft_pad(N) float2) may be in use by
  // the caller until this call: the first write waits on a barrier.
  template <bool INV>
  __device__ __forceinline__ static void run(float2 (&v)[E], float2* s, const float2* __restrict__ tw, int t) {
    static_assert(N >= 256 && (N & (N - 1)) == 0, "power of two >= 256");
    // pass NS = 1: butterfly t + T*g reads elements t + T*(g + G*r), all
    // held by this thread (slots g + G*r)
    float2 w[G][16];
#pragma unroll
    for (int g = 0; g < G; g++) {
#pragma unroll
      for (int r = 0; r < 16; r++) w[g][r] = v[g + G * r];
      dft<16, INV>(w[g]);
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < G; g++)
#pragma unroll
      for (int r = 0; r < 16; r++) s[pidx(16 * (t + T * g) + r)] = w[g][dft_slot<16>(r)];
    __syncthreads();
    rest<16, INV>(v, s, tw, t);
  }
};

}  // namespace cuvhs
