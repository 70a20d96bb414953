// Capture sample conversion (reference src/io/raw_reader.cpp:71-101): u8 is
// (x - 128) * 256, s16 is x, u16 is x - 32768; with DC correction the chunk
// mean of the converted samples read is subtracted.  Chunk positions past the
// samples read are 0, the reference's zero fill after conversion
// (src/pipeline/pipeline.cu:1539-1541).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cuvhs {

enum InputFormat { kInU8 = 0, kInS16 = 1, kInU16 = 2 };

template <int FMT>
__device__ __forceinline__ float raw_convert(const uint8_t* __restrict__ raw, int p) {
  // u8: 2^23 + x as a float by setting the exponent bits (no integer-to-float
  // conversion, which issues at a quarter of the FP32 rate), then one exact
  // FMA: (2^23 + x) * 256 - (2^31 + 2^15) = (x - 128) * 256.
  if constexpr (FMT == kInU8)
    return fmaf(__int_as_float(0x4B000000 | (int)__ldg(raw + p)), 256.0f, -2147516416.0f);
  if constexpr (FMT == kInS16) return (float)__ldg(reinterpret_cast<const int16_t*>(raw) + p);
  return (float)__ldg(reinterpret_cast<const uint16_t*>(raw) + p) - 32768.0f;
}

// Sample p of the chunk: converted, DC removed, 0 past the samples read.
template <int FMT>
__device__ __forceinline__ float raw_sample(const uint8_t* __restrict__ raw, int p, int n_read, float dc) {
  return p < n_read ? raw_convert<FMT>(raw, p) - dc : 0.0f;
}

}  // namespace cuvhs
