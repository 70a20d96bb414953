// Calibration decode model and its adjoint (device side).
//
// The model re-runs the parameter-dependent part of the decode on fixed
// inputs from a normal decode (demod, colour-under pre-band-pass, line
// locations, tracks) and compares it with target TBC planes:
//   video  = demod (*) g_theta        de-emphasis H(z) = N(z)/D(z) times the
//                                      3 MHz super-Gaussian, overlap-save
//   Y      = ((CR(video, x) - carrier) / deviation) * A + B
//   C      = g * BP(CR(pre, x) * -cos(2 pi u + lp pi/2 + phase))  + 32768,
//            g = the decoder's ACC: burst reference / rms of BP(...) over the burst window
//   x      = (ll[r] + off[r]) + (c / 910) ((ll[r+1] + off[r+1]) - (ll[r] + off[r]))
//   L      = mean over back porch, burst and picture (Y - Y*)^2 + mean (C - C*)^2
// CR is the decoder's Catmull-Rom resampler, BP its 1024-point line band-pass
// (bins 256 +/- 36; a real symmetric operator, so its own adjoint).
#pragma once
#include <cuda_runtime.h>

#include "cuvhs_internal.h"

namespace cuvhs {

constexpr int kAdjRowVals = 10;  // per-row partial sums, see AdjRow
enum AdjRow {
  kRowLossY = 0,
  kRowLossC,
  kRowCarrier,
  kRowDeviation,
  kRowLumaX0,    // sum over columns of dL/dx * (1 - c/910): the row's own start
  kRowLumaX1,    // ... * c/910: the next row's start
  kRowChromaX0,
  kRowChromaX1,
  kRowPhase,
  kRowSpare
};

struct AdjArgs {
  // fixed inputs
  const float* dem;       // [total] demod - ire0 (Hz)
  const float* pre;       // [total] colour-under pre-band-passed signal
  const double* ll;       // [fields * lpf] line starts
  const int* track;       // [fields]
  const float* tgt_y;     // [fields * out_h * out_w]
  const float* tgt_c;
  const double* col_frac; // [out_w]
  long long total;
  int fields, lpf, out_w, out_h, row0, row1;  // loss rows [row0, row1) of every field
  int col0, col1;                              // loss columns [col0, col1): back porch, burst, picture
  double luma_gain, luma_offset;
  double het_scale;
  int fsc_bin, bw_bins, burst_start;
  float burst_abs_ref;
  const float2* tw_b;
  const float2* tw_b_inv;
  const float2* tw_l;
  const float2* tw_l_inv;
  int b_pos, b_out, blocks;  // video filter support, outputs per block, blocks over [0, total)
  double inv_ny, inv_nc;     // 1 / pixel counts of the two means
  // parameters
  const float2* gv;          // [kNb] video filter block spectrum / kNb (real kernel)
  const float2* dg;          // [4 * kNb] its derivatives by n1, n2, m1, m2
  double carrier, deviation;
  const double* line_off;    // [fields * (out_h + 1)]
  const double* phase;       // [fields * out_h]
  // work and outputs
  float* video;              // [total]
  float* gvideo;             // [total] dL/dvideo (zeroed before the backward pass)
  float* y_out;              // optional [fields * out_h * out_w]
  float* c_out;
  float* gain_out;           // [fields * out_h] ACC gains of the last pass
  double* row;               // [fields * out_h * kAdjRowVals]
  double* blk;               // [blocks * 4]
};

void launch_adj_video(const AdjArgs& a, cudaStream_t st);
// mode 0: forward (loss, optional planes); 1: forward + backward
void launch_adj_luma(const AdjArgs& a, int mode, cudaStream_t st);
// mode 0: forward; 1: forward + backward
void launch_adj_chroma(const AdjArgs& a, int mode, cudaStream_t st);
void launch_adj_deemph(const AdjArgs& a, cudaStream_t st);

}  // namespace cuvhs
