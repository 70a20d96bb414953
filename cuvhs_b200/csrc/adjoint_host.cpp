// Calibration decode model: host side of the adjoint pair (extern "C"
// cuvhs_adjoint_*).  The device kernels are in adjoint.cu.
//
// The video filter's block spectrum and its four parameter derivatives are
// built here in FP64 for every call, directly on the 8192-point block grid:
// the response R = H(z) S(f) there is the spectrum of the filter's time
// kernel wrapped to 8192 samples, whose taps beyond the +/-b_pos support of
// the overlap-save blocks (the support the decoder's K1b uses) are below
// ~5e-9 of the peak, so the blocks see the filter itself.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cuvhs.h"
#include "adjoint.h"
#include "pipeline.h"

namespace cuvhs {
cuvhs_status create_context(const cuvhs_config& cfg, cuvhs_ctx** out);
}  // namespace cuvhs

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;
constexpr int kN = cuvhs::Design::kNb;
constexpr int kRowFirst = 10, kRowEnd = 262;   // loss rows of every field
// Loss columns: the back porch with the colour burst and the active picture
// (which ends at 894).  Further left lies the sync trailing edge, which a
// line's start offset does not move on the tape but does move in the model.
constexpr int kColFirst = 80, kColEnd = 894;

double super_gauss(double f, double corner, int order) {
  const double scale = std::pow(std::log(2.0) / 2.0, 1.0 / (2.0 * order));
  const double x = 2.0 * f * scale / corner;
  return std::exp(-2.0 * std::pow(x, 2.0 * order));
}

}  // namespace

struct cuvhs_adjoint {
  cuvhs_ctx* ctx = nullptr;
  int P = 0;
  long long total = 0;
  int blocks = 0;
  cuvhs::AdjArgs args{};
  std::vector<void*> allocs;
  // device
  float *d_dem = nullptr, *d_pre = nullptr, *d_video = nullptr, *d_gvideo = nullptr;
  float *d_tgt_y = nullptr, *d_tgt_c = nullptr, *d_gain = nullptr, *d_y = nullptr, *d_c = nullptr;
  double *d_ll = nullptr, *d_off = nullptr, *d_phase = nullptr, *d_row = nullptr, *d_blk = nullptr;
  int* d_track = nullptr;
  float2 *d_gv = nullptr, *d_dg = nullptr;
  bool has_target = false;
  double nominal[4] = {0, 0, 0, 0};
  std::string err;
  // host staging
  std::vector<double> h_row, h_blk;
  std::vector<float2> h_gv, h_dg;

  ~cuvhs_adjoint() {
    for (void* p : allocs) cudaFree(p);
    if (ctx) cuvhs_destroy(ctx);
  }
  template <typename T>
  T* alloc(size_t n, bool& ok) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    allocs.push_back(p);
    return static_cast<T*>(p);
  }
  cuvhs::Context& c() { return ctx->c; }

  // Block spectrum of the video filter for (n1, n2, m1, m2) and its derivatives.
  void build_filter(const double th[4]) {
    const double fs = c().fmt.fs_hz;
    const double n1 = th[0], n2 = th[1], m1 = th[2], m2 = th[3];
    const double n0 = 1.0 + m1 + m2 - n1 - n2;
    std::vector<cd> R(kN), dR[4];
    for (auto& v : dR) v.assign(kN, cd(0.0, 0.0));
    for (int k = 0; k < kN; k++) {
      const int kk = k <= kN / 2 ? k : k - kN;
      const double w = 2.0 * kPi * (double)kk / (double)kN;
      const cd z1 = std::exp(cd(0.0, -w)), z2 = z1 * z1;
      const cd num = n0 + n1 * z1 + n2 * z2, den = 1.0 + m1 * z1 + m2 * z2;
      const cd H = num / den;
      const double S = super_gauss(std::fabs((double)kk) * fs / (double)kN, 3.0e6, 9);
      R[k] = H * S;
      dR[0][k] = (z1 - 1.0) / den * S;            // n0 moves with n1
      dR[1][k] = (z2 - 1.0) / den * S;
      dR[2][k] = (1.0 / den - H * z1 / den) * S;  // n0 moves with m1
      dR[3][k] = (1.0 / den - H * z2 / den) * S;
    }
    h_gv.resize(kN);
    h_dg.resize((size_t)4 * kN);
    for (int k = 0; k < kN; k++) {
      h_gv[k] = make_float2((float)(R[k].real() / kN), (float)(R[k].imag() / kN));
      for (int j = 0; j < 4; j++)
        h_dg[(size_t)j * kN + k] = make_float2((float)(dR[j][k].real() / kN), (float)(dR[j][k].imag() / kN));
    }
  }

  void upload_params(const cuvhs_adjoint_params* p, bool derivs) {
    build_filter(p->deemph);
    cudaStream_t st = c().stream;
    cudaMemcpyAsync(d_gv, h_gv.data(), sizeof(float2) * kN, cudaMemcpyHostToDevice, st);
    if (derivs) cudaMemcpyAsync(d_dg, h_dg.data(), sizeof(float2) * 4 * kN, cudaMemcpyHostToDevice, st);
    const int H = c().fmt.output_field_lines;
    cudaMemcpyAsync(d_off, p->line_offset, sizeof(double) * P * (H + 1), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_phase, p->chroma_phase, sizeof(double) * P * H, cudaMemcpyHostToDevice, st);
  }

  bool finish(const char* where) {
    cudaError_t e = cudaStreamSynchronize(c().stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
      err = std::string(where) + ": " + cudaGetErrorString(e);
      return false;
    }
    return true;
  }
};

extern "C" {

cuvhs_status cuvhs_adjoint_create(const cuvhs_config* cfg, const uint8_t* samples, size_t n, int fields,
                                  cuvhs_adjoint** out) {
  if (!cfg || !samples || !out || fields < 1) return CUVHS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (cfg->system != 0) {
    fprintf(stderr, "cuvhs_adjoint_create: the calibration model is NTSC only\n");
    return CUVHS_ERR_UNSUPPORTED;
  }
  cuvhs_adjoint* a = new (std::nothrow) cuvhs_adjoint();
  if (!a) return CUVHS_ERR_OUT_OF_MEMORY;
  cuvhs_config cc = *cfg;
  cc.batch_fields = fields;
  cuvhs_status s = cuvhs::create_context(cc, &a->ctx);
  if (s != CUVHS_OK) {
    delete a;
    return s;
  }
  cuvhs::Context& c = a->c();
  // the normal decode: line locations, tracks, pre-band-pass
  cuvhs::ChunkResult r;
  if (!c.decode_chunk(samples, false, n, 0, fields, r) || r.fields < 1) {
    fprintf(stderr, "cuvhs_adjoint_create: %s\n", r.fields < 1 ? "no field decoded" : c.err.c_str());
    s = c.status != CUVHS_OK ? c.status : CUVHS_ERR_INVALID_ARGUMENT;
    delete a;
    return s;
  }
  const int P = r.fields;
  const int H = c.fmt.output_field_lines, W = c.fmt.output_line_len, LPF = c.fmt.lines_per_frame;
  const long long total = (long long)P * c.spp;
  a->P = P;
  a->total = total;
  a->blocks = (int)((total + c.des.b_out - 1) / c.des.b_out);
  const size_t spf = (size_t)c.fmt.samples_per_field;
  const int T = (int)std::min(std::min((size_t)fields * c.spp, n) / spf, (size_t)fields);  // K1a tiles, >= P
  bool ok = true;
  a->d_dem = a->alloc<float>((size_t)T * c.spp, ok);
  a->d_pre = a->alloc<float>(total, ok);
  a->d_video = a->alloc<float>(total, ok);
  a->d_gvideo = a->alloc<float>(total, ok);
  a->d_tgt_y = a->alloc<float>((size_t)P * H * W, ok);
  a->d_tgt_c = a->alloc<float>((size_t)P * H * W, ok);
  a->d_y = a->alloc<float>((size_t)P * H * W, ok);
  a->d_c = a->alloc<float>((size_t)P * H * W, ok);
  a->d_gain = a->alloc<float>((size_t)P * H, ok);
  a->d_ll = a->alloc<double>((size_t)P * LPF, ok);
  a->d_off = a->alloc<double>((size_t)P * (H + 1), ok);
  a->d_phase = a->alloc<double>((size_t)P * H, ok);
  a->d_row = a->alloc<double>((size_t)P * H * cuvhs::kAdjRowVals, ok);
  a->d_blk = a->alloc<double>((size_t)a->blocks * 4, ok);
  a->d_track = a->alloc<int>(P, ok);
  a->d_gv = a->alloc<float2>(kN, ok);
  a->d_dg = a->alloc<float2>((size_t)4 * kN, ok);
  if (!ok) {
    fprintf(stderr, "cuvhs_adjoint_create: device allocation failed\n");
    delete a;
    return CUVHS_ERR_OUT_OF_MEMORY;
  }
  cudaStream_t st = c.stream;
  // the pre-band-pass is still in the decoder's demod buffer; the demod itself
  // is recomputed from the raw window into the model's own buffer
  cudaMemcpyAsync(a->d_pre, c.d_dem, sizeof(float) * total, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(a->d_ll, c.d_ll, sizeof(double) * P * LPF, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(a->d_track, c.computed_track.data(), sizeof(int) * P, cudaMemcpyHostToDevice, st);
  cuvhs::DemodArgs da = c.demod_args(T);
  da.dem = a->d_dem;
  cuvhs::launch_k1a(da, 0, T, st);
  cudaMemsetAsync(a->d_off, 0, sizeof(double) * P * (H + 1), st);
  cudaMemsetAsync(a->d_phase, 0, sizeof(double) * P * H, st);
  // model arguments
  cuvhs::AdjArgs& g = a->args;
  g.dem = a->d_dem;
  g.pre = a->d_pre;
  g.ll = a->d_ll;
  g.track = a->d_track;
  g.tgt_y = a->d_tgt_y;
  g.tgt_c = a->d_tgt_c;
  g.col_frac = c.d_col_frac;
  g.total = total;
  g.fields = P;
  g.lpf = LPF;
  g.out_w = W;
  g.out_h = H;
  g.row0 = kRowFirst;
  g.row1 = kRowEnd;
  g.col0 = kColFirst;
  g.col1 = kColEnd;
  g.luma_gain = c.fmt.output_scale / c.fmt.hz_ire;
  g.luma_offset = -c.fmt.vsync_ire * c.fmt.output_scale + c.fmt.output_zero;
  g.het_scale = c.des.het_scale;
  g.fsc_bin = c.des.fsc_bin;
  g.bw_bins = c.des.bw_bins;
  g.burst_start = c.fmt.burst_start;
  g.burst_abs_ref = (float)c.fmt.burst_abs_ref;
  g.tw_b = c.d_twb;
  g.tw_b_inv = c.d_twb_inv;
  g.tw_l = c.d_twl;
  g.tw_l_inv = c.d_twl_inv;
  g.b_pos = c.des.b_pos;
  g.b_out = c.des.b_out;
  g.blocks = a->blocks;
  const double npix = (double)P * (kRowEnd - kRowFirst) * (kColEnd - kColFirst);
  g.inv_ny = 1.0 / npix;
  g.inv_nc = 1.0 / npix;
  g.gv = a->d_gv;
  g.dg = a->d_dg;
  g.carrier = 0.0;
  g.deviation = 1.0;
  g.line_off = a->d_off;
  g.phase = a->d_phase;
  g.video = a->d_video;
  g.gvideo = a->d_gvideo;
  g.y_out = nullptr;
  g.c_out = nullptr;
  g.gain_out = a->d_gain;
  g.row = a->d_row;
  g.blk = a->d_blk;
  // nominal de-emphasis: the inverse of the pre-emphasis shelf (its numerator
  // and denominator swapped, src/pipeline/fm_demod.cu:310-331 of the
  // reference), normalised to a unit leading denominator coefficient
  {
    const double fs = c.fmt.fs_hz;
    const double A = std::pow(10.0, 13.9794 / 40.0), w0 = 2.0 * kPi * 273755.82 / fs;
    const double alpha = std::sin(w0) / (2.0 * 0.462088186), cw = std::cos(w0), sa = std::sqrt(A);
    const double b0 = A * ((A + 1) + (A - 1) * cw + 2 * sa * alpha);
    const double b1 = -2 * A * ((A - 1) + (A + 1) * cw);
    const double b2 = A * ((A + 1) + (A - 1) * cw - 2 * sa * alpha);
    const double a1 = 2 * ((A - 1) - (A + 1) * cw);
    const double a2 = (A + 1) - (A - 1) * cw - 2 * sa * alpha;
    a->nominal[0] = a1 / b0;
    a->nominal[1] = a2 / b0;
    a->nominal[2] = b1 / b0;
    a->nominal[3] = b2 / b0;
  }
  // one pass at the nominal parameters leaves the ACC gains for inspection
  a->build_filter(a->nominal);
  cudaMemcpyAsync(a->d_gv, a->h_gv.data(), sizeof(float2) * kN, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(a->d_tgt_c, 0, sizeof(float) * P * H * W, st);
  cuvhs::launch_adj_video(g, st);
  cuvhs::launch_adj_chroma(g, 0, st);
  if (!a->finish("adjoint create")) {
    fprintf(stderr, "cuvhs_adjoint_create: %s\n", a->err.c_str());
    delete a;
    return CUVHS_ERR_CUDA;
  }
  a->h_row.resize((size_t)P * H * cuvhs::kAdjRowVals);
  a->h_blk.resize((size_t)a->blocks * 4);
  *out = a;
  return CUVHS_OK;
}

void cuvhs_adjoint_destroy(cuvhs_adjoint* a) { delete a; }

int cuvhs_adjoint_fields(const cuvhs_adjoint* a) { return a ? a->P : 0; }

cuvhs_status cuvhs_adjoint_default_params(const cuvhs_adjoint* a, cuvhs_adjoint_params* p) {
  if (!a || !p) return CUVHS_ERR_INVALID_ARGUMENT;
  for (int j = 0; j < 4; j++) p->deemph[j] = a->nominal[j];
  p->carrier_hz = 0.0;
  p->deviation = 1.0;
  const int H = CUVHS_FIELD_HEIGHT;
  if (p->line_offset) std::fill(p->line_offset, p->line_offset + (size_t)a->P * (H + 1), 0.0);
  if (p->chroma_phase) std::fill(p->chroma_phase, p->chroma_phase + (size_t)a->P * H, 0.0);
  return CUVHS_OK;
}

cuvhs_status cuvhs_adjoint_set_target(cuvhs_adjoint* a, const float* luma, const float* chroma) {
  if (!a || !luma || !chroma) return CUVHS_ERR_INVALID_ARGUMENT;
  const size_t np = (size_t)a->P * CUVHS_FIELD_HEIGHT * CUVHS_FIELD_WIDTH;
  cudaStream_t st = a->c().stream;
  cudaMemcpyAsync(a->d_tgt_y, luma, sizeof(float) * np, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(a->d_tgt_c, chroma, sizeof(float) * np, cudaMemcpyHostToDevice, st);
  if (!a->finish("set target")) return CUVHS_ERR_CUDA;
  a->has_target = true;
  return CUVHS_OK;
}

static bool check_params(const cuvhs_adjoint* a, const cuvhs_adjoint_params* p) {
  return a && p && p->line_offset && p->chroma_phase && std::isfinite(p->deviation) && p->deviation != 0.0 &&
         std::isfinite(p->carrier_hz);
}

static double sum_loss(cuvhs_adjoint* a) {
  const int rows = a->P * CUVHS_FIELD_HEIGHT;
  double ly = 0.0, lc = 0.0;
  for (int r = 0; r < rows; r++) {
    ly += a->h_row[(size_t)r * cuvhs::kAdjRowVals + cuvhs::kRowLossY];
    lc += a->h_row[(size_t)r * cuvhs::kAdjRowVals + cuvhs::kRowLossC];
  }
  return ly * a->args.inv_ny + lc * a->args.inv_nc;
}

cuvhs_status cuvhs_adjoint_fwd(cuvhs_adjoint* a, const cuvhs_adjoint_params* p, double* loss, float* luma,
                               float* chroma) {
  if (!check_params(a, p)) return CUVHS_ERR_INVALID_ARGUMENT;
  if (loss && !a->has_target) return CUVHS_ERR_INVALID_ARGUMENT;
  cudaStream_t st = a->c().stream;
  a->upload_params(p, false);
  cuvhs::AdjArgs g = a->args;
  g.carrier = p->carrier_hz;
  g.deviation = p->deviation;
  g.y_out = luma ? a->d_y : nullptr;
  g.c_out = chroma ? a->d_c : nullptr;
  cudaMemsetAsync(a->d_row, 0, sizeof(double) * a->h_row.size(), st);
  cuvhs::launch_adj_video(g, st);
  cuvhs::launch_adj_luma(g, 0, st);
  cuvhs::launch_adj_chroma(g, 0, st);
  const size_t np = (size_t)a->P * CUVHS_FIELD_HEIGHT * CUVHS_FIELD_WIDTH;
  if (luma) cudaMemcpyAsync(luma, a->d_y, sizeof(float) * np, cudaMemcpyDeviceToHost, st);
  if (chroma) cudaMemcpyAsync(chroma, a->d_c, sizeof(float) * np, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(a->h_row.data(), a->d_row, sizeof(double) * a->h_row.size(), cudaMemcpyDeviceToHost, st);
  if (!a->finish("adjoint forward")) return CUVHS_ERR_CUDA;
  if (loss) *loss = sum_loss(a);
  return CUVHS_OK;
}

cuvhs_status cuvhs_adjoint_bwd(cuvhs_adjoint* a, const cuvhs_adjoint_params* p, double* loss,
                               cuvhs_adjoint_params* grad) {
  if (!check_params(a, p) || !grad || !grad->line_offset || !grad->chroma_phase || !a->has_target)
    return CUVHS_ERR_INVALID_ARGUMENT;
  cudaStream_t st = a->c().stream;
  a->upload_params(p, true);
  cuvhs::AdjArgs g = a->args;
  g.carrier = p->carrier_hz;
  g.deviation = p->deviation;
  cudaMemsetAsync(a->d_row, 0, sizeof(double) * a->h_row.size(), st);
  cudaMemsetAsync(a->d_gvideo, 0, sizeof(float) * a->total, st);
  cuvhs::launch_adj_video(g, st);  // recomputed: the forward keeps nothing for the backward
  cuvhs::launch_adj_luma(g, 1, st);
  cuvhs::launch_adj_chroma(g, 1, st);
  cuvhs::launch_adj_deemph(g, st);
  cudaMemcpyAsync(a->h_row.data(), a->d_row, sizeof(double) * a->h_row.size(), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(a->h_blk.data(), a->d_blk, sizeof(double) * a->h_blk.size(), cudaMemcpyDeviceToHost, st);
  if (!a->finish("adjoint backward")) return CUVHS_ERR_CUDA;
  if (loss) *loss = sum_loss(a);
  const int H = CUVHS_FIELD_HEIGHT;
  const double* R = a->h_row.data();
  auto row = [&](int f, int r, int k) { return R[((size_t)f * H + r) * cuvhs::kAdjRowVals + k]; };
  double dcar = 0.0, ddev = 0.0;
  for (int f = 0; f < a->P; f++)
    for (int r = 0; r < H; r++) {
      dcar += row(f, r, cuvhs::kRowCarrier);
      ddev += row(f, r, cuvhs::kRowDeviation);
    }
  grad->carrier_hz = dcar;
  grad->deviation = ddev;
  for (int j = 0; j < 4; j++) {
    double s = 0.0;
    for (int b = 0; b < a->blocks; b++) s += a->h_blk[(size_t)b * 4 + j];
    grad->deemph[j] = s;
  }
  for (int f = 0; f < a->P; f++) {
    for (int r = 0; r <= H; r++) {
      double s = 0.0;
      if (r < H) s += row(f, r, cuvhs::kRowLumaX0) + row(f, r, cuvhs::kRowChromaX0);
      if (r > 0) s += row(f, r - 1, cuvhs::kRowLumaX1) + row(f, r - 1, cuvhs::kRowChromaX1);
      grad->line_offset[(size_t)f * (H + 1) + r] = s;
    }
    for (int r = 0; r < H; r++) grad->chroma_phase[(size_t)f * H + r] = row(f, r, cuvhs::kRowPhase);
  }
  return CUVHS_OK;
}

long long cuvhs_adjoint_array(const cuvhs_adjoint* a, const char* name, void* dst, long long cap) {
  if (!a || !name) return -1;
  const std::string s(name);
  const int H = CUVHS_FIELD_HEIGHT;
  const void* src = nullptr;
  size_t n = 0, es = 0;
  if (s == "linelocs") {
    src = a->d_ll;
    n = (size_t)a->P * a->ctx->c.fmt.lines_per_frame;
    es = sizeof(double);
  } else if (s == "gains") {
    src = a->d_gain;
    n = (size_t)a->P * H;
    es = sizeof(float);
  } else if (s == "tracks") {
    src = a->d_track;
    n = (size_t)a->P;
    es = sizeof(int);
  } else if (s == "demod" || s == "pre") {
    src = s == "demod" ? a->d_dem : a->d_pre;
    n = (size_t)a->total;
    es = sizeof(float);
  } else {
    return -1;
  }
  if (dst && cap > 0) cudaMemcpy(dst, src, es * std::min<size_t>(n, (size_t)cap), cudaMemcpyDeviceToHost);
  return (long long)n;
}

}  // extern "C"
