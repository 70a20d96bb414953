// NTSC constants and filter design.
//
// The reference filters every tile in the frequency domain with FP64 cuFFT:
// an RF band-pass times the one-sided Hilbert weighting, then a de-emphasis x
// 3 MHz super-Gaussian video filter and the same times a 0.5 MHz FIR for sync
// (src/pipeline/fm_demod.cu:273-374), and a |Butterworth|^2 colour-under
// band-pass on zero-padded tiles (src/pipeline/chroma_decode.cu:568-633).
// Each of those is a circular convolution with a kernel whose time response
// decays below 1e-10 of its energy within a few hundred to a few thousand
// samples.  Here the exact per-tile frequency response is built in FP64, taken
// to the time domain once, truncated to a support of a few thousand taps and
// re-transformed to the block size of a shared-memory overlap-save kernel.
// The GPU then evaluates the same circular tile convolution block by block in
// one HBM pass per stage instead of 500k-point transforms.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <map>
#include <mutex>

#include "cuvhs_internal.h"
#include "host_fft.h"

namespace cuvhs {
namespace {

constexpr double kPi = 3.14159265358979323846;

int next_smooth7(int n) {
  for (;; n++) {
    int m = n;
    for (int p : {2, 3, 5, 7})
      while (m % p == 0) m /= p;
    if (m == 1) return n;
  }
}

// Butterworth magnitudes on the bilinear-warped axis
// (src/pipeline/fm_demod.cu:35-63).
double bw_lowpass(double w, double wc, int order) {
  if (wc <= 0.0 || wc >= kPi) return 1.0;
  const double tc = std::tan(wc / 2.0);
  if (tc == 0.0) return 1.0;
  return 1.0 / std::sqrt(1.0 + std::pow(std::tan(w / 2.0) / tc, 2.0 * order));
}
double bw_highpass(double w, double wc, int order) {
  if (w <= 0.0) return 0.0;
  if (wc <= 0.0 || wc >= kPi) return 1.0;
  const double t = std::tan(w / 2.0);
  if (t == 0.0) return 0.0;
  return 1.0 / std::sqrt(1.0 + std::pow(std::tan(wc / 2.0) / t, 2.0 * order));
}
double bw_bandpass(double w, double wl, double wh, int order) {
  if (w <= 0.0 || w >= kPi) return 0.0;
  const double tl = std::tan(wl / 2.0), th = std::tan(wh / 2.0), t = std::tan(w / 2.0);
  const double bw = th - tl;
  if (bw <= 0.0 || t == 0.0) return 0.0;
  const double s = (t * t - tl * th) / (bw * t);
  return 1.0 / std::sqrt(1.0 + std::pow(s, 2.0 * order));
}
// (src/pipeline/fm_demod.cu:65-70)
double super_gauss(double f, double corner, int order) {
  const double scale = std::pow(std::log(2.0) / 2.0, 1.0 / (2.0 * order));
  const double x = 2.0 * f * scale / corner;
  return std::exp(-2.0 * std::pow(x, 2.0 * order));
}
// RBJ high shelf; the decoder uses its inverse as de-emphasis
// (src/pipeline/fm_demod.cu:72-86, used with num/den swapped at :331).
void high_shelf(double f0, double db, double fs, double q, double b[3], double a[3]) {
  const double A = std::pow(10.0, db / 40.0);
  const double w0 = 2.0 * kPi * f0 / fs;
  const double alpha = std::sin(w0) / (2.0 * q);
  const double c = std::cos(w0), sa = std::sqrt(A);
  b[0] = A * ((A + 1) + (A - 1) * c + 2 * sa * alpha);
  b[1] = -2 * A * ((A - 1) + (A + 1) * c);
  b[2] = A * ((A + 1) + (A - 1) * c - 2 * sa * alpha);
  a[0] = (A + 1) - (A - 1) * c + 2 * sa * alpha;
  a[1] = 2 * ((A - 1) - (A + 1) * c);
  a[2] = (A + 1) - (A - 1) * c - 2 * sa * alpha;
}
cd biquad(const double num[3], const double den[3], double w) {
  const cd z1 = std::exp(cd(0.0, -w)), z2 = z1 * z1;
  return (num[0] + num[1] * z1 + num[2] * z2) / (den[0] + den[1] * z1 + den[2] * z2);
}
// Hamming-windowed sinc low-pass, unit DC gain (src/pipeline/fm_demod.cu:96-115).
std::vector<double> windowed_sinc(int taps, double cut) {
  std::vector<double> h(taps);
  const double mid = (taps - 1) / 2.0;
  double sum = 0.0;
  for (int n = 0; n < taps; n++) {
    const double m = n - mid;
    const double s = std::fabs(m) < 1e-12 ? cut : std::sin(kPi * cut * m) / (kPi * m);
    h[n] = s * (0.54 - 0.46 * std::cos(2.0 * kPi * n / (taps - 1)));
    sum += h[n];
  }
  for (double& v : h) v /= sum;
  return h;
}
cd fir_response(const std::vector<double>& h, double w, int delay) {
  cd acc(0.0, 0.0);
  for (size_t n = 0; n < h.size(); n++) acc += h[n] * std::exp(cd(0.0, -(double)n * w));
  if (delay > 0) acc *= std::exp(cd(0.0, w * delay));
  return acc;
}

// Truncate the circular kernel k (length L) to offsets [-neg, pos] and place it
// circularly in an N-point block.  Returns the relative l2 energy dropped.
double place_kernel(const std::vector<cd>& k, int neg, int pos, int N, std::vector<cd>& blk) {
  const int L = (int)k.size();
  blk.assign(N, cd(0.0, 0.0));
  double kept = 0.0, total = 0.0;
  for (int i = 0; i < L; i++) total += std::norm(k[i]);
  for (int m = -neg; m <= pos; m++) {
    const cd v = k[(size_t)((m % L + L) % L)];
    blk[(size_t)((m % N + N) % N)] = v;
    kept += std::norm(v);
  }
  return total > 0 ? std::max(0.0, total - kept) / total : 0.0;
}

// Kernel half-support for sample rate fs: the filters are specified in Hz, so
// their time responses stretch in proportion to fs.  per_mhz samples per MHz
// keep every dropped tap below ~5e-9 of the kernel's peak (below FP32
// resolution) at 28, 35.8 and 40 MHz; rounded up to a multiple of quantum.
int half_support(double fs_hz, double per_mhz, int quantum, int cap) {
  const int n = (int)std::ceil(fs_hz * 1e-6 * per_mhz / quantum) * quantum;
  return std::min(n, cap);
}

// Smallest half-support h (a multiple of quantum, at most cap) of the circular
// kernel k such that every tap at an offset beyond +/-h lies below rel times
// the largest tap (real parts only when real_only).
int tail_half_support(const std::vector<cd>& k, bool real_only, double rel, int quantum, int cap) {
  const int L = (int)k.size();
  auto mag = [&](int i) { return real_only ? std::fabs(k[(size_t)i].real()) : std::abs(k[(size_t)i]); };
  double peak = 0.0;
  for (int i = 0; i < L; i++) peak = std::max(peak, mag(i));
  int last = 0;  // largest offset whose tap (either side) is above the bound
  for (int m = 1; m < L / 2; m++)
    if (mag(m) > rel * peak || mag(L - m) > rel * peak) last = m;
  return std::min(cap, (last + quantum) / quantum * quantum);
}

// Per-pass twiddles of the shared-memory FFT (smem_fft.cuh): pass NS >= 16 of
// radix R holds W_{NS*R}^{r*k} at (NS - 16) + (r - 1) * NS + k.
std::vector<float2> twiddles(int n) {
  std::vector<float2> t;
  for (int ns = 16; ns < n; ns *= 16) {
    const int R = ns * 16 <= n ? 16 : n / ns;
    for (int r = 1; r < R; r++)
      for (int k = 0; k < ns; k++) {
        const double a = -2.0 * kPi * (double)r * (double)k / (double)(ns * R);
        t.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
      }
  }
  return t;
}

}  // namespace

int k1a_half_support(double fs_hz) { return half_support(fs_hz, 13.7, 64, 1024); }

void Format::init(double mhz, int sys) {
  system = sys == kPal ? kPal : kNtsc;
  fs_hz = mhz * 1e6;
  if (system == kNtsc) {
    lines_per_frame = 525;
    lines_per_field = 263;
    output_line_len = 910;
    output_field_lines = 263;
    field_lines_first = 263;
    field_lines_second = 262;
    num_eq_pulses = 6;
    active_line_start = 10;
    line_rate = 15734.264;
    fsc = 3579545.0;
    chroma_under = (525.0 * (30.0 / 1.001)) * 40.0;
    burst_abs_ref = 4416.0;
    burst_start_us = 5.3;
    burst_end_us = 7.8;
    hz_ire = 1e6 / 140.0;
    ire0 = 4.4e6 - (hz_ire * 100.0);
    vsync_ire = -40.0;
    output_zero = 1024.0;
    output_scale = (51200.0 - 1024.0) / (100.0 - vsync_ire);
    vsync_width = 27.1e-6 * fs_hz;
  } else {
    lines_per_frame = 625;
    lines_per_field = 313;
    output_line_len = 1135;
    output_field_lines = 313;
    field_lines_first = 312;
    field_lines_second = 313;
    num_eq_pulses = 5;
    active_line_start = 8;
    line_rate = 15625.0;
    fsc = 4433618.75;
    chroma_under = ((625.0 * 25.0) * 40.0) + 1953.0;
    burst_abs_ref = 5000.0;
    burst_start_us = 5.6;
    burst_end_us = 7.85;
    vsync_ire = -0.3 * (100.0 / 0.7);
    hz_ire = 1e6 / (100.0 + (-vsync_ire));
    ire0 = 4.8e6 - (hz_ire * 100.0);
    output_zero = 256.0;
    output_scale = (54016.0 - 256.0) / (100.0 - vsync_ire);
    vsync_width = 27.3e-6 * fs_hz;
  }
  pulse_threshold_hz = ire0 + hz_ire * (-20.0);
  output_rate = 4.0 * fsc;
  samples_per_line = (int)std::round(fs_hz / line_rate);
  samples_per_field = samples_per_line * lines_per_field;
  spp = samples_per_field + kFieldMarginLines * samples_per_line;
  hsync_width = 4.7e-6 * fs_hz;
  eq_pulse_width = 2.3e-6 * fs_hz;
  burst_start = (int)(burst_start_us * 1e-6 * output_rate + 0.5);
  burst_end = (int)(burst_end_us * 1e-6 * output_rate + 0.5);
  burst_len = burst_end - burst_start;
  line_fft = 1;
  while (line_fft < output_line_len) line_fft <<= 1;
}

void Design::build(const Format& fmt) {
  const double fs = fmt.fs_hz, ny = fs / 2.0;
  tile = next_smooth7(fmt.spp + kOverlap);
  bins = tile / 2 + 1;

  // ---- K1a: one-sided RF response (band-pass x low-pass x high-pass x Hilbert weight)
  {
    std::vector<cd> H(tile, cd(0.0, 0.0));
    const double wbl = kPi * 1.3e6 / ny, wbh = kPi * 7.5e6 / ny, wl = kPi * 8e6 / ny, wh = kPi * 1e6 / ny;
    for (int k = 0; k < bins; k++) {
      const double w = kPi * (double)k / (double)(bins - 1);
      const double hil = (k == 0 || k == bins - 1) ? 1.0 : 2.0;
      H[k] = bw_bandpass(w, wbl, wbh, 8) * bw_lowpass(w, wl, 8) * bw_highpass(w, wh, 8) * hil;
    }
    std::vector<cd> g = host_dft(H, +1);  // unnormalised inverse, as the reference's C2C
    a_neg = a_pos = k1a_half_support(fs);
    a_out = kNa - a_neg - a_pos - 1;
    // FP64 taps for the guard-band re-evaluation of sync samples
    ga64_half = tail_half_support(g, false, kGuardTailRel, 64, kGuardMaxHalf);
    ga64.resize((size_t)(2 * ga64_half + 1) * 2);
    for (int m = -ga64_half; m <= ga64_half; m++) {
      const cd v = g[(size_t)((m % tile + tile) % tile)];
      ga64[(size_t)(m + ga64_half) * 2] = v.real();
      ga64[(size_t)(m + ga64_half) * 2 + 1] = v.imag();
    }
    {
      const int N = kGuardN;
      std::vector<cd> w(N);
      for (int k = 0; k < N; k++) w[k] = std::polar(1.0, -2.0 * kPi * (double)k / (double)N);
      guard_tw.resize((size_t)N * 2);
      for (int k = 0; k < N; k++) {
        guard_tw[(size_t)k * 2] = w[k].real();
        guard_tw[(size_t)k * 2 + 1] = w[k].imag();
      }
      guard_g.assign((size_t)N * 2, 0.0);
      if (2 * ga64_half + 1 <= N) {
        for (int k = 0; k < N; k++) {
          cd acc(0.0, 0.0);
          for (int m = -ga64_half; m <= ga64_half; m++) {
            const cd tap(ga64[(size_t)(m + ga64_half) * 2], ga64[(size_t)(m + ga64_half) * 2 + 1]);
            const long long e = ((long long)m * k % N + N) % N;
            acc += tap * w[(size_t)e];
          }
          guard_g[(size_t)k * 2] = acc.real() / N;
          guard_g[(size_t)k * 2 + 1] = acc.imag() / N;
        }
      }
    }
    std::vector<cd> blk;
    a_tail = place_kernel(g, a_neg, a_pos, kNa, blk);
    std::vector<cd> G = host_dft(blk, -1);
    ga.resize(kNa);
    // halved: the paired-block kernel separates two spectra as (U +/- conj(U'))
    for (int k = 0; k < kNa; k++)
      ga[k] = make_float2((float)(G[k].real() / kNa) * 0.5f, (float)(G[k].imag() / kNa) * 0.5f);
    demod_scale = (float)(fs / (2.0 * kPi));
    d0 = fmt.ire0 * 2.0 * kPi / fs;
    const float d0f = (float)d0;
    rot_re = (float)std::cos((double)d0f);
    rot_im = (float)-std::sin((double)d0f);
    demod_offset = (float)((double)d0f * (fs / (2.0 * kPi)) - fmt.ire0);
  }

  // ---- K1b: video = de-emphasis x super-Gaussian; sync = video x 65-tap FIR
  {
    double bs[3], as[3];
    high_shelf(273755.82, 13.9794, fs, 0.462088186, bs, as);
    const std::vector<double> fir = windowed_sinc(65, 500000.0 / ny);
    const double inv_n = 1.0 / (double)tile;
    std::vector<cd> FV(tile), FS(tile);
    for (int k = 0; k < bins; k++) {
      const double w = kPi * (double)k / (double)(bins - 1);
      const double f_hz = (double)k * ny / (double)(bins - 1);
      const cd de = biquad(as, bs, w);
      const double v = super_gauss(f_hz, 3.0e6, 9);
      FV[k] = de * v * inv_n;
      FS[k] = de * v * fir_response(fir, w, 32) * inv_n;
    }
    // A complex-to-real inverse reads the half spectrum as Hermitian and drops
    // the imaginary parts of DC and (even lengths) Nyquist.
    FV[0] = cd(FV[0].real(), 0.0);
    FS[0] = cd(FS[0].real(), 0.0);
    if (tile % 2 == 0) {
      FV[tile / 2] = cd(FV[tile / 2].real(), 0.0);
      FS[tile / 2] = cd(FS[tile / 2].real(), 0.0);
    }
    for (int k = bins; k < tile; k++) {
      FV[k] = std::conj(FV[tile - k]);
      FS[k] = std::conj(FS[tile - k]);
    }
    std::vector<cd> hv = host_dft(FV, +1), hs = host_dft(FS, +1);
    std::vector<cd> c(tile);
    for (int n = 0; n < tile; n++) c[n] = cd(hv[n].real(), hs[n].real());
    hs64_half = tail_half_support(hs, true, kGuardTailRel, 64, kGuardMaxHalf);
    hs64.resize((size_t)(2 * hs64_half + 1));
    for (int m = -hs64_half; m <= hs64_half; m++) hs64[(size_t)(m + hs64_half)] = hs[(size_t)((m % tile + tile) % tile)].real();
    b_neg = b_pos = half_support(fs, 25.6, 64, 2048);
    b_out = kNb - b_neg - b_pos;
    std::vector<cd> blk;
    b_tail = place_kernel(c, b_neg, b_pos, kNb, blk);
    std::vector<cd> G = host_dft(blk, -1);
    gb.resize(kNb);
    for (int k = 0; k < kNb; k++)  // halved, as ga
      gb[k] = make_float2((float)(G[k].real() / kNb) * 0.5f, (float)(G[k].imag() / kNb) * 0.5f);
    // Output relative to ire0: the constant ire0 passes with the filters' DC gain.
    corr_video = (float)(fmt.ire0 * (FV[0].real() * tile - 1.0));
    corr_sync = (float)(fmt.ire0 * (FS[0].real() * tile - 1.0));
  }

  // ---- colour-under pre-band-pass: |Butterworth 60 kHz - 1.2 MHz, order 4|^2 / R
  {
    ctile = next_smooth7(fmt.spp);
    const int rb = ctile / 2 + 1;
    const double wlo = 2.0 * kPi * 60000.0 / fs, whi = 2.0 * kPi * 1200000.0 / fs;
    std::vector<cd> H(ctile);
    for (int k = 0; k < rb; k++) {
      const double w = kPi * (double)k / (double)(rb - 1);
      const double m = bw_bandpass(w, wlo, whi, 4);
      H[k] = m * m * (1.0 / (double)ctile);
    }
    if (ctile % 2 == 0) H[ctile / 2] = cd(H[ctile / 2].real(), 0.0);
    for (int k = rb; k < ctile; k++) H[k] = std::conj(H[ctile - k]);
    std::vector<cd> h = host_dft(H, +1);
    for (auto& v : h) v = cd(v.real(), 0.0);
    c_half = half_support(fs, 102.0, 1024, 6144);
    c_out = kNc - 2 * c_half;
    std::vector<cd> blk;
    c_tail = place_kernel(h, c_half, c_half, kNc, blk);
    std::vector<cd> G = host_dft(blk, -1);
    gc.resize(kNc);
    for (int k = 0; k < kNc; k++) gc[k] = (float)(G[k].real() / kNc);
  }

  tw_a = twiddles(kNa);
  tw_b = twiddles(kNb);
  tw_c = twiddles(kNc);
  tw_line = twiddles(fmt.line_fft);
  het_scale = (fmt.fsc + fmt.chroma_under) / fmt.output_rate;
  fsc_bin = (int)(fmt.fsc / fmt.output_rate * fmt.line_fft + 0.5);
  bw_bins = (int)(500000.0 / fmt.output_rate * fmt.line_fft + 0.5);
  if (bw_bins < 10) bw_bins = 10;
}

}  // namespace cuvhs

namespace cuvhs {

void Design::build_cached(const Format& fmt) {
  static std::mutex mu;
  static std::map<std::pair<double, int>, Design> cache;
  std::lock_guard<std::mutex> lock(mu);
  const std::pair<double, int> key(fmt.fs_hz, fmt.system);
  auto it = cache.find(key);
  if (it == cache.end()) {
    Design d;
    d.build(fmt);
    it = cache.emplace(key, std::move(d)).first;
  }
  *this = it->second;
}

}  // namespace cuvhs
