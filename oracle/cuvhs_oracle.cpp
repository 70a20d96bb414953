// FP64 CPU oracle of the cuVHS decode -- TEST INFRASTRUCTURE ONLY.
//
// A restatement of the reference decoder (hunterschuler/cuVHS) in plain C++,
// stage by stage, with the reference's tiling and host logic, so that the
// tests can check the CUDA product against it and bench.py can time it on the
// host cores.  The product never links or calls this file.  Citations are
// reference file:line.
#include "cuvhs_oracle.h"

#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <climits>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "oracle_fft.h"

namespace oracle {
namespace {

constexpr double PI = 3.14159265358979323846;
constexpr double TAU = 2.0 * PI;
constexpr int OVERLAP = 2048;            // fm_demod.cu:17
constexpr int MAX_PULSES = 800;          // sync_pulses.h:6
constexpr int MAX_DO = 512;              // dropout_detect.h:5
constexpr int FIELD_MARGIN_LINES = 20;   // pipeline.cu:1339
enum { PULSE_HSYNC = 0, PULSE_EQ1 = 1, PULSE_VSYNC = 2, PULSE_EQ2 = 3 };  // line_locs.h

template <typename F>
void parallel_for(int n, int threads, F fn) {
  if (threads <= 1 || n <= 1) {
    for (int i = 0; i < n; i++) fn(i);
    return;
  }
  std::atomic<int> next(0);
  std::vector<std::thread> pool;
  int nt = std::min(threads, n);
  for (int t = 0; t < nt; t++)
    pool.emplace_back([&] {
      for (;;) {
        int i = next.fetch_add(1);
        if (i >= n) break;
        fn(i);
      }
    });
  for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------- format
// VideoFormat::VideoFormat (video_format.cpp:23-104), NTSC and PAL branches.
struct Format {
  bool pal = false;
  double sample_rate;
  int lines_per_frame = 525, lines_per_field = 263;
  double line_rate = 15734.264;
  double fsc = 3579545.0;
  double chroma_under = (525.0 * (30.0 / 1.001)) * 40.0;
  double burst_abs_ref = 4416.0, burst_start_us = 5.3, burst_end_us = 7.8;
  int output_line_len = 910, output_field_lines = 263;
  int num_eq_pulses = 6, field_lines_first = 263, field_lines_second = 262;
  double hz_ire, ire0, vsync_ire;
  double sync_tip_hz, pulse_threshold_hz;
  double output_zero, output_scale;
  int active_line_start = 10;
  double output_rate;
  int samples_per_line, samples_per_field;
  double hsync_width, eq_pulse_width, bp_width, vsync_width;

  explicit Format(double mhz, bool is_pal = false) : pal(is_pal), sample_rate(mhz * 1e6) {
    if (!pal) {
      hz_ire = 1e6 / 140.0;
      ire0 = 4.4e6 - (hz_ire * 100.0);
      vsync_ire = -40.0;
    } else {
      lines_per_frame = 625;
      lines_per_field = 313;
      line_rate = 15625.0;
      fsc = 4433618.75;
      chroma_under = ((625.0 * 25.0) * 40.0) + 1953.0;
      burst_abs_ref = 5000.0;
      burst_start_us = 5.6;
      burst_end_us = 7.85;
      output_line_len = 1135;
      output_field_lines = 313;
      num_eq_pulses = 5;
      field_lines_first = 312;
      field_lines_second = 313;
      vsync_ire = -0.3 * (100.0 / 0.7);
      hz_ire = 1e6 / (100.0 + (-vsync_ire));
      ire0 = 4.8e6 - (hz_ire * 100.0);
    }
    sync_tip_hz = ire0 + hz_ire * vsync_ire;
    pulse_threshold_hz = ire0 + hz_ire * (-20.0);
    if (!pal) {
      output_zero = 1024.0;
      output_scale = (51200.0 - 1024.0) / (100.0 - vsync_ire);
      active_line_start = 10;
    } else {
      output_zero = 256.0;
      output_scale = (54016.0 - 256.0) / (100.0 - vsync_ire);
      active_line_start = 8;
    }
    output_rate = 4.0 * fsc;
    samples_per_line = (int)std::round(sample_rate / line_rate);
    samples_per_field = samples_per_line * lines_per_field;
    hsync_width = 4.7e-6 * sample_rate;
    eq_pulse_width = 2.3e-6 * sample_rate;
    bp_width = 1.5e-6 * sample_rate;
    vsync_width = (pal ? 27.3e-6 : 27.1e-6) * sample_rate;
  }
};

int next_7smooth(int n) {  // fm_demod.cu:22-33
  auto ok = [](int m) {
    for (int p : {2, 3, 5, 7}) while (m % p == 0) m /= p;
    return m == 1;
  };
  while (!ok(n)) n++;
  return n;
}

// ------------------------------------------------- filter design (fm_demod.cu:35-127)
double lpf_mag(double w, double wc, int order) {
  if (wc <= 0.0 || wc >= PI) return 1.0;
  double tc = std::tan(wc / 2.0);
  if (tc == 0.0) return 1.0;
  double t = std::tan(w / 2.0);
  double ratio = t / tc;
  return 1.0 / std::sqrt(1.0 + std::pow(ratio, 2.0 * order));
}
double hpf_mag(double w, double wc, int order) {
  if (w <= 0.0) return 0.0;
  if (wc <= 0.0 || wc >= PI) return 1.0;
  double tc = std::tan(wc / 2.0);
  double t = std::tan(w / 2.0);
  if (t == 0.0) return 0.0;
  double ratio = tc / t;
  return 1.0 / std::sqrt(1.0 + std::pow(ratio, 2.0 * order));
}
double bpf_mag(double w, double wl, double wh, int order) {
  if (w <= 0.0 || w >= PI) return 0.0;
  double tl = std::tan(wl / 2.0), th = std::tan(wh / 2.0), t = std::tan(w / 2.0);
  double bw = th - tl;
  if (bw <= 0.0 || t == 0.0) return 0.0;
  double s = (t * t - tl * th) / (bw * t);
  return 1.0 / std::sqrt(1.0 + std::pow(s, 2.0 * order));
}
double supergauss(double f, double fc, int order) {
  double ln2_half = std::log(2.0) / 2.0;
  double scale = std::pow(ln2_half, 1.0 / (2.0 * order));
  double x = 2.0 * f * scale / fc;
  return std::exp(-2.0 * std::pow(x, 2.0 * order));
}
void shelf_high(double f0, double db, double fs, double q, double b[3], double a[3]) {
  double A = std::pow(10.0, db / 40.0);
  double w0 = TAU * f0 / fs;
  double alpha = std::sin(w0) / (2.0 * q);
  double c = std::cos(w0);
  double sa = std::sqrt(A);
  b[0] = A * ((A + 1) + (A - 1) * c + 2 * sa * alpha);
  b[1] = -2 * A * ((A - 1) + (A + 1) * c);
  b[2] = A * ((A + 1) + (A - 1) * c - 2 * sa * alpha);
  a[0] = (A + 1) - (A - 1) * c + 2 * sa * alpha;
  a[1] = 2 * ((A - 1) - (A + 1) * c);
  a[2] = (A + 1) - (A - 1) * c - 2 * sa * alpha;
}
cplx biquad_resp(const double num[3], const double den[3], double w) {
  cplx z1 = std::exp(cplx(0.0, -w));
  cplx z2 = z1 * z1;
  cplx nn = num[0] + num[1] * z1 + num[2] * z2;
  cplx dd = den[0] + den[1] * z1 + den[2] * z2;
  return nn / dd;
}
std::vector<double> hamming_sinc(int taps, double cut) {
  std::vector<double> h(taps);
  double alpha = (taps - 1) / 2.0, sum = 0.0;
  for (int n = 0; n < taps; n++) {
    double m = n - alpha;
    double s = (std::fabs(m) < 1e-12) ? cut : std::sin(PI * cut * m) / (PI * m);
    double w = 0.54 - 0.46 * std::cos(TAU * n / (taps - 1));
    h[n] = s * w;
    sum += h[n];
  }
  for (int n = 0; n < taps; n++) h[n] /= sum;
  return h;
}
cplx fir_resp(const std::vector<double>& h, double w, int delay) {
  cplx acc(0.0, 0.0);
  for (size_t n = 0; n < h.size(); n++) acc += h[n] * std::exp(cplx(0.0, -(double)n * w));
  if (delay > 0) acc *= std::exp(cplx(0.0, w * delay));
  return acc;
}

// Demod filter set: FMDemodState::init (fm_demod.cu:273-374).
struct DemodFilters {
  int fs = 0, fb = 0;
  std::vector<double> rf;
  std::vector<cplx> fv, fv05;
};
void design_demod(const Format& fmt, int spp, DemodFilters& F) {
  F.fs = next_7smooth(spp + OVERLAP);
  F.fb = F.fs / 2 + 1;
  const int fb = F.fb;
  double fs = fmt.sample_rate, ny = fs / 2.0;
  double wbl = PI * 1300000.0 / ny, wbh = PI * 7500000.0 / ny;
  double wl = PI * 8000000.0 / ny, wh = PI * 1000000.0 / ny;
  F.rf.resize(fb);
  for (int k = 0; k < fb; k++) {
    double w = PI * (double)k / (double)(fb - 1);
    double hil = (k == 0 || k == fb - 1) ? 1.0 : 2.0;
    F.rf[k] = bpf_mag(w, wbl, wbh, 8) * lpf_mag(w, wl, 8) * hpf_mag(w, wh, 8) * hil;
  }
  double bs[3], as[3];
  shelf_high(273755.82, 13.9794, fs, 0.462088186, bs, as);
  auto fir = hamming_sinc(65, 500000.0 / ny);
  double inv_n = 1.0 / (double)F.fs;
  F.fv.resize(fb);
  F.fv05.resize(fb);
  for (int k = 0; k < fb; k++) {
    double w = PI * (double)k / (double)(fb - 1);
    double f_hz = (double)k * ny / (double)(fb - 1);
    cplx de = biquad_resp(as, bs, w);  // inverted shelf = de-emphasis
    double v = supergauss(f_hz, 3000000.0, 9);
    cplx sy = fir_resp(fir, w, 32);
    F.fv[k] = de * v * inv_n;
    F.fv05[k] = de * v * sy * inv_n;
  }
}

// ---------------------------------------------------------------- state
struct ChromaState {  // chroma_decode.h:9-15
  bool valid = false;
  int current_track = 0;
  double good_metric_threshold = 0.0;
  int cycle_start = 0;
};

struct FieldMeta {
  bool is_first = true;
  int phase_id = 0;
  size_t file_loc = 0;
  std::vector<int> dl, ds, de;
};

struct ChunkRec {
  long long meta[6] = {0, 0, 0, 0, 0, 0};
  std::vector<int> vsync, k2c, k2s, k2l, k2bc, k2bs, k2bl, k2bt, is_first, doc, dol, dos, doe;
  std::vector<long long> offs;
  std::vector<double> ll_coarse, ll, demod, demod05, env, cpre;
};

}  // namespace
}  // namespace oracle

struct oracle_ctx {
  oracle::Format fmt;
  int batch;
  int threads;
  bool keep_signals = false;
  int in_fmt = 0;         // 0 u8, 1 s16, 2 u16
  bool dc_correct = false;
  bool single_pass = false;  // K3 line locations in place of K2b (as CUVHS_K2B_DISABLE)
  oracle::DemodFilters filt;
  int spp;
  // carried state (pipeline.h:92-97, chroma_decode.h:9-15, pipeline.cu:2575)
  int k2b_prev_first_field = -1;
  int k2b_prev_progressive_field = -1;
  long long k2b_prev_first_hsync_readloc = -1;
  double k2b_prev_first_hsync_loc = -1.0;
  double k2b_prev_first_hsync_diff = -1.0;
  oracle::ChromaState cstate;
  bool last_parity = true;
  // results
  std::vector<uint16_t> luma, chroma;
  std::vector<oracle::FieldMeta> meta;
  std::vector<oracle::ChunkRec> chunks;
  std::string json;
  oracle_ctx(double mhz, bool pal) : fmt(mhz, pal) {}
};

namespace oracle {
namespace {

// ======================================================== K1 FM demod
// fm_demod (fm_demod.cu:396-485): overlap-save tiles of fs samples at stride spp.
void fm_demod(oracle_ctx* c, const std::vector<double>& raw, int T, std::vector<double>& demod,
              std::vector<double>& demod05, std::vector<double>& env) {
  const DemodFilters& F = c->filt;
  const int fs = F.fs, fb = F.fb, spp = c->spp;
  const long long total_src = (long long)T * spp;
  demod.assign((size_t)total_src, 0.0);
  demod05.assign((size_t)total_src, 0.0);
  env.assign((size_t)total_src, 0.0);
  RealFFT rfft(fs);
  ComplexFFT cfft(fs);
  const double scale = c->fmt.sample_rate / TAU;
  // Part A: RF band-pass x Hilbert weight -> analytic -> envelope, phase step.
  parallel_for(T, c->threads, [&](int f) {
    std::vector<double> x(fs);
    std::vector<cplx> X(fb), full(fs), a(fs), work(std::max(rfft.work_size(), (size_t)fs));
    for (int j = 0; j < fs; j++) {  // k_copy_and_pad (fm_demod.cu:133-153)
      long long s = (long long)f * spp + j - OVERLAP;
      x[j] = s < 0 ? raw[0] : (s < total_src ? raw[(size_t)s] : raw[(size_t)total_src - 1]);
    }
    rfft.forward(x.data(), X.data(), work.data());
    for (int k = 0; k < fs; k++) full[k] = k < fb ? X[k] * F.rf[k] : cplx(0.0, 0.0);
    cfft.run(full.data(), a.data(), work.data(), true);
    double* out = demod.data() + (size_t)f * spp;
    double* ev = env.data() + (size_t)f * spp;
    double prev = std::atan2(a[OVERLAP - 1].imag(), a[OVERLAP - 1].real());
    for (int i = 0; i < spp; i++) {
      const cplx& z = a[OVERLAP + i];
      ev[i] = std::sqrt(z.real() * z.real() + z.imag() * z.imag());
      double cur = std::atan2(z.imag(), z.real());
      double d = cur - prev;  // k_unwrap_to_hz (fm_demod.cu:222-244)
      if (d > PI) d -= TAU;
      if (d < -PI) d += TAU;
      out[i] = d * scale;
      prev = cur;
    }
  });
  // Part B: video (de-emphasis x 3 MHz super-Gaussian) and sync (x 0.5 MHz FIR).
  std::vector<double> vid((size_t)total_src), syn((size_t)total_src);
  parallel_for(T, c->threads, [&](int f) {
    std::vector<double> z(fs), y(fs);
    std::vector<cplx> Z(fb), V(fb), work(rfft.work_size());
    for (int j = 0; j < fs; j++) {
      long long s = (long long)f * spp + j - OVERLAP;
      z[j] = s < 0 ? demod[0] : (s < total_src ? demod[(size_t)s] : demod[(size_t)total_src - 1]);
    }
    rfft.forward(z.data(), Z.data(), work.data());
    for (int pass = 0; pass < 2; pass++) {
      const std::vector<cplx>& H = pass ? F.fv05 : F.fv;
      for (int k = 0; k < fb; k++) {  // k_apply_complex_filter (fm_demod.cu:246-257)
        V[k] = cplx(Z[k].real() * H[k].real() - Z[k].imag() * H[k].imag(),
                    Z[k].real() * H[k].imag() + Z[k].imag() * H[k].real());
      }
      rfft.inverse(V.data(), y.data(), work.data());
      double* dst = (pass ? syn.data() : vid.data()) + (size_t)f * spp;
      for (int i = 0; i < spp; i++) {  // k_trim (fm_demod.cu:155-169)
        int si = i + OVERLAP;
        if (si >= fs) si = fs - 1;
        dst[i] = y[si];
      }
    }
  });
  demod.swap(vid);
  demod05.swap(syn);
}

// ======================================================== VSYNC discovery
// k_discover_vsyncs (vsync_discover.cu:5-45) as a serial scan.
std::vector<int> discover_vsyncs(const std::vector<double>& s05, long long total, const Format& fmt) {
  int minw = (int)(20.0e-6 * fmt.sample_rate), maxw = (int)(35.0e-6 * fmt.sample_rate);
  double thr = fmt.pulse_threshold_hz;
  std::vector<int> out;
  for (long long i = 0; i < total; i++) {
    bool start = s05[i] <= thr && (i == 0 || s05[i - 1] > thr);
    if (!start) continue;
    int w = 0;
    while (i + w < total && s05[i + w] <= thr && w <= maxw) w++;
    if (w >= minw && w <= maxw) out.push_back((int)i);
  }
  return out;
}

// ======================================================== K2 sync pulses
// k_find_pulses (sync_pulses.cu:10-58).  Samples past the demodulated range
// (the reference reads stale device memory there) read as "not in pulse".
int find_pulses(const std::vector<double>& s05, long long total, size_t off, int spp, double thr,
                int* starts, int* lengths) {
  auto at = [&](long long i) { return i < total ? s05[(size_t)i] : 1e300; };
  bool in_pulse = at((long long)off) <= thr;
  int cur = 0, count = 0;
  for (int i = 0; i < spp; i++) {
    double v = at((long long)off + i);
    if (in_pulse) {
      if (v > thr) {
        int len = i - cur;
        if (len > 0 && cur != 0 && count < MAX_PULSES) {
          starts[count] = (int)(off + cur);
          lengths[count] = len;
          count++;
        }
        in_pulse = false;
      }
    } else if (v <= thr) {
      cur = i;
      in_pulse = true;
    }
  }
  return count;
}

// ======================================================== K2b host line locations
// pipeline.cu:410-893, restated.
struct Pulse { int start = 0, len = 0; };
struct VPulse { int type = PULSE_HSYNC; Pulse p; bool good = false; };
struct Timings { double hmin, hmax, emin, emax, vmin, vmax, hnom; };
struct Anchor {
  bool valid = false;
  double line0loc = 0, first_hsync_loc = 0, first_hsync_line = 0, next_field = 0;
  int first_field = -1, progressive_field = 0;
  double prev_hsync_diff = -1.0;
};

bool inrange(double v, double lo, double hi) { return v >= lo && v <= hi; }  // :432-434
double round_line(double x) { return std::round(0.5 * std::round(x / 0.5) * 10.0) / 10.0; }  // :436-438

bool qualitycheck(int pt, int t, int delta, int linelen) {  // :133-148
  double lo, hi;
  if (pt > 0 && t > 0) { lo = 0.4; hi = 0.6; }
  else if (pt == 0 && t == 0) { lo = 0.9; hi = 1.1; }
  else { lo = 0.4; hi = 1.1; }
  double span = (double)delta / (double)linelen;
  return span >= lo && span <= hi;
}

Timings line_timings(const int* lens, int n, const Format& fmt) {  // :450-477
  Timings t;
  double tol = fmt.sample_rate * 0.5e-6;
  double gmin = fmt.hsync_width - 3.5 * tol, gmax = fmt.hsync_width + 4.0 * tol;
  double sum = 0.0;
  int cnt = 0;
  int npc = std::max(0, std::min(n, MAX_PULSES));
  for (int i = 0; i < npc; i++) {
    double l = (double)lens[i];
    if (l >= gmin && l <= gmax) { sum += l; cnt++; }
  }
  double est = cnt > 0 ? (sum / cnt) : fmt.hsync_width;
  double off = est - fmt.hsync_width;
  t.hnom = fmt.hsync_width + off;
  t.hmin = t.hnom - tol;
  t.hmax = t.hnom + tol;
  t.emin = fmt.eq_pulse_width + off - tol;
  t.emax = fmt.eq_pulse_width + off + tol;
  t.vmin = (fmt.vsync_width + off) * 0.5;
  t.vmax = fmt.vsync_width + off + 2.0 * tol;
  return t;
}

double mean_line_len(const std::vector<VPulse>& vp, double nominal) {  // :479-517
  int lstart = -1, llen = -1, cstart = -1, clen = 0;
  for (int i = 0; i < (int)vp.size(); i++) {
    if (vp[i].type != PULSE_HSYNC) {
      if (cstart >= 0 && clen > llen) { lstart = cstart; llen = clen; }
      cstart = -1;
      clen = 0;
    } else if (cstart < 0) {
      cstart = i;
      clen = 0;
    } else {
      clen++;
    }
  }
  if (cstart >= 0 && clen > llen) { lstart = cstart; llen = clen; }
  std::vector<double> lens;
  if (lstart >= 1 && llen >= 1) {
    for (int i = lstart + 1; i < lstart + llen; i++) {
      double l = (double)(vp[i].p.start - vp[i - 1].p.start);
      double r = l / nominal;
      if (r >= 0.95 && r <= 1.05) lens.push_back(l);
    }
  }
  if (lens.empty()) return nominal;
  double s = 0.0;
  for (double x : lens) s += x;
  return s / (double)lens.size();
}

bool vblank_machine(const std::vector<Pulse>& raw, size_t start, const Timings& lt, int npulses,
                    int linelen, std::vector<VPulse>& out) {  // :519-609
  bool done = false;
  double half = npulses / 2.0;
  int vsync_start = -1;
  double state_end = 0.0, state_len = -1.0;
  for (size_t i = start; i < raw.size() && i < start + 26; i++) {
    const Pulse& p = raw[i];
    VPulse sp;
    bool have = false;
    int state = out.empty() ? -1 : out.back().type;
    double len = (double)p.len;
    if (state == -1) {
      if (inrange(len, lt.hmin, lt.hmax)) { sp = {PULSE_HSYNC, p, false}; have = true; }
    } else if (state == PULSE_HSYNC) {
      if (inrange(len, lt.hmin, lt.hmax)) { sp = {PULSE_HSYNC, p, false}; have = true; }
      else if (inrange(len, lt.emin, lt.emax)) { sp = {PULSE_EQ1, p, false}; state_len = half; have = true; }
      else if (inrange(len, lt.vmin, lt.vmax)) { vsync_start = (int)out.size() - 1; sp = {PULSE_VSYNC, p, false}; have = true; }
    } else if (state == PULSE_EQ1) {
      if (inrange(len, lt.emin, lt.emax)) { sp = {PULSE_EQ1, p, false}; have = true; }
      else if (inrange(len, lt.vmin, lt.vmax)) { vsync_start = (int)out.size() - 1; sp = {PULSE_VSYNC, p, false}; state_len = half; have = true; }
      else if (inrange(len, lt.hmin, lt.hmax)) { sp = {PULSE_HSYNC, p, false}; have = true; }
    } else if (state == PULSE_VSYNC) {
      if (inrange(len, lt.emin, lt.emax)) { sp = {PULSE_EQ2, p, false}; state_len = half; have = true; }
      else if (inrange(len, lt.vmin, lt.vmax)) { sp = {PULSE_VSYNC, p, false}; have = true; }
      else if ((double)p.start > state_end && inrange(len, lt.hmin, lt.hmax)) { sp = {PULSE_HSYNC, p, false}; have = true; }
    } else if (state == PULSE_EQ2) {
      if (inrange(len, lt.emin, lt.emax)) { sp = {PULSE_EQ2, p, false}; have = true; }
      else if (inrange(len, lt.hmin, lt.hmax)) { sp = {PULSE_HSYNC, p, false}; have = true; done = true; }
    }
    if (have && sp.type != state) {
      if ((double)sp.p.start < state_end) {
        have = false;
      } else if (state_len > 0.0) {
        state_end = (double)sp.p.start + ((state_len - 0.1) * (double)linelen);
        state_len = -1.0;
      }
    }
    if (have) {
      sp.good = out.empty() ? false : qualitycheck(out.back().type, sp.type, sp.p.start - out.back().p.start, linelen);
      out.push_back(sp);
    }
    if (done && vsync_start >= 0) return true;
  }
  return done;
}

std::vector<VPulse> refine_pulses(const int* starts, const int* lens, int count, const Format& fmt) {  // :611-648
  std::vector<VPulse> vp;
  int npc = std::max(0, std::min(count, MAX_PULSES));
  if (npc <= 0) return vp;
  Timings lt = line_timings(lens, npc, fmt);
  std::vector<Pulse> raw((size_t)npc);
  for (int i = 0; i < npc; i++) raw[i] = {starts[i], lens[i]};
  for (int i = 0; i < npc;) {
    Pulse cur = raw[i];
    if (inrange((double)cur.len, lt.hmin, lt.hmax)) {
      bool good = !vp.empty() && qualitycheck(vp.back().type, PULSE_HSYNC, cur.start - vp.back().p.start, fmt.samples_per_line);
      vp.push_back({PULSE_HSYNC, cur, good});
      i++;
    } else if (i > 2 && inrange((double)cur.len, lt.emin, lt.emax) && !vp.empty() && vp.back().type == PULSE_HSYNC) {
      std::vector<VPulse> seq = vp;
      bool done = vblank_machine(raw, (size_t)(i - 2), lt, fmt.num_eq_pulses, fmt.samples_per_line, seq);
      if (done && seq.size() > vp.size()) {
        vp = seq;
        // As in the reference, the index advance is computed after the
        // assignment, so it always advances by exactly one (pipeline.cu:636-639).
        i += (int)(seq.size() - vp.size()) + 1;
        i = std::min(i, npc);
      } else {
        i++;
      }
    } else {
      i++;
    }
  }
  return vp;
}

Anchor first_hsync(const std::vector<VPulse>& vp, double mll, const Format& fmt, int prev_first_field,
                   double last_off_lines, double prev_loc, double prev_diff, int confidence) {  // :650-855
  Anchor out;
  if (vp.empty() || mll <= 0.0) return out;
  const int field_lines[2] = {fmt.field_lines_first, fmt.field_lines_second};
  const double TOL = 0.5;
  double fol[4] = {-1, -1, -1, -1};
  int vbp[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
  double vbl[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
  int last = -1, group = 0, fgroup = 0;
  for (int i = 0; i < (int)vp.size(); i++) {
    if (last != -1 && vp[i].good) {
      if (group == 0 && vp[i].p.start > vp[0].p.start + field_lines[0] * mll) {
        group = 4;
        fgroup = 2;
      }
      int lt = vp[last].type, t = vp[i].type;
      if (lt == PULSE_HSYNC && t > PULSE_HSYNC) {
        vbp[0 + group] = vp[i].p.start;
        fol[0 + fgroup] = round_line((vp[i].p.start - vp[last].p.start) / mll);
      } else if (lt == PULSE_EQ1 && t == PULSE_VSYNC) {
        vbp[1 + group] = vp[i].p.start;
      } else if (lt == PULSE_VSYNC && t == PULSE_EQ2) {
        vbp[2 + group] = vp[i].p.start;
      } else if (lt > PULSE_HSYNC && t == PULSE_HSYNC) {
        vbp[3 + group] = vp[last].p.start;
        fol[1 + fgroup] = round_line((vp[i].p.start - vp[last].p.start) / mll);
      }
    }
    last = i;
  }
  double ffl[4] = {1, 0.5, 0.5, 1}, sfl[4] = {0.5, 1, 1, 0.5}, pfl[4] = {1, 0.5, 1, 0.5};
  if (fmt.pal) {  // pipeline.cu:711-715
    const double pf[4] = {0.5, 0.5, 1, 1}, ps[4] = {1, 1, 0.5, 0.5}, pp[4] = {0.5, 0.5, 0.5, 0.5};
    for (int i = 0; i < 4; i++) {
      ffl[i] = pf[i];
      sfl[i] = ps[i];
      pfl[i] = pp[i];
    }
  }
  double ic = 0.0, id = 0.0, pc = 0.0, pd = 0.0;
  for (int i = 0; i < 4; i++) {
    double fl = fol[i];
    if (fl == ffl[i]) { ic += 1.0; id += 1.0; }
    if (fl == sfl[i]) id += 1.0;
    if (fl == pfl[i]) { pc += 1.0; pd += 1.0; }
    if (fl != -1) pd += 1.0;
  }
  (void)pc;
  (void)pd;
  bool first_field;
  if (prev_first_field == -1)
    first_field = id == 0.0 || std::round(ic / std::max(1.0, id)) == 1.0;
  else
    first_field = !prev_first_field;
  if (id > 0.0) {
    if (prev_loc < 0.0) confidence = std::min(confidence, 50);
    double wgt = id / 4.0;
    int ffc = (int)std::llround((ic / id) * wgt * 100.0);
    int sfc = (int)std::llround(((id - ic) / id) * wgt * 100.0);
    if (ffc >= confidence && ffc > sfc) first_field = true;
    else if (sfc >= confidence && sfc > ffc) first_field = false;
  }
  double vsl = fmt.num_eq_pulses / 2.0;
  double cur_lines = first_field ? field_lines[0] : field_lines[1];
  double prev_lines = first_field ? field_lines[1] : field_lines[0];
  double* cfl = first_field ? ffl : sfl;
  vbl[0] = 0.0 + cfl[0];
  vbl[1] = vbl[0] + vsl;
  vbl[2] = vbl[1] + vsl;
  vbl[3] = vbl[2] + vsl - 0.5;
  double hsl = vbl[3] + cfl[1];
  vbl[4] = cur_lines + cfl[2];
  vbl[5] = vbl[4] + vsl;
  vbl[6] = vbl[5] + vsl;
  vbl[7] = vbl[6] + vsl - 0.5;
  auto calc = [&](int a, int b, double& loc, int& cnt, double& off) {
    int fp = vbp[a], sp = vbp[b];
    if (fp == -1 || sp == -1 || mll == 0.0) return;
    double actual = ((double)fp - (double)sp) / mll;
    double expect = vbl[a] - vbl[b];
    if (actual < expect + TOL && actual > expect - TOL) {
      off += actual - expect;
      loc += (double)sp + mll * (hsl - vbl[b]);
      cnt += 1;
    }
  };
  double f_loc = 0.0, f_off = 0.0, l_loc = 0.0, l_off = 0.0;
  int f_cnt = 0, l_cnt = 0;
  const int fi[4] = {0, 1, 2, 3}, li[4] = {4, 5, 6, 7};
  for (int a = 0; a < 4; a++) for (int b = a + 1; b < 4; b++) calc(fi[a], fi[b], f_loc, f_cnt, f_off);
  for (int a = 0; a < 4; a++) for (int b = a + 1; b < 4; b++) calc(li[a], li[b], l_loc, l_cnt, l_off);
  double loc = 0.0, off = 0.0;
  int cnt = 0;
  double fe = f_cnt ? f_loc / f_cnt : 0.0, le = l_cnt ? l_loc / l_cnt : 0.0;
  if (f_cnt && l_cnt && fe < le + TOL * mll && fe > le - TOL * mll) {
    loc = f_loc + l_loc;
    cnt = f_cnt + l_cnt;
    off = f_off + l_off;
    for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++) calc(fi[a], li[b], loc, cnt, off);
  } else if (f_cnt == 6 || (prev_loc <= 0.0 && f_cnt > l_cnt)) {
    loc = f_loc; cnt = f_cnt; off = f_off;
  } else if (l_cnt == 6 || (prev_loc <= 0.0 && l_cnt > f_cnt)) {
    loc = l_loc; cnt = l_cnt; off = l_off;
  }
  double est_lines = fmt.pal ? cur_lines : prev_lines;  // pipeline.cu:811
  int est_loc = (int)std::llround((last_off_lines + est_lines + prev_loc / mll) * mll);
  bool used_est = false;
  if (cnt == 0 && prev_loc > 0.0) {
    double ewo = (prev_diff <= 0.5 && prev_diff >= -0.5) ? est_loc + mll * prev_diff : (double)est_loc;
    if (ewo <= 0.0) ewo = vp.empty() ? 0.0 : (double)vp.front().p.start;
    loc += ewo;
    cnt += 1;
    used_est = true;
  }
  if (cnt <= 0) return out;
  off /= cnt;
  loc = std::round((loc + off) / cnt);
  if (!used_est) prev_diff = (loc - est_loc) / mll;
  double hoff = 0.0;
  int hcnt = 0;
  for (const VPulse& p : vp) {
    if (p.type != PULSE_HSYNC || !p.good) continue;
    double ll = ((double)p.p.start - loc) / mll + hsl;
    int rl = (int)std::llround(ll);
    if (rl > cur_lines) break;
    if (rl >= hsl) {
      hoff += loc + mll * ((double)rl - hsl) - (double)p.p.start;
      hcnt++;
    }
  }
  if (hcnt > 0) {
    hoff /= hcnt;
    loc -= hoff;
  }
  out.valid = true;
  out.line0loc = loc - mll * hsl;
  out.first_hsync_loc = loc;
  out.first_hsync_line = hsl;
  out.next_field = loc + mll * (vbl[4] - hsl);
  out.first_field = first_field ? 1 : 0;
  out.progressive_field = 0;
  out.prev_hsync_diff = prev_diff;
  return out;
}

std::vector<double> pulses_to_linelocs(const std::vector<VPulse>& vp, double ref_pulse, double ref_line,
                                       double mll, int nlines) {  // :857-893
  std::vector<double> locs((size_t)nlines, 0.0);
  std::vector<double> ps;
  for (const VPulse& p : vp) ps.push_back((double)p.p.start);
  std::sort(ps.begin(), ps.end());
  double max_allowed = mll / 1.5;
  size_t cur = 0;
  for (int line = 0; line < nlines; line++) {
    locs[line] = ref_pulse + mll * ((double)line - ref_line);
    if (cur >= ps.size()) continue;
    double cd = std::fabs(ps[cur] - locs[line]);
    double best = max_allowed, pos = -1.0;
    size_t si = cur;
    while (si + 1 < ps.size()) {
      if (cd <= best) { best = cd; cur = si; pos = ps[si]; }
      double nd = std::fabs(ps[si + 1] - locs[line]);
      if (nd > cd) break;
      cd = nd;
      si++;
    }
    if (pos >= 0.0) { locs[line] = pos; cur++; }
  }
  return locs;
}

// ======================================================== K4 hsync refine
// hsync_refine.cu:21-239.
double falling_cross(const double* s, int start, int count, double target, long long total) {
  if (start < 0 || start + count > total || count < 2) return -1.0;
  for (int i = start + 1; i < start + count; i++) {
    double p = s[i - 1], q = s[i];
    if (p >= target && q < target) {
      double a = p - target, b = q - target;
      double fr = (a - b != 0.0) ? (a / (a - b)) : 0.0;
      return (double)(i - 1) + fr;
    }
  }
  return -1.0;
}
double rising_cross(const double* s, int start, int count, double target, long long total) {
  if (start < 0 || start + count > total || count < 2) return -1.0;
  if (s[start] > target) return -1.0;
  for (int i = start + 1; i < start + count; i++) {
    double p = s[i - 1], q = s[i];
    if (p < target && q >= target) {
      double a = target - p, b = target - q;
      double fr = (a + b != 0.0) ? (a / (a - b)) : 0.0;
      return (double)(i - 1) + fr;
    }
  }
  return -1.0;
}
double window_median(const double* s, int start, int count, long long total) {
  if (start < 0 || start + count > total || count <= 0) return 0.0;
  int n = std::min(count, 64);
  double buf[64];
  for (int i = 0; i < n; i++) buf[i] = s[start + i];
  std::nth_element(buf, buf + n / 2, buf + n);
  return buf[n / 2];
}
void hsync_refine(const std::vector<double>& s05, std::vector<double>& ll, int P, long long total, const Format& fmt) {
  const double us = 1.0e-6 * fmt.sample_rate;
  const double redge = 2.25 * ((fmt.sample_rate / 1.0e6) / 40.0);
  const double hw = fmt.hsync_width, thr = fmt.pulse_threshold_hz;
  const double* s = s05.data();
  for (int f = 0; f < P; f++) {
    for (int line = fmt.active_line_start; line < fmt.lines_per_frame; line++) {
      double& loc = ll[(size_t)f * fmt.lines_per_frame + line];
      double orig = loc;
      int ou = (int)(us + 0.5);
      double zc = falling_cross(s, (int)(orig - ou), ou * 2, thr, total);
      double left = -1.0;
      if (zc >= 0.0) {
        int zi = (int)(zc + 0.5);
        double sl = window_median(s, zi + (int)(1.0 * us), (int)(1.5 * us), total);
        double pl = window_median(s, zi + (int)(8.0 * us), (int)(1.0 * us), total);
        if (pl > sl) {
          double mid = (sl + pl) / 2.0;
          double zc2 = falling_cross(s, (int)(orig - ou * 2), (int)(us * 4), mid, total);
          if (zc2 >= 0.0 && std::fabs(zc2 - zc) <= us * 0.5) left = zc2;
        }
      }
      double right = -1.0;
      int rs = (int)(orig + hw - us), rc = (int)(hw * 2);
      double rx = rising_cross(s, rs, rc, thr, total);
      if (rx >= 0.0) {
        double zfr = rx - hw;
        int zfi = (int)(zfr + 0.5);
        double rsl = window_median(s, zfi + (int)(1.0 * us), (int)(1.5 * us), total);
        double rpl = window_median(s, zfi + (int)(hw + 1.0 * us), (int)(1.0 * us), total);
        if (rpl > rsl) {
          double rmid = (rsl + rpl) / 2.0;
          double zc2r = rising_cross(s, (int)(orig + hw - us), (int)(hw * 2), rmid, total);
          if (zc2r >= 0.0 && std::fabs(zc2r - rx) <= us * 0.5) {
            double cand = rx - hw + redge;
            double ref = (left >= 0.0) ? left : orig;
            if (std::fabs(cand - ref) <= us * 2.0) right = cand;
          }
        }
      }
      if (right >= 0.0) loc = right;
      else if (left >= 0.0) loc = left;
    }
  }
}

// ======================================================== K5 TBC luma
// k_tbc_resample (tbc_resample.cu:19-133).
void tbc_resample(const std::vector<double>& demod, const std::vector<double>& ll, uint16_t* out, int P,
                  long long total, const Format& fmt) {
  const int W = fmt.output_line_len, H = fmt.output_field_lines, LPF = fmt.lines_per_frame;
  for (int f = 0; f < P; f++) {
    for (int r = 0; r < H; r++) {
      uint16_t* row = out + ((size_t)f * H + r) * W;
      if (r + 1 >= LPF) { for (int c = 0; c < W; c++) row[c] = (uint16_t)fmt.output_zero; continue; }
      double a0 = ll[(size_t)f * LPF + r], a1 = ll[(size_t)f * LPF + r + 1];
      double len = a1 - a0;
      for (int c = 0; c < W; c++) {
        double fr = (double)c / (double)W;
        double coord = a0 + fr * len;
        int ci = (int)coord;
        double x = coord - (double)ci;
        if (ci < 1 || ci + 2 >= total) { row[c] = (uint16_t)fmt.output_zero; continue; }
        double p0 = demod[ci - 1], p1 = demod[ci], p2 = demod[ci + 1], p3 = demod[ci + 2];
        double a = p2 - p0, b = 2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3, cc = 3.0 * (p1 - p2) + p3 - p0;
        double hz = p1 + 0.5 * x * (a + x * (b + x * cc));
        double ire = (hz - fmt.ire0) / fmt.hz_ire - fmt.vsync_ire;
        double v = ire * fmt.output_scale + fmt.output_zero;
        if (v < 0.0) v = 0.0;
        if (v > 65535.0) v = 65535.0;
        row[c] = (uint16_t)(v + 0.5);
      }
    }
  }
}

// ======================================================== K6 chroma
// chroma_decode.cu:13-1002.
struct PhaseEntry { int is_first, quadrant, delta, phase_id, offset; };
const PhaseEntry kPhaseTable[] = {  // chroma_decode.cu:337-351
    {1, 2, 0, 3, 0}, {0, 3, 1, 2, 1}, {1, 1, 2, 1, 1}, {0, 0, 3, 4, 0},
    {1, 0, 0, 3, 2}, {0, 1, 1, 2, 3}, {1, 3, 2, 1, 3}, {0, 2, 3, 4, 2},
    {1, 2, -1, 3, 0}, {0, 3, -1, 2, 1}, {1, 1, -1, 1, 1}, {0, 0, -1, 4, 0},
    {1, 0, -1, 3, 2}, {0, 1, -1, 2, 3}, {1, 3, -1, 1, 3}, {0, 2, -1, 4, 2},
};
int lookup_phase_id(int is_first, int quadrant, int delta) {  // :359-377
  for (const auto& e : kPhaseTable)
    if (e.is_first == is_first && e.quadrant == quadrant && e.delta == delta) return e.phase_id;
  for (const auto& e : kPhaseTable)
    if (e.is_first == is_first && e.quadrant == quadrant && e.delta == -1) return e.phase_id;
  return 1;
}

struct ChromaGeom {
  int W, H, LPF, fft, bins, fsc_bin, bw, b0, b1;
  double het_scale, fft_scale;
};

// Het + per-line FFT band-pass of `nfields` fields starting at `f0` into
// out[(f-f0)*H + line][1024] (k_resample_raw_het + D2Z + k_chroma_bandpass + Z2D).
void chroma_lines(const std::vector<double>& pre, const std::vector<double>& ll, long long total_raw,
                  const ChromaGeom& g, int f0, int nfields, const std::vector<int>& track,
                  std::vector<double>& out, int threads) {
  out.assign((size_t)nfields * g.H * g.fft, 0.0);
  RealFFT rf(g.fft);
  parallel_for(nfields * g.H, threads, [&](int li) {
    int f = f0 + li / g.H, r = li % g.H;
    std::vector<double> row(g.fft, 0.0);
    std::vector<cplx> X(g.bins), work(rf.work_size());
    if (r + 1 < g.LPF) {
      double a0 = ll[(size_t)f * g.LPF + r], a1 = ll[(size_t)f * g.LPF + r + 1];
      int rot = track[f] ? 1 : 3;
      int lp = (r * rot + 0) & 3;
      double poff = (double)lp * (PI * 0.5);
      for (int c = 0; c < g.W; c++) {
        double fr = (double)c / (double)g.W;
        double coord = a0 + fr * (a1 - a0);
        int ci = (int)coord;
        double x = coord - (double)ci;
        if (ci < 1 || ci + 2 >= total_raw) continue;
        double p0 = pre[ci - 1], p1 = pre[ci], p2 = pre[ci + 1], p3 = pre[ci + 2];
        double a = p2 - p0, b = 2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3, cc = 3.0 * (p1 - p2) + p3 - p0;
        double v = p1 + 0.5 * x * (a + x * (b + x * cc));
        double abs_sample = (double)(r * g.W + c);
        double het = -std::cos(2.0 * PI * g.het_scale * abs_sample + poff);
        row[c] = v * het;
      }
    }
    rf.forward(row.data(), X.data(), work.data());
    for (int k = 0; k < g.bins; k++)
      if (k < g.fsc_bin - g.bw || k > g.fsc_bin + g.bw) X[k] = cplx(0.0, 0.0);
    rf.inverse(X.data(), out.data() + (size_t)li * g.fft, work.data());
  });
}

// Host metric (measure_burst_cancellation, chroma_decode.cu:383-411).
double host_burst_metric(const double* h, const ChromaGeom& g) {
  const int SKIP = 16;
  int blen = g.b1 - g.b0;
  double total = 0.0;
  int count = 0;
  for (int line = SKIP; line < g.H - SKIP - 1; line += 2) {
    const double* a = h + (size_t)line * g.fft;
    const double* b = h + (size_t)(line + 1) * g.fft;
    double s = 0.0;
    for (int i = g.b0; i < g.b1 && i < g.W; i++) s += std::fabs(a[i] * g.fft_scale + b[i] * g.fft_scale);
    total += s / blen;
    count++;
  }
  return count > 0 ? total / count : 1e9;
}

// Device metric (k_burst_cancellation, chroma_decode.cu:242-296) with its
// 256-thread tree reduction order.
double device_burst_metric(const double* h, const ChromaGeom& g) {
  const int SKIP = 16;
  int blen = g.b1 - g.b0;
  if (blen <= 0) return 0.0;
  int npairs = (g.H - 2 * SKIP - 1) / 2;
  double sum[256];
  int cnt[256];
  for (int t = 0; t < 256; t++) {
    double ms = 0.0;
    int mc = 0;
    for (int pr = t; pr < npairs; pr += 256) {
      int line = SKIP + pr * 2;
      const double* a = h + (size_t)line * g.fft;
      const double* b = a + g.fft;
      double ps = 0.0;
      for (int i = g.b0; i < g.b1; i++) ps += std::fabs(a[i] * g.fft_scale + b[i] * g.fft_scale);
      ms += ps / blen;
      mc++;
    }
    sum[t] = ms;
    cnt[t] = mc;
  }
  for (int s = 128; s > 0; s >>= 1)
    for (int t = 0; t < s; t++) { sum[t] += sum[t + s]; cnt[t] += cnt[t + s]; }
  return cnt[0] > 0 ? sum[0] / cnt[0] : 1e9;
}

double host_burst_phase(const double* h, const ChromaGeom& g, const Format& fmt) {  // :415-450
  const int SKIP = 16;
  double It = 0.0, Qt = 0.0;
  for (int line = SKIP; line < g.H - SKIP; line++) {
    const double* d = h + (size_t)line * g.fft;
    double I = 0.0, Q = 0.0;
    for (int i = g.b0; i < g.b1 && i < g.W; i++) {
      double v = d[i] * g.fft_scale;
      double t = 2.0 * PI * fmt.fsc / fmt.output_rate * (double)i;
      I += v * std::cos(t);
      Q += v * std::sin(t);
    }
    double m = std::sqrt(I * I + Q * Q);
    if (m > 0.0) { It += I / m; Qt += Q / m; }
  }
  double ph = std::atan2(Qt, It);
  return std::fmod(ph * 180.0 / PI + 360.0, 360.0);
}

void chroma_decode(oracle_ctx* c, const std::vector<double>& raw, const std::vector<double>& ll,
                   std::vector<double>& pre, uint16_t* out, int P, std::vector<int>& phase_ids) {
  const Format& fmt = c->fmt;
  ChromaGeom g;
  g.W = fmt.output_line_len;
  g.H = fmt.output_field_lines;
  g.LPF = fmt.lines_per_frame;
  g.fft = 1;
  while (g.fft < g.W) g.fft <<= 1;
  g.bins = g.fft / 2 + 1;
  g.het_scale = (fmt.fsc + fmt.chroma_under) / fmt.output_rate;
  g.fsc_bin = (int)(fmt.fsc / fmt.output_rate * g.fft + 0.5);
  g.bw = (int)(500000.0 / fmt.output_rate * g.fft + 0.5);
  if (g.bw < 10) g.bw = 10;
  g.b0 = (int)(fmt.burst_start_us * 1e-6 * fmt.output_rate + 0.5);
  g.b1 = (int)(fmt.burst_end_us * 1e-6 * fmt.output_rate + 0.5);
  g.fft_scale = 1.0 / (double)g.fft;
  const long long total_raw = (long long)P * c->spp;
  const int stride = (int)(total_raw / P);
  // Step 0: colour-under pre-band-pass per tile, zero padded (chroma_decode.cu:568-633).
  const int R = next_7smooth(stride), rb = R / 2 + 1;
  std::vector<double> hb(rb);
  double wlo = 2.0 * PI * 60000.0 / fmt.sample_rate, whi = 2.0 * PI * 1200000.0 / fmt.sample_rate;
  for (int i = 0; i < rb; i++) {
    double w = PI * (double)i / (double)(rb - 1);
    double m = bpf_mag(w, wlo, whi, 4);
    hb[i] = m * m * (1.0 / (double)R);
  }
  pre.assign((size_t)total_raw, 0.0);
  {
    RealFFT rf(R);
    parallel_for(P, c->threads, [&](int f) {
      std::vector<double> x(R, 0.0), y(R);
      std::vector<cplx> X(rb), work(rf.work_size());
      size_t o = (size_t)f * stride;
      for (int i = 0; i < stride; i++) x[i] = raw[o + i];
      rf.forward(x.data(), X.data(), work.data());
      for (int k = 0; k < rb; k++) X[k] *= hb[k];
      rf.inverse(X.data(), y.data(), work.data());
      for (int i = 0; i < stride; i++) pre[o + i] = y[i];
    });
  }
  static const int cycle[8] = {3, 2, 1, 4, 3, 2, 1, 4};
  int det_track, cycle_start;
  double thr;
  std::vector<int> track(P, 0);
  if (c->cstate.valid) {
    det_track = c->cstate.current_track;
    thr = c->cstate.good_metric_threshold;
    cycle_start = c->cstate.cycle_start;
  } else {
    // Step 1-2: track and burst-phase detection on field 0 (chroma_decode.cu:684-743).
    std::vector<double> h;
    double metric[2];
    for (int t = 0; t < 2; t++) {
      track[0] = t;
      chroma_lines(pre, ll, total_raw, g, 0, 1, track, h, c->threads);
      metric[t] = host_burst_metric(h.data(), g);
    }
    det_track = (metric[1] < metric[0]) ? 1 : 0;
    thr = metric[det_track] * 4.0;
    track[0] = det_track;
    chroma_lines(pre, ll, total_raw, g, 0, 1, track, h, c->threads);
    double ph = host_burst_phase(h.data(), g, fmt);
    int q = ((int)(ph / 90.0 + 0.5)) % 4;
    int pid = lookup_phase_id(1, q, -1);
    cycle_start = 0;
    for (int i = 0; i < 8; i += 2)
      if (cycle[i] == pid) { cycle_start = i; break; }
  }
  int cur = det_track;
  phase_ids.assign(P, 0);
  for (int f = 0; f < P; f++) {
    track[f] = (f & 1) ? (1 - cur) : cur;
    phase_ids[f] = cycle[(cycle_start + f) % 8];
  }
  // Step 4: chunks of at most 15 fields with track-flip retries (chroma_decode.cu:782-981).
  int max_chunk_lines = (4096 / g.H) * g.H;
  int chunk_lines = std::min(max_chunk_lines, P * g.H);
  chunk_lines = (chunk_lines / g.H) * g.H;
  if (chunk_lines < g.H) chunk_lines = g.H;
  int fpc = chunk_lines / g.H;
  std::vector<double> h;
  for (int fs0 = 0; fs0 < P; fs0 += fpc) {
    int nf = std::min(fpc, P - fs0);
    int retries = 3;
    bool ok = false;
    while (!ok && retries-- > 0) {
      chroma_lines(pre, ll, total_raw, g, fs0, nf, track, h, c->threads);
      int first_bad = INT_MAX;
      for (int f = 0; f < nf; f++) {
        double m = device_burst_metric(h.data() + (size_t)f * g.H * g.fft, g);
        if (m > thr) { first_bad = f; break; }
      }
      if (first_bad == INT_MAX) {
        ok = true;
      } else {
        int af = fs0 + first_bad;
        cur = 1 - cur;
        for (int ff = af; ff < P; ff++) track[ff] = (ff & 1) ? (1 - cur) : cur;
      }
    }
    // ACC + u16 (k_chroma_acc_output, chroma_decode.cu:188-231).
    for (int li = 0; li < nf * g.H; li++) {
      const double* d = h.data() + (size_t)li * g.fft;
      uint16_t* o = out + ((size_t)fs0 * g.H + li) * g.W;
      int blen = g.b1 - g.b0;
      double ss = 0.0;
      for (int i = 0; i < blen; i++) {
        double v = d[g.b0 + i] * g.fft_scale;
        ss += v * v;
      }
      double rms = std::sqrt(ss / (double)blen);
      double acc = (rms > 1.0) ? (fmt.burst_abs_ref / rms) : 0.0;
      for (int col = 0; col < g.W; col++) {
        double v = d[col] * g.fft_scale * acc;
        double ov = v + 32768.0;
        if (ov < 0.0) ov = 0.0;
        if (ov > 65535.0) ov = 65535.0;
        o[col] = (uint16_t)(ov + 0.5);
      }
    }
  }
  c->cstate.valid = true;
  c->cstate.current_track = (P & 1) ? (1 - cur) : cur;
  c->cstate.good_metric_threshold = thr;
  c->cstate.cycle_start = (cycle_start + P) % 8;
}

// ======================================================== K7 dropouts
// dropout_detect.cu:17-291.
int find_tbc_line(const double* ll, int als, int n, double pos) {
  if (pos < ll[als] || pos >= ll[als + n]) return -1;
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) / 2;
    if (ll[als + mid] <= pos) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

void dropout_detect(const std::vector<double>& env, const std::vector<double>& llv, uint16_t* luma,
                    uint16_t* chroma, int P, int spp, const Format& fmt, std::vector<int>& cnt,
                    std::vector<int>& dl, std::vector<int>& ds, std::vector<int>& de) {
  cnt.assign(P, 0);
  dl.assign((size_t)P * MAX_DO, 0);
  ds.assign((size_t)P * MAX_DO, 0);
  de.assign((size_t)P * MAX_DO, 0);
  const int W = fmt.output_line_len, H = fmt.output_field_lines;
  for (int f = 0; f < P; f++) {
    // k_field_mean_env: 256-thread strided sums, warp shuffle tree, warp totals in order.
    const double* fe = env.data() + (size_t)f * spp;
    double tsum[256];
    for (int t = 0; t < 256; t++) {
      double s = 0.0;
      for (int i = t; i < spp; i += 256) s += fe[i];
      tsum[t] = s;
    }
    double wsum[8];
    for (int w = 0; w < 8; w++) {
      double v[32];
      for (int l = 0; l < 32; l++) v[l] = tsum[w * 32 + l];
      for (int o = 16; o > 0; o >>= 1)
        for (int l = 0; l < 32; l++) v[l] = v[l] + (l + o < 32 ? v[l + o] : v[l]);
      wsum[w] = v[0];
    }
    double total = 0.0;
    for (int w = 0; w < 8; w++) total += wsum[w];
    double mean = total / (double)spp;
    double down = mean * 0.18, up = down * 1.25;
    const double* ll = llv.data() + (size_t)f * fmt.lines_per_frame;
    int als = fmt.active_line_start;
    int fstart = f * spp;
    int s0 = std::max((int)ll[als], fstart);
    int s1 = std::min((int)ll[als + H], fstart + spp);
    if (s1 <= s0) continue;
    std::vector<int> rs, rend;
    int dstart = -1;
    int nb = (s1 - s0 + 16 - 1) / 16;
    for (int bk = 0; bk < nb; bk++) {
      int b0 = s0 + bk * 16, b1 = std::min(b0 + 16, s1);
      double bs = 0.0;
      for (int i = b0; i < b1; i++) bs += env[i];
      double bm = bs / (double)(b1 - b0);
      if (bm <= down) {
        if (dstart < 0) dstart = b0;
      } else if (bm >= up) {
        if (dstart >= 0) {
          if (!rs.empty() && dstart - rend.back() <= 30) rend.back() = b0;
          else if ((int)rs.size() < 128) { rs.push_back(dstart); rend.push_back(b0); }
          dstart = -1;
        }
      }
    }
    if (dstart >= 0) {
      if (!rs.empty() && dstart - rend.back() <= 30) rend.back() = s1;
      else if ((int)rs.size() < 128) { rs.push_back(dstart); rend.push_back(s1); }
    }
    std::vector<int> fs_, fe_;
    for (size_t i = 0; i < rs.size(); i++)
      if (rend[i] - rs[i] >= 10) { fs_.push_back(rs[i]); fe_.push_back(rend[i]); }
    int n = 0;
    int* ol = dl.data() + (size_t)f * MAX_DO;
    int* os = ds.data() + (size_t)f * MAX_DO;
    int* oe = de.data() + (size_t)f * MAX_DO;
    for (size_t i = 0; i < fs_.size() && n < MAX_DO; i++) {
      double a = (double)fs_[i], b = (double)fe_[i];
      int sl = find_tbc_line(ll, als, H, a);
      if (sl < 0) continue;
      int el = find_tbc_line(ll, als, H, b - 1.0);
      if (el < 0) el = H - 1;
      for (int l = sl; l <= el && n < MAX_DO; l++) {
        double l0 = ll[als + l], l1 = ll[als + l + 1], len = l1 - l0;
        if (len <= 0.0) continue;
        int sx = (l == sl) ? std::max(0, (int)((a - l0) / len * (double)W)) : 0;
        int ex = (l == el) ? std::min(W, (int)((b - l0) / len * (double)W + 0.999)) : W;
        if (ex > sx) { ol[n] = l; os[n] = sx; oe[n] = ex; n++; }
      }
    }
    cnt[f] = n;
    // k_conceal: entries of one warp copy in lock-step (load all, then store all,
    // per column step); warps in order.
    uint16_t* lf = luma + (size_t)f * H * W;
    uint16_t* cf = chroma + (size_t)f * H * W;
    for (int w0 = 0; w0 < n; w0 += 32) {
      int w1 = std::min(n, w0 + 32);
      int maxlen = 0;
      for (int d = w0; d < w1; d++) maxlen = std::max(maxlen, oe[d] - os[d]);
      for (int it = 0; it < maxlen; it++) {
        uint16_t vl[32], vc[32];
        bool act[32];
        for (int d = w0; d < w1; d++) {
          int line = ol[d], src = line > 0 ? line - 1 : line + 1, col = os[d] + it;
          act[d - w0] = src < H && col < oe[d];
          if (act[d - w0]) { vl[d - w0] = lf[src * W + col]; vc[d - w0] = cf[src * W + col]; }
        }
        for (int d = w0; d < w1; d++) {
          if (!act[d - w0]) continue;
          int col = os[d] + it;
          lf[ol[d] * W + col] = vl[d - w0];
          cf[ol[d] * W + col] = vc[d - w0];
        }
      }
    }
  }
}

// ======================================================== writer JSON
// TBCWriter::write_json (tbc_writer.cpp:89-175).
std::string make_json(const Format& fmt, const std::vector<FieldMeta>& meta) {
  std::string s;
  char buf[256];
  auto add = [&](const char* f, ...) {};
  (void)add;
  double black = (0.0 - fmt.vsync_ire) * fmt.output_scale + fmt.output_zero;
  double white = (100.0 - fmt.vsync_ire) * fmt.output_scale + fmt.output_zero;
  int bs = (int)(fmt.burst_start_us * 1e-6 * fmt.output_rate + 0.5);
  int be = (int)(fmt.burst_end_us * 1e-6 * fmt.output_rate + 0.5);
  s += fmt.pal ? "{\n  \"videoParameters\": {\n    \"system\": \"PAL\",\n    \"isSubcarrierLocked\": false,\n    \"isSourcePal\": true,\n"
               : "{\n  \"videoParameters\": {\n    \"system\": \"NTSC\",\n    \"isSubcarrierLocked\": false,\n    \"isSourcePal\": false,\n";
  snprintf(buf, sizeof buf, "    \"numberOfSequentialFields\": %d,\n", (int)meta.size()); s += buf;
  snprintf(buf, sizeof buf, "    \"black16bIre\": %.1f,\n", black); s += buf;
  snprintf(buf, sizeof buf, "    \"white16bIre\": %.1f,\n", white); s += buf;
  snprintf(buf, sizeof buf, "    \"sampleRate\": %.0f,\n", fmt.output_rate); s += buf;
  snprintf(buf, sizeof buf, "    \"fieldWidth\": %d,\n    \"fieldHeight\": %d,\n", fmt.output_line_len, fmt.output_field_lines); s += buf;
  snprintf(buf, sizeof buf, "    \"colourBurstStart\": %d,\n    \"colourBurstEnd\": %d,\n", bs, be); s += buf;
  snprintf(buf, sizeof buf, "    \"activeVideoStart\": %d,\n    \"activeVideoEnd\": %d,\n", fmt.pal ? 185 : 134,
           fmt.pal ? 1107 : 894);  // tbc_writer.cpp:107-108
  s += buf;
  s += "    \"tapeFormat\": \"VHS\",\n    \"isMapped\": false\n  },\n";
  s += "  \"fields\": [\n";
  for (size_t i = 0; i < meta.size(); i++) {
    const FieldMeta& m = meta[i];
    s += "    {\n";
    snprintf(buf, sizeof buf, "      \"isFirstField\": %s,\n      \"seqNo\": %d,\n      \"fileLoc\": %zu,\n",
             m.is_first ? "true" : "false", (int)i + 1, m.file_loc);
    s += buf;
    if (m.phase_id > 0) { snprintf(buf, sizeof buf, "      \"fieldPhaseID\": %d,\n", m.phase_id); s += buf; }
    s += "      \"dropOuts\": {\n        \"fieldLine\": [";
    for (size_t j = 0; j < m.dl.size(); j++) { snprintf(buf, sizeof buf, "%s%d", j ? ", " : "", m.dl[j]); s += buf; }
    s += "],\n        \"startx\": [";
    for (size_t j = 0; j < m.ds.size(); j++) { snprintf(buf, sizeof buf, "%s%d", j ? ", " : "", m.ds[j]); s += buf; }
    s += "],\n        \"endx\": [";
    for (size_t j = 0; j < m.de.size(); j++) { snprintf(buf, sizeof buf, "%s%d", j ? ", " : "", m.de[j]); s += buf; }
    s += "]\n      }\n";
    s += (i + 1 < meta.size()) ? "    },\n" : "    }\n";
  }
  s += "  ]\n}\n";
  return s;
}

// ======================================================== K3 line locations
// line_locs() (line_locs.cu:544-593): the device line locator the reference
// runs instead of K2b when CUVHS_K2B_DISABLE is set.  Phase 1 writes nominal
// width classes into the pulse-type list (k_classify_pulses, :18-49); phase 2
// (k_compute_linelocs, :62-543) works per field from adaptive classes.  The
// device compiler fuses a + b * c into one rounding; std::fma restates that.
void k3_classify(const int* lens, int npc, const Format& fmt, int* types) {  // :18-49, :551-558
  double tol = 0.5e-6 * fmt.sample_rate;
  double hmin = fmt.hsync_width - tol, hmax = fmt.hsync_width + tol;
  double emin = fmt.eq_pulse_width - tol, emax = fmt.eq_pulse_width + tol;
  double vmin = fmt.vsync_width * 0.5, vmax = fmt.vsync_width + 1.0e-6 * fmt.sample_rate;
  for (int p = 0; p < npc && p < MAX_PULSES; p++) {
    double len = (double)lens[p];
    int t;
    if (len >= vmin && len <= vmax) t = PULSE_VSYNC;
    else if (len >= hmin && len <= hmax) t = PULSE_HSYNC;
    else if (len >= emin && len <= emax) t = PULSE_EQ1;
    else t = PULSE_HSYNC;
    types[p] = t;
  }
}

void k3_linelocs(const int* starts, const int* lengths, int npc, const Format& fmt, double* locs,
                 int* is_first) {  // :62-543
  const double tol = 0.5e-6 * fmt.sample_rate;
  const double inlinelen = (double)fmt.samples_per_line;
  const double hnom = fmt.hsync_width, enom = fmt.eq_pulse_width, vnom = fmt.vsync_width;
  double gmin = std::fma(-3.5, tol, hnom), gmax = std::fma(4.0, tol, hnom);
  double hs = 0.0;
  int hc = 0;
  for (int i = 0; i < npc; i++) {
    double len = (double)lengths[i];
    if (len >= gmin && len <= gmax) { hs += len; hc++; }
  }
  double est = (hc > 0) ? (hs / hc) : hnom;
  double off = est - hnom;
  double ahmin = hnom + off - tol, ahmax = hnom + off + tol;
  double aemin = enom + off - tol, aemax = enom + off + tol;
  double avmin = (vnom + off) * 0.5, avmax = std::fma(2.0, tol, vnom + off);
  int types[800];
  int n = npc < 800 ? npc : 800;
  for (int i = 0; i < n; i++) {
    double len = (double)lengths[i];
    if (len >= avmin && len <= avmax) types[i] = PULSE_VSYNC;
    else if (len >= ahmin && len <= ahmax) types[i] = PULSE_HSYNC;
    else if (len >= aemin && len <= aemax) types[i] = PULSE_EQ1;
    else types[i] = PULSE_HSYNC;
  }
  int ref = -1, last_h = -1, first_eq1 = -1, last_eq2 = -1, state = -1;
  for (int i = 0; i < n; i++) {  // :148-201
    int t = types[i];
    if (state == -1) {
      if (t == PULSE_HSYNC) { state = PULSE_HSYNC; last_h = i; }
    } else if (state == PULSE_HSYNC) {
      if (t == PULSE_HSYNC) last_h = i;
      else if (t == PULSE_EQ1) { state = PULSE_EQ1; first_eq1 = i; }
      else if (t == PULSE_VSYNC) state = PULSE_VSYNC;
    } else if (state == PULSE_EQ1) {
      if (t == PULSE_VSYNC) state = PULSE_VSYNC;
      else if (t == PULSE_HSYNC) { state = PULSE_HSYNC; last_h = i; first_eq1 = -1; }
    } else if (state == PULSE_VSYNC) {
      if (t == PULSE_EQ1) { state = PULSE_EQ2; last_eq2 = i; }
      else if (t == PULSE_HSYNC) { ref = i; break; }
    } else if (state == PULSE_EQ2) {
      if (t == PULSE_EQ1) last_eq2 = i;
      else if (t == PULSE_HSYNC) { if (last_eq2 < 0) last_eq2 = i - 1; ref = i; break; }
    }
  }
  int parity = -1;  // :203-236
  if (ref >= 0 && last_h >= 0 && first_eq1 >= 0) {
    double el = (double)(starts[first_eq1] - starts[last_h]) / inlinelen;
    parity = !fmt.pal ? (el > 0.75 ? 1 : 0) : (el > 0.75 ? 0 : 1);
  }
  if (parity < 0 && ref >= 0 && last_eq2 >= 0) {
    double xl = (double)(starts[ref] - starts[last_eq2]) / inlinelen;
    parity = !fmt.pal ? (xl > 0.75 ? 1 : 0) : (xl > 0.75 ? 0 : 1);
  }
  *is_first = parity;
  int brs = -1, brl = 0, crs = -1, crl = 0;  // :246-284
  for (int i = 0; i < n; i++) {
    if (types[i] == PULSE_HSYNC) {
      if (crs == -1) { crs = i; crl = 1; } else crl++;
    } else {
      if (crl > brl) { brs = crs; brl = crl; }
      crs = -1;
      crl = 0;
    }
  }
  if (crl > brl) { brs = crs; brl = crl; }
  double mll = inlinelen;
  if (brl >= 2) {
    double sum = 0.0;
    int cnt = 0;
    for (int i = brs + 1; i < brs + brl; i++) {
      double sp = (double)(starts[i] - starts[i - 1]);
      if (sp >= inlinelen * 0.95 && sp <= inlinelen * 1.05) { sum += sp; cnt++; }
    }
    if (cnt > 0) mll = sum / cnt;
  }
  double ref_pos, ref_line;  // :295-337
  if (ref >= 0) {
    ref_pos = (double)starts[ref];
    ref_line = 10.0;
    if (ref > n / 2) {
      double corr = ref_pos - (double)fmt.samples_per_field;
      if (corr > 0.0) ref_pos = corr;
    }
  } else {
    ref = 0;
    for (int i = 0; i < n; i++) if (types[i] == PULSE_HSYNC) { ref = i; break; }
    ref_pos = (double)starts[ref];
    ref_line = 0.0;
  }
  int ms[800], ml[800], mc = 0;  // :365-399
  double tiny = hnom * 0.75, sgap = inlinelen * 0.25;
  for (int i = 0; i < n && mc < 800; i++) {
    bool sur = false;
    if ((types[i] == PULSE_EQ1 || types[i] == PULSE_EQ2) && i + 1 < n && types[i + 1] == PULSE_HSYNC &&
        (double)lengths[i + 1] <= tiny && (double)(starts[i + 1] - starts[i]) <= sgap)
      sur = true;
    bool sup = false;
    if (types[i] == PULSE_HSYNC && (double)lengths[i] <= tiny && i > 0 &&
        (types[i - 1] == PULSE_EQ1 || types[i - 1] == PULSE_EQ2) && (double)(starts[i] - starts[i - 1]) <= sgap)
      sup = true;
    if (sur || (types[i] == PULSE_HSYNC && !sup)) { ms[mc] = starts[i]; ml[mc] = lengths[i]; mc++; }
  }
  int hsl[800], nh = 0;  // :401-425
  double dgap = inlinelen * 0.75;
  int c0 = 0;
  while (c0 < mc && nh < 800) {
    int bi = c0;
    double bs = std::fabs((double)ml[c0] - hnom);
    int c1 = c0 + 1;
    while (c1 < mc && (double)(ms[c1] - ms[c0]) < dgap) {
      double sc = std::fabs((double)ml[c1] - hnom);
      if (sc < bs || (sc == bs && ms[c1] < ms[bi])) { bi = c1; bs = sc; }
      c1++;
    }
    hsl[nh++] = ms[bi];
    c0 = c1;
  }
  double maxd = mll / 1.5;  // :429-470
  int cur = 0;
  for (int line = 0; line < fmt.lines_per_frame; line++) {
    double expected = std::fma(mll, (double)line - ref_line, ref_pos);
    locs[line] = expected;
    if (cur >= nh) continue;
    double bd = maxd;
    int bp = -1, sidx = cur;
    while (sidx < nh) {
      double d = std::fabs((double)hsl[sidx] - expected);
      if (d <= bd) { bd = d; bp = hsl[sidx]; cur = sidx; }
      if (sidx + 1 < nh) {
        double nd = std::fabs((double)hsl[sidx + 1] - expected);
        if (nd > d) break;
      } else {
        break;
      }
      sidx++;
    }
    if (bp >= 0) { locs[line] = (double)bp; cur++; }
  }
}

// ======================================================== chunk driver
// Pipeline::process_chunk (pipeline.cu:1525-2624).
int process_chunk(oracle_ctx* c, const uint8_t* data, size_t n, size_t raw_offset, int num_fields,
                  size_t& next_raw_offset) {
  const Format& fmt = c->fmt;
  const size_t spf = fmt.samples_per_field;
  const int spp = c->spp;
  const size_t total_samples = (size_t)num_fields * spp;
  size_t n_read = raw_offset < n ? std::min(total_samples, n - raw_offset) : 0;
  if (n_read < spf) return 0;
  // RawReader::convert (src/io/raw_reader.cpp:71-99): per-format conversion,
  // then the mean of the samples read subtracted; the zero fill past them is
  // applied after (pipeline.cu:1539-1541)
  std::vector<double> raw(total_samples, 0.0);
  for (size_t i = 0; i < n_read; i++) {
    const size_t k = raw_offset + i;
    if (c->in_fmt == 1) raw[i] = (double)reinterpret_cast<const int16_t*>(data)[k];
    else if (c->in_fmt == 2) raw[i] = (double)reinterpret_cast<const uint16_t*>(data)[k] - 32768.0;
    else raw[i] = ((double)data[k] - 128.0) * 256.0;
  }
  if (c->dc_correct && n_read > 0) {
    double sum = 0.0;
    for (size_t i = 0; i < n_read; i++) sum += raw[i];
    const double mean = sum / (double)n_read;
    for (size_t i = 0; i < n_read; i++) raw[i] -= mean;
  }
  int T = (int)(n_read / spf);
  if (T > num_fields) T = num_fields;
  if (T == 0) return 0;
  ChunkRec rec;
  std::vector<double> demod, s05, env;
  fm_demod(c, raw, T, demod, s05, env);
  const long long total_chunk = (long long)T * spp;
  std::vector<int> cand = discover_vsyncs(s05, total_chunk, fmt);
  std::sort(cand.begin(), cand.end());
  rec.vsync = cand;
  std::vector<size_t> offs;
  for (int pos : cand) {
    if (offs.empty() || ((size_t)pos - offs.back() > (size_t)(fmt.samples_per_field / 2))) {
      size_t safe = (pos > 5 * fmt.samples_per_line) ? (size_t)(pos - 5 * fmt.samples_per_line) : 0;
      offs.push_back(safe);
    }
  }
  if (offs.empty())
    for (int i = 0; i < T; i++) offs.push_back((size_t)i * spf);
  int P = (int)offs.size();
  if (P > num_fields) { P = num_fields; offs.resize(P); }
  size_t actual_spf = spf;
  if (offs.size() >= 2) actual_spf = (offs.back() - offs.front()) / (offs.size() - 1);
  size_t pred = offs.back() + actual_spf, margin = 10 * (size_t)fmt.samples_per_line;
  next_raw_offset = pred > margin ? raw_offset + pred - margin : raw_offset + pred;
  rec.offs.assign(offs.begin(), offs.end());
  // K2 + K2b (pipeline.cu:1686-1807)
  rec.k2c.assign(P, 0);
  rec.k2s.assign((size_t)P * MAX_PULSES, 0);
  rec.k2l.assign((size_t)P * MAX_PULSES, 0);
  for (int f = 0; f < P; f++)
    rec.k2c[f] = find_pulses(s05, total_chunk, offs[f], spp, fmt.pulse_threshold_hz,
                             rec.k2s.data() + (size_t)f * MAX_PULSES, rec.k2l.data() + (size_t)f * MAX_PULSES);
  const int LPF = fmt.lines_per_frame;
  std::vector<double> ll((size_t)P * LPF);
  std::vector<int> is_first(P);
  rec.k2bc.assign(P, 0);
  rec.k2bs.assign((size_t)P * MAX_PULSES, 0);
  rec.k2bl.assign((size_t)P * MAX_PULSES, 0);
  rec.k2bt.assign((size_t)P * MAX_PULSES, PULSE_HSYNC);
  // pipeline.cu:1694: the switch is read on every chunk
  const bool k2b_disabled = c->single_pass || std::getenv("CUVHS_K2B_DISABLE") != nullptr;
  for (int f = 0; f < P && k2b_disabled; f++) {  // pipeline.cu:1848-1856: K3 leaves the pulses as found
    int npc = std::max(0, std::min(rec.k2c[f], MAX_PULSES));
    const int* ps = rec.k2s.data() + (size_t)f * MAX_PULSES;
    const int* pl = rec.k2l.data() + (size_t)f * MAX_PULSES;
    std::copy(ps, ps + npc, rec.k2bs.begin() + (size_t)f * MAX_PULSES);
    std::copy(pl, pl + npc, rec.k2bl.begin() + (size_t)f * MAX_PULSES);
    k3_classify(pl, npc, fmt, rec.k2bt.data() + (size_t)f * MAX_PULSES);
    rec.k2bc[f] = npc;
    k3_linelocs(ps, pl, npc, fmt, ll.data() + (size_t)f * LPF, &is_first[f]);
  }
  for (int f = 0; f < P && !k2b_disabled; f++) {
    int before = std::max(0, std::min(rec.k2c[f], MAX_PULSES));
    const int* ps = rec.k2s.data() + (size_t)f * MAX_PULSES;
    std::vector<VPulse> vp = refine_pulses(ps, rec.k2l.data() + (size_t)f * MAX_PULSES, before, fmt);
    double mll = mean_line_len(vp, (double)fmt.samples_per_line);
    double prev_off = 0.0;
    if (c->k2b_prev_first_hsync_readloc != -1 && mll > 0.0)
      prev_off = ((double)c->k2b_prev_first_hsync_readloc - (double)(raw_offset + offs[f])) / mll;
    Anchor an = first_hsync(vp, mll, fmt, c->k2b_prev_first_field, prev_off, c->k2b_prev_first_hsync_loc,
                            c->k2b_prev_first_hsync_diff, 75);
    int after = std::min((int)vp.size(), MAX_PULSES);
    for (int i = 0; i < after; i++) {
      rec.k2bs[(size_t)f * MAX_PULSES + i] = vp[i].p.start;
      rec.k2bl[(size_t)f * MAX_PULSES + i] = vp[i].p.len;
      rec.k2bt[(size_t)f * MAX_PULSES + i] = vp[i].type;
    }
    rec.k2bc[f] = after;
    std::vector<double> locs;
    if (an.valid) {
      locs = pulses_to_linelocs(vp, an.first_hsync_loc, an.first_hsync_line, mll, LPF);
      is_first[f] = an.first_field;
      c->k2b_prev_first_field = an.first_field;
      c->k2b_prev_progressive_field = an.progressive_field;
      c->k2b_prev_first_hsync_readloc = (long long)(raw_offset + offs[f]);
      c->k2b_prev_first_hsync_loc = an.first_hsync_loc;
      c->k2b_prev_first_hsync_diff = an.prev_hsync_diff;
    } else {
      locs.resize(LPF);
      double ref = before > 0 ? (double)ps[0] : 0.0;
      for (int line = 0; line < LPF; line++) locs[line] = ref + mll * (double)line;
      is_first[f] = (c->k2b_prev_first_field >= 0) ? (1 - c->k2b_prev_first_field) : 1;
    }
    std::copy(locs.begin(), locs.end(), ll.begin() + (size_t)f * LPF);
  }
  rec.ll_coarse = ll;
  const long long totalP = (long long)P * spp;
  // K4-K7
  hsync_refine(s05, ll, P, totalP, fmt);
  rec.ll = ll;
  const size_t F = (size_t)fmt.output_line_len * fmt.output_field_lines;
  std::vector<uint16_t> luma((size_t)P * F), chroma((size_t)P * F);
  tbc_resample(demod, ll, luma.data(), P, totalP, fmt);
  std::vector<double> pre;
  std::vector<int> phase_ids;
  chroma_decode(c, raw, ll, pre, chroma.data(), P, phase_ids);
  dropout_detect(env, ll, luma.data(), chroma.data(), P, spp, fmt, rec.doc, rec.dol, rec.dos, rec.doe);
  rec.is_first = is_first;
  // Output + parity (pipeline.cu:2575-2610)
  for (int i = 0; i < P; i++) {
    FieldMeta m;
    m.file_loc = raw_offset + offs[i];
    bool ff;
    if (is_first[i] >= 0 && (is_first[i] == 1) != c->last_parity) ff = (is_first[i] == 1);
    else ff = !c->last_parity;
    c->last_parity = ff;
    m.is_first = ff;
    if (i < (int)phase_ids.size() && phase_ids[i] > 0) m.phase_id = phase_ids[i];
    for (int d = 0; d < rec.doc[i]; d++) {
      m.dl.push_back(rec.dol[(size_t)i * MAX_DO + d]);
      m.ds.push_back(rec.dos[(size_t)i * MAX_DO + d]);
      m.de.push_back(rec.doe[(size_t)i * MAX_DO + d]);
    }
    c->meta.push_back(m);
  }
  c->luma.insert(c->luma.end(), luma.begin(), luma.end());
  c->chroma.insert(c->chroma.end(), chroma.begin(), chroma.end());
  rec.meta[0] = (long long)raw_offset;
  rec.meta[1] = P;
  rec.meta[2] = spp;
  rec.meta[3] = T;
  rec.meta[4] = num_fields;
  rec.meta[5] = (long long)next_raw_offset;
  if (c->keep_signals && c->chunks.empty()) {
    rec.demod = demod;
    rec.demod05 = s05;
    rec.env = env;
    rec.cpre = pre;
  }
  c->chunks.push_back(std::move(rec));
  return P;
}

}  // namespace
}  // namespace oracle

extern "C" {

oracle_ctx* oracle_create_system(double mhz, int batch_fields, int threads, int system) {
  oracle_ctx* c = new oracle_ctx(mhz, system == 1);
  c->batch = batch_fields > 0 ? batch_fields : 1;
  c->threads = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
  c->spp = c->fmt.samples_per_field + oracle::FIELD_MARGIN_LINES * c->fmt.samples_per_line;
  oracle::design_demod(c->fmt, c->spp, c->filt);
  return c;
}

oracle_ctx* oracle_create(double mhz, int batch_fields, int threads) {
  return oracle_create_system(mhz, batch_fields, threads, 0);
}

int oracle_field_width(const oracle_ctx* c) { return c->fmt.output_line_len; }
int oracle_field_height(const oracle_ctx* c) { return c->fmt.output_field_lines; }
int oracle_lines_per_frame(const oracle_ctx* c) { return c->fmt.lines_per_frame; }

void oracle_destroy(oracle_ctx* c) { delete c; }
void oracle_keep_signals(oracle_ctx* c, int keep) { c->keep_signals = keep != 0; }
void oracle_set_single_pass(oracle_ctx* c, int on) { c->single_pass = on != 0; }

void oracle_set_input(oracle_ctx* c, int format, int dc_correct) {
  c->in_fmt = format;
  c->dc_correct = dc_correct != 0;
}

int oracle_decode(oracle_ctx* c, const uint8_t* data, size_t n) {
  c->luma.clear();
  c->chroma.clear();
  c->meta.clear();
  c->chunks.clear();
  size_t raw_offset = 0;
  const size_t spf = c->fmt.samples_per_field;
  while (true) {
    if (raw_offset >= n) break;
    size_t remaining = n - raw_offset;
    int remaining_fields = (int)(remaining / spf);
    if (remaining_fields <= 0) break;
    int nf = std::min(c->batch, remaining_fields);
    size_t next = 0;
    int done = oracle::process_chunk(c, data, n, raw_offset, nf, next);
    if (done == 0) break;
    raw_offset = next;
  }
  c->json = oracle::make_json(c->fmt, c->meta);
  return (int)c->meta.size();
}

int oracle_num_fields(const oracle_ctx* c) { return (int)c->meta.size(); }
const uint16_t* oracle_luma(const oracle_ctx* c) { return c->luma.data(); }
const uint16_t* oracle_chroma(const oracle_ctx* c) { return c->chroma.data(); }
const char* oracle_json(const oracle_ctx* c) { return c->json.c_str(); }
int oracle_num_chunks(const oracle_ctx* c) { return (int)c->chunks.size(); }
void oracle_chunk_meta(const oracle_ctx* c, int k, long long meta[6]) {
  for (int i = 0; i < 6; i++) meta[i] = c->chunks[k].meta[i];
}

long long oracle_chunk_array(const oracle_ctx* c, int k, const char* name, void* dst, long long cap) {
  if (k < 0 || k >= (int)c->chunks.size()) return -1;
  const oracle::ChunkRec& r = c->chunks[k];
  auto put_i = [&](const std::vector<int>& v) -> long long {
    if (dst) std::memcpy(dst, v.data(), sizeof(int) * (size_t)std::min<long long>(cap, (long long)v.size()));
    return (long long)v.size();
  };
  auto put_d = [&](const std::vector<double>& v) -> long long {
    if (dst) std::memcpy(dst, v.data(), sizeof(double) * (size_t)std::min<long long>(cap, (long long)v.size()));
    return (long long)v.size();
  };
  std::string s(name);
  if (s == "vsync_candidates") return put_i(r.vsync);
  if (s == "field_offsets") {
    if (dst) std::memcpy(dst, r.offs.data(), sizeof(long long) * (size_t)std::min<long long>(cap, (long long)r.offs.size()));
    return (long long)r.offs.size();
  }
  if (s == "k2_pulse_count") return put_i(r.k2c);
  if (s == "k2_pulse_starts") return put_i(r.k2s);
  if (s == "k2_pulse_lengths") return put_i(r.k2l);
  if (s == "k2b_pulse_count") return put_i(r.k2bc);
  if (s == "k2b_pulse_starts") return put_i(r.k2bs);
  if (s == "k2b_pulse_lengths") return put_i(r.k2bl);
  if (s == "k2b_pulse_types") return put_i(r.k2bt);
  if (s == "is_first") return put_i(r.is_first);
  if (s == "do_count") return put_i(r.doc);
  if (s == "do_lines") return put_i(r.dol);
  if (s == "do_starts") return put_i(r.dos);
  if (s == "do_ends") return put_i(r.doe);
  if (s == "linelocs_coarse") return put_d(r.ll_coarse);
  if (s == "linelocs") return put_d(r.ll);
  if (s == "demod") return put_d(r.demod);
  if (s == "demod05") return put_d(r.demod05);
  if (s == "envelope") return put_d(r.env);
  if (s == "chroma_prefilt") return put_d(r.cpre);
  return -1;
}

}  // extern "C"
