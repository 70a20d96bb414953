// Seeded synthetic NTSC or PAL VHS RF generator.
//
// Produces an 8-bit RF capture of the kind cuVHS decodes: an FM luma carrier
// (NTSC: sync tip 3.4 MHz, white 4.4 MHz; PAL: 3.8 / 4.8 MHz; the IRE maps of
// src/format/video_format.cpp:23-104 of the reference) carrying the system's
// timing (hsync 4.7 us; NTSC 6 + 6 + 6 EQ / broad / EQ half-line pulses of
// 2.3 us and a 5.3-7.8 us burst, PAL 5 + 5 + 5 of 2.35 us and a 5.6-7.85 us
// burst; broad pulses with 4.7 us serrations), pre-emphasised with the same
// high-shelf biquad the decoder inverts (src/pipeline/fm_demod.cu:310-314), plus
// a colour-under chroma signal at 40 fH with the VHS +/-90 degree per-line
// rotation that src/pipeline/chroma_decode.cu:143-148 undoes.  Noise, a bounded
// per-line timebase random walk, amplitude-collapse dropouts, a head-switch
// time jump and slow speed drift are all seeded and deterministic: the same
// parameters give byte-identical output on any machine and thread count.
#include "cuvhs_synth.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

// Timing and levels of the video system.
struct Timing {
  bool pal;
  double line_rate;
  double chroma_under;  // colour-under carrier, Hz
  double hz_ire, ire0, sync_ire;
  int frame_lines;      // 525 / 625: field 2 starts at half-line frame_lines
  int eq_pulses;        // half-line pulses per EQ or broad group (6 / 5)
  double eq_us, half_line_us;
  double burst_a, burst_b;  // burst window, us after the line's sync
  int burst_line;           // first field line with a burst
  int pic_first, pic_last;  // field lines with picture
  double pic_a, pic_b;      // picture window, us
  int bars_end, sine_end;   // field lines of the colour bars and the sine pattern
  int headswitch_lines[2];  // frame lines of the head-switch jumps (6 lines before each vertical interval)
  double start_lines;       // range of the seeded start line within a frame
};

Timing timing(int system) {
  Timing t;
  if (system == 1) {
    t.pal = true;
    t.line_rate = 15625.0;
    t.chroma_under = ((625.0 * 25.0) * 40.0) + 1953.0;
    t.sync_ire = -0.3 * (100.0 / 0.7);
    t.hz_ire = 1e6 / (100.0 - t.sync_ire);
    t.ire0 = 4.8e6 - t.hz_ire * 100.0;
    t.frame_lines = 625;
    t.eq_pulses = 5;
    t.eq_us = 2.35;
    t.half_line_us = 32.0;
    t.burst_a = 5.6;
    t.burst_b = 7.85;
    t.burst_line = 8;
    t.pic_first = 23;
    t.pic_last = 310;
    t.pic_a = 10.5;
    t.pic_b = 62.0;
    t.bars_end = 200;
    t.sine_end = 240;
    t.headswitch_lines[0] = 619;
    t.headswitch_lines[1] = 306;
    t.start_lines = 580.0;
  } else {
    t.pal = false;
    t.line_rate = 15734.264;
    t.chroma_under = (525.0 * (30.0 / 1.001)) * 40.0;
    t.hz_ire = 1e6 / 140.0;
    t.ire0 = 4.4e6 - t.hz_ire * 100.0;
    t.sync_ire = -40.0;
    t.frame_lines = 525;
    t.eq_pulses = 6;
    t.eq_us = 2.3;
    t.half_line_us = 31.777;
    t.burst_a = 5.3;
    t.burst_b = 7.8;
    t.burst_line = 9;
    t.pic_first = 20;
    t.pic_last = 262;
    t.pic_a = 9.4;
    t.pic_b = 62.4;
    t.bars_end = 170;
    t.sine_end = 200;
    t.headswitch_lines[0] = 519;
    t.headswitch_lines[1] = 256;
    t.start_lines = 480.0;
  }
  return t;
}

// SplitMix64: counter-based stream so every block of samples has its own
// reproducible generator.
struct SplitMix {
  uint64_t s;
  explicit SplitMix(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double gauss() {
    double u1 = uniform();
    double u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
  }
};

uint64_t mix_seed(uint64_t a, uint64_t b) {
  SplitMix m(a * 0x632BE59BD9B4E019ull + b + 0x8CB92BA72F3D8DD7ull);
  m.next();
  return m.next();
}

double smoothstep01(double x) {
  if (x <= 0.0) return 0.0;
  if (x >= 1.0) return 1.0;
  return 0.5 - 0.5 * std::cos(kPi * x);
}

// A level that is `inside` on [a, b) and `outside` elsewhere, with raised-cosine
// edges `edge` wide centred on a and b.
double window_level(double t, double a, double b, double edge) {
  double up = smoothstep01((t - (a - 0.5 * edge)) / edge);
  double down = smoothstep01((t - (b - 0.5 * edge)) / edge);
  return up - down;
}

struct Bar {
  double ire;   // luma level
  double u, v;  // chroma components in IRE
};

// 75% colour bars: white, yellow, cyan, green, magenta, red, blue.
void make_bars(Bar bars[7]) {
  const double rgb[7][3] = {{1, 1, 1}, {1, 1, 0}, {0, 1, 1}, {0, 1, 0},
                            {1, 0, 1}, {1, 0, 0}, {0, 0, 1}};
  for (int i = 0; i < 7; i++) {
    double r = 0.75 * rgb[i][0], g = 0.75 * rgb[i][1], b = 0.75 * rgb[i][2];
    double y = 0.299 * r + 0.587 * g + 0.114 * b;
    bars[i].ire = 7.5 + 92.5 * y;
    bars[i].u = 92.5 * 0.492 * (b - y);
    bars[i].v = 92.5 * 0.877 * (r - y);
  }
}

struct LineGeom {
  int field_line;   // line index within its field (0-based), from the field's first EQ pulse
  int frame_half;   // half-line index at the line start within the 1050 half-line frame
  int field_index;  // running field counter (for moving content and track alternation)
};

// Composite luma (IRE) and chroma components (u, v in IRE) at program time
// `tau` (samples) measured from the start of frame-aligned line `lam`.
struct Content {
  Timing tm;
  double spl;      // nominal samples per line
  double fs;
  Bar bars[7];
  double us;       // samples per microsecond

  // du: delay of the picture and burst against the line's sync, samples
  void eval(long long lam, double u, double du, double* ire, double* cu, double* cv) const {
    // Frame-relative line and half-line.
    const int FL = tm.frame_lines;
    long long fl = lam % FL;
    if (fl < 0) fl += FL;
    double half = spl * 0.5;
    int hidx = (int)(2 * fl + (u >= half ? 1 : 0));
    double v = (u >= half) ? u - half : u;
    double t_us = u / us;
    double tp_us = (u - du) / us;  // picture and burst time
    double tv_us = v / us;
    long long frame = (lam >= 0 ? lam : lam - (FL - 1)) / FL;
    // Field-relative line numbering (field 1 starts at frame line 0, field 2 at
    // half-line FL, i.e. the middle of line (FL - 1) / 2).
    bool field2 = (hidx >= FL);
    double field_line_d = field2 ? (hidx - FL) * 0.5 : hidx * 0.5;
    long long field_index = frame * 2 + (field2 ? 1 : 0);

    const double edge = 0.2;  // us, sync edge width
    double level = 0.0;       // blanking
    double cu_ = 0.0, cv_ = 0.0;
    int rel = field2 ? hidx - FL : hidx;  // half-lines since the field's first EQ
    const int E = tm.eq_pulses;
    bool vert = rel >= 0 && rel < 3 * E;
    if (vert) {
      bool broad = rel >= E && rel < 2 * E;
      double w = broad ? (tm.half_line_us - 4.7) : tm.eq_us;
      level = tm.sync_ire * window_level(tv_us, 0.0, w, edge);
      // The half-line slot before the first EQ (second half of the previous
      // line) is handled by the previous line's eval; nothing else here.
    } else {
      // Full line with hsync at its start (only even half-lines start lines;
      // odd half-lines are second halves of normal lines).
      double sync = window_level(t_us, 0.0, 4.7, edge);
      level = tm.sync_ire * sync;
      // Colour burst on lines after the vertical interval: NTSC at 180
      // degrees (-U), PAL swinging +/-45 degrees about it with the V switch.
      int fline = (int)field_line_d;
      const double vsw = (tm.pal && (fline & 1)) ? -1.0 : 1.0;
      if (fline >= tm.burst_line) {
        double bw = window_level(tp_us, tm.burst_a, tm.burst_b, 0.3);
        if (tm.pal) {
          cu_ += -20.0 * 0.70710678118654752 * bw;
          cv_ += vsw * 20.0 * 0.70710678118654752 * bw;
        } else {
          cu_ += -20.0 * bw;
        }
      }
      if (fline >= tm.pic_first && fline < tm.pic_last) {
        double a0 = tm.pic_a, a1 = tm.pic_b;
        double act = window_level(tp_us, a0, a1, 0.25);
        double x = (tp_us - a0) / (a1 - a0);
        double yl = 7.5, uu = 0.0, vv = 0.0;
        if (fline < tm.bars_end) {
          // bars with raised-cosine transitions
          double pos = x * 7.0;
          int bi = (int)std::floor(pos);
          bi = std::max(0, std::min(6, bi));
          double frac = pos - std::floor(pos);
          const Bar& b0 = bars[bi];
          const Bar& b1 = bars[std::min(6, bi + 1)];
          const Bar& bm = bars[std::max(0, bi - 1)];
          // blend near edges over +-0.03 of a bar width
          double wr = smoothstep01((frac - 0.97) / 0.06);
          double wl = smoothstep01((0.03 - frac) / 0.06);
          yl = b0.ire * (1.0 - wr - wl) + b1.ire * wr + bm.ire * wl;
          uu = b0.u * (1.0 - wr - wl) + b1.u * wr + bm.u * wl;
          vv = vsw * (b0.v * (1.0 - wr - wl) + b1.v * wr + bm.v * wl);
        } else if (fline < tm.sine_end) {
          yl = 7.5 + 45.0 * (1.0 + std::sin(2.0 * kPi * (2.0 * x)));
        } else {
          // moving triangle ramp
          double ph = x + 0.013 * (double)field_index;
          ph -= std::floor(ph);
          double tri = ph < 0.5 ? 2.0 * ph : 2.0 - 2.0 * ph;
          yl = 7.5 + 92.5 * tri;
        }
        level += act * yl;
        cu_ += act * uu;
        cv_ += act * vv;
      }
    }
    *ire = level;
    *cu = cu_;
    *cv = cv_;
  }
};

void shelf_high(double f0, double dbgain, double fs, double q, double b[3], double a[3]) {
  double A = std::pow(10.0, dbgain / 40.0);
  double w0 = 2.0 * kPi * f0 / fs;
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

// Seeded per-program-line perturbations, independent of threads and ranges.
double line_uniform(uint64_t seed, uint64_t salt, long long lam) {
  SplitMix m(mix_seed(seed ^ salt, (uint64_t)lam));
  return 2.0 * m.uniform() - 1.0;
}
double line_offset(const cuvhs_synth_params* p, long long lam) {
  return p->line_offset_bound > 0 ? p->line_offset_bound * line_uniform(p->seed, 0x11F5E7ull, lam) : 0.0;
}
double line_phase(const cuvhs_synth_params* p, long long lam) {
  return p->chroma_phase_bound > 0 ? p->chroma_phase_bound * line_uniform(p->seed, 0xC4A5Eull, lam) : 0.0;
}

// The pre-emphasis shelf (the one the decoder inverts), its design parameters
// optionally perturbed, normalised to a0 = 1.
void preemphasis(const cuvhs_synth_params* p, double b[3], double a[3]) {
  shelf_high(273755.82 * (1.0 + p->preemph_perturb[0]), 13.9794 * (1.0 + p->preemph_perturb[1]),
             p->sample_rate_hz, 0.462088186 * (1.0 + p->preemph_perturb[2]), b, a);
  for (int i = 0; i < 3; i++) b[i] /= a[0];
  a[1] /= a[0];
  a[2] /= a[0];
  a[0] = 1.0;
}

// Line-start table: r[k] is the RF sample where program line lam0 + k starts
// (seeded start phase, per-line timebase random walk, speed drift, head
// switch jumps).
void line_table(const cuvhs_synth_params* p, size_t n, long long& lam0_out, std::vector<double>& r) {
  const Timing tm = timing(p->system);
  const double fs = p->sample_rate_hz;
  const double spl = fs / tm.line_rate;
  SplitMix master(mix_seed(p->seed, 0x5EED));
  // Start position: seeded phase within the first frame, so the file starts mid-field.
  double start_line = p->start_line >= 0 ? p->start_line : 20.0 + tm.start_lines * master.uniform();
  long long lam0 = (long long)std::floor(start_line);
  double u0 = (start_line - (double)lam0) * spl;

  size_t n_lines = (size_t)std::ceil((double)n / (spl * 0.95)) + 8;
  r.assign(n_lines + 1, 0.0);
  {
    SplitMix jr(mix_seed(p->seed, 0x717));
    double delta = 0.0, prev_delta = 0.0;
    r[0] = -u0;
    for (size_t k = 1; k <= n_lines; k++) {
      long long lam = lam0 + (long long)k;
      double step = jr.gauss() * p->jitter_step;
      delta += step;
      if (p->jitter_bound > 0) {
        if (delta > p->jitter_bound) delta = 2 * p->jitter_bound - delta;
        if (delta < -p->jitter_bound) delta = -2 * p->jitter_bound - delta;
        delta = std::max(-p->jitter_bound, std::min(p->jitter_bound, delta));
      } else {
        delta = 0.0;
      }
      double speed = 1.0;
      if (p->speed_drift != 0.0) {
        speed = 1.0 + p->speed_drift * std::sin(2.0 * kPi * (double)lam / 21000.0);
      }
      double len = spl * speed + (delta - prev_delta);
      prev_delta = delta;
      // head switch: a time jump 6 lines before each field's vertical interval
      long long fl = lam % tm.frame_lines;
      if (p->headswitch_max > 0 && (fl == tm.headswitch_lines[0] || fl == tm.headswitch_lines[1])) {
        int span = std::max(0, p->headswitch_max - p->headswitch_min);
        int jump = p->headswitch_min + (int)(jr.uniform() * (span + 1));
        len += (double)jump;
      }
      r[k] = r[k - 1] + len;
    }
  }

  lam0_out = lam0;
}

template <typename F>
void parallel_for(size_t n, int threads, F fn) {
  if (threads <= 1 || n < 2) {
    fn(0, n);
    return;
  }
  std::vector<std::thread> pool;
  size_t per = (n + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    size_t a = (size_t)t * per, b = std::min(n, a + per);
    if (a >= b) break;
    pool.emplace_back([=] { fn(a, b); });
  }
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" void cuvhs_synth_default_params(cuvhs_synth_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->sample_rate_hz = 28e6;
  p->n_fields = 40;
  p->seed = 1;
  p->snr_db = 40.0;
  p->jitter_bound = 0.5;
  p->jitter_step = 0.15;
  p->dropout_line_rate = 0.0;
  p->dropout_min = 5;
  p->dropout_max = 200;
  p->headswitch_min = 0;
  p->headswitch_max = 0;
  p->speed_drift = 0.0;
  p->start_line = -1.0;
  p->tail_lines = 40;
  p->chroma_level = 0.2;
  p->carrier_offset_hz = 0.0;
  p->deviation_scale = 1.0;
  p->first_track = 0;
  p->threads = 0;
}

extern "C" long long cuvhs_synth_length(const cuvhs_synth_params* p) {
  const Timing tm = timing(p->system);
  double spl = p->sample_rate_hz / tm.line_rate;
  double lines = p->n_fields * (tm.frame_lines * 0.5) + (double)p->tail_lines;
  return (long long)std::floor(lines * spl);
}

// A capture generated front to back in units of kUnit samples: passes 1 and 3
// of a unit run in parallel, pass 2 (the pre-emphasis filter and the FM phase,
// both recursive) carries its state from unit to unit, so memory stays at a
// few unit-sized buffers whatever the capture's length, and the bytes equal a
// one-piece generation of the whole capture.
struct cuvhs_synth_stream {
  cuvhs_synth_params p;
  Timing tm;
  double fs = 0, spl = 0;
  size_t n = 0, pos = 0;
  int threads = 1;
  long long lam0 = 0;
  std::vector<double> r;
  struct Span {
    double a, b;
  };
  std::vector<Span> drops;
  Content content;
  double b[3], a[3];
  double x1 = 0, x2 = 0, y1 = 0, y2 = 0, phase = 0;
  double sigma = 0, peak = 0, amp_l = 1.0, amp_c = 0;
  std::vector<float> ire, chroma;
  std::vector<uint8_t> unit;  // the current unit's bytes
  size_t unit_start = 0, unit_len = 0;
  static constexpr size_t kBlock = 65536;  // noise blocks, seeded by their index
  static constexpr size_t kUnit = kBlock * 64;

  bool open(const cuvhs_synth_params* pp, size_t n_out) {
    p = *pp;
    tm = timing(p.system);
    fs = p.sample_rate_hz;
    spl = fs / tm.line_rate;
    n = n_out;
    threads = p.threads > 0 ? p.threads : (int)std::max(1u, std::thread::hardware_concurrency());
    line_table(&p, n, lam0, r);
    const size_t n_lines = r.size() - 1;
    // ---- dropouts: per-line seeded events, stored as RF sample spans
    if (p.dropout_line_rate > 0) {
      SplitMix dr(mix_seed(p.seed, 0xD0D0));
      for (size_t k = 0; k < n_lines; k++) {
        if (dr.uniform() < p.dropout_line_rate) {
          int span = std::max(0, p.dropout_max - p.dropout_min);
          int len = p.dropout_min + (int)(dr.uniform() * (span + 1));
          double pos0 = r[k] + dr.uniform() * (r[k + 1] - r[k]);
          drops.push_back({pos0, pos0 + len});
        }
      }
    }
    content.tm = tm;
    content.spl = spl;
    content.fs = fs;
    content.us = fs * 1e-6;
    make_bars(content.bars);
    preemphasis(&p, b, a);
    amp_c = p.chroma_level / 40.0;  // chroma components are in IRE (burst 20)
    const double sig_rms = amp_l / std::sqrt(2.0);
    sigma = sig_rms / std::pow(10.0, p.snr_db / 20.0);
    peak = amp_l + 2.5 * p.chroma_level;
    return true;
  }

  // Samples [i0, i0 + len) into out (i0 a multiple of kBlock).
  void generate(size_t i0, size_t len, uint8_t* out) {
    ire.resize(len);
    chroma.resize(len);
    // ---- pass 1 (parallel): program-time content per RF sample
    parallel_for(len, threads, [&](size_t aa, size_t bb) {
      const size_t ga = i0 + aa;
      size_t k = (size_t)(std::upper_bound(r.begin(), r.end(), (double)ga) - r.begin());
      if (k > 0) k--;
      for (size_t j = aa; j < bb; j++) {
        const size_t i = i0 + j;
        while (k + 1 < r.size() && r[k + 1] <= (double)i) k++;
        double lenk = r[k + 1] - r[k];
        double u = ((double)i - r[k]) * (spl / lenk);
        long long lam = lam0 + (long long)k;
        double y, cu, cv;
        // picture timebase: the delay runs linearly from this line's offset at
        // its start to the next line's at its end
        const double d0 = line_offset(&p, lam), d1 = line_offset(&p, lam + 1);
        const double du = d0 + (u / spl) * (d1 - d0);
        content.eval(lam, u, du, &y, &cu, &cv);
        ire[j] = (float)y;
        // colour-under: rotation by +/-90 degrees per line, alternating by field track
        const int FL = tm.frame_lines;
        long long fl = lam % FL;
        bool field2 = (2 * fl + (u >= spl * 0.5 ? 1 : 0)) >= FL;
        long long field_index = (lam / FL) * 2 + (field2 ? 1 : 0);
        long long field_line = field2 ? fl - (FL - 1) / 2 : fl;
        int track = (int)((field_index + p.first_track) & 1);
        int rot = track ? 1 : 3;
        int q = (int)(((field_line * rot) % 4 + 4) % 4);
        // the picture delay moves the colour-under carrier with the picture
        double theta = 2.0 * kPi * std::fmod(tm.chroma_under * ((double)i - du) / fs, 1.0) + q * (kPi * 0.5) +
                       line_phase(&p, lam);
        chroma[j] = (float)(cu * std::sin(theta) + cv * std::cos(theta));
      }
    });
    // ---- pass 2 (sequential, state carried): pre-emphasis IIR on the IRE signal, then FM phase
    {
      if (i0 == 0) {
        x1 = x2 = ire[0];
        y1 = y2 = ire[0];  // the shelf's DC gain is 1
        phase = 0.0;
      }
      const double dev = p.deviation_scale * tm.hz_ire;
      const double fc = tm.ire0 + p.carrier_offset_hz;
      for (size_t j = 0; j < len; j++) {
        double x0 = ire[j];
        double y0 = b[0] * x0 + b[1] * x1 + b[2] * x2 - a[1] * y1 - a[2] * y2;
        x2 = x1;
        x1 = x0;
        y2 = y1;
        y1 = y0;
        double f = fc + dev * y0;
        phase += 2.0 * kPi * f / fs;
        if (phase > 2.0 * kPi) phase -= 2.0 * kPi * std::floor(phase / (2.0 * kPi));
        ire[j] = (float)phase;  // reuse the buffer for the carrier phase
      }
    }
    // ---- pass 3 (parallel): RF = luma carrier + colour-under, dropouts, noise, u8
    const size_t b0 = i0 / kBlock, n_blocks = (len + kBlock - 1) / kBlock;
    parallel_for(n_blocks, threads, [&](size_t ba, size_t bb) {
      size_t di = 0;
      for (size_t lb = ba; lb < bb; lb++) {
        const size_t blk = b0 + lb;
        SplitMix nr(mix_seed(p.seed, 0xA0000000ull + blk));
        size_t g0 = blk * kBlock, g1 = std::min(i0 + len, g0 + kBlock);
        if (!drops.empty()) {
          di = (size_t)(std::upper_bound(drops.begin(), drops.end(), (double)g0,
                                         [](double v, const Span& sp) { return v < sp.b; }) - drops.begin());
        }
        for (size_t i = g0; i < g1; i++) {
          double rf = amp_l * std::cos((double)ire[i - i0]) + amp_c * (double)chroma[i - i0];
          if (!drops.empty()) {
            while (di < drops.size() && drops[di].b <= (double)i) di++;
            if (di < drops.size() && drops[di].a <= (double)i && (double)i < drops[di].b) rf *= 0.03;
          }
          rf += sigma * nr.gauss();
          double qv = std::nearbyint(128.0 + 100.0 * rf / peak);
          if (qv < 0) qv = 0;
          if (qv > 255) qv = 255;
          out[i - i0] = (uint8_t)qv;
        }
      }
    });
  }

  // The next `count` samples of the capture.
  size_t next(uint8_t* out, size_t count) {
    size_t done = 0;
    while (done < count && pos < n) {
      if (pos >= unit_start + unit_len) {  // the next unit
        unit_start = pos;
        unit_len = std::min(kUnit, n - pos);
        if (unit_len == kUnit && done + kUnit <= count) {  // straight into the caller's buffer
          generate(unit_start, unit_len, out + done);
          pos += unit_len;
          done += unit_len;
          continue;
        }
        unit.resize(unit_len);
        generate(unit_start, unit_len, unit.data());
      }
      const size_t take = std::min(count - done, unit_start + unit_len - pos);
      std::memcpy(out + done, unit.data() + (pos - unit_start), take);
      pos += take;
      done += take;
    }
    return done;
  }
};

namespace {
bool valid_params(const cuvhs_synth_params* p) {
  return p && p->sample_rate_hz > 4e6 && (p->system == 0 || p->system == 1);
}
}  // namespace

extern "C" cuvhs_synth_stream* cuvhs_synth_open(const cuvhs_synth_params* p, long long n_out) {
  if (!valid_params(p) || n_out <= 0) return nullptr;
  cuvhs_synth_stream* s = new (std::nothrow) cuvhs_synth_stream();
  if (!s) return nullptr;
  s->open(p, (size_t)n_out);
  return s;
}

extern "C" long long cuvhs_synth_next(cuvhs_synth_stream* s, uint8_t* out, long long count) {
  if (!s || !out || count < 0) return -1;
  return (long long)s->next(out, (size_t)count);
}

extern "C" void cuvhs_synth_close(cuvhs_synth_stream* s) { delete s; }

extern "C" int cuvhs_synth_ntsc(const cuvhs_synth_params* p, uint8_t* out, long long n_out) {
  if (!p || !out || n_out <= 0) return -1;
  if (!(p->sample_rate_hz > 4e6)) return -2;
  if (p->system != 0 && p->system != 1) return -3;
  cuvhs_synth_stream* s = cuvhs_synth_open(p, n_out);
  if (!s) return -4;
  const long long got = cuvhs_synth_next(s, out, n_out);
  cuvhs_synth_close(s);
  return got == n_out ? 0 : -5;
}

extern "C" long long cuvhs_synth_lines(const cuvhs_synth_params* p, long long n, double* start, double* offset,
                                       double* phase, long long cap) {
  if (!p || n <= 0 || !(p->sample_rate_hz > 4e6)) return -1;
  long long lam0 = 0;
  std::vector<double> r;
  line_table(p, (size_t)n, lam0, r);
  const long long m = (long long)r.size() - 1;
  for (long long k = 0; k < std::min(m, cap); k++) {
    if (start) start[k] = r[(size_t)k];
    if (offset) offset[k] = line_offset(p, lam0 + k);
    if (phase) phase[k] = line_phase(p, lam0 + k);
  }
  return m;
}

extern "C" void cuvhs_synth_preemphasis(const cuvhs_synth_params* p, double b[3], double a[3]) { preemphasis(p, b, a); }
