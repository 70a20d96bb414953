// Line locations from sync pulses (the reference's default host path,
// src/pipeline/pipeline.cu:410-893 driven from :1717-1778).
//
// Works on one field's pulses (chunk-relative starts, lengths) in the order
// the pulse finder produced them.  Everything is FP64 with the reference's
// operation order, so identical pulses give bit-identical line locations.
#include <algorithm>
#include <cmath>

#include "cuvhs_internal.h"

namespace cuvhs {
namespace {


struct Windows {  // adaptive pulse-width classes (pipeline.cu:450-477)
  double h_lo, h_hi, e_lo, e_hi, v_lo, v_hi;
};

bool within(double v, double lo, double hi) { return v >= lo && v <= hi; }

// Spacings (lines) of the last hsync -> first EQ and last EQ -> first hsync
// around this field's blanking interval, then around the next one, for a
// first (or second) field of the system (pipeline.cu:704-716).
const double* field_pattern(const Format& fmt, bool first) {
  static const double ntsc_first[4] = {1, 0.5, 0.5, 1}, ntsc_second[4] = {0.5, 1, 1, 0.5};
  static const double pal_first[4] = {0.5, 0.5, 1, 1}, pal_second[4] = {1, 1, 0.5, 0.5};
  if (fmt.system == kPal) return first ? pal_first : pal_second;
  return first ? ntsc_first : ntsc_second;
}

// Field length (lines) from the previous field's first hsync to this one's:
// NTSC counts the previous field's lines, PAL the current one's (pipeline.cu:811).
double predicted_field_lines(const Format& fmt, bool first) {
  const int cur = first ? fmt.field_lines_first : fmt.field_lines_second;
  const int prev = first ? fmt.field_lines_second : fmt.field_lines_first;
  return fmt.system == kPal ? cur : prev;
}

// Quantise a line count to 0.5-line steps, then to 0.1 (pipeline.cu:436-438).
double half_line_round(double lines) { return std::round(0.5 * std::round(lines / 0.5) * 10.0) / 10.0; }

// Spacing check between consecutive validated pulses (pipeline.cu:133-148).
bool spacing_ok(int prev_type, int type, int delta, int line_len) {
  double lo, hi;
  if (prev_type > 0 && type > 0) {
    lo = 0.4;
    hi = 0.6;
  } else if (prev_type == 0 && type == 0) {
    lo = 0.9;
    hi = 1.1;
  } else {
    lo = 0.4;
    hi = 1.1;
  }
  const double span = (double)delta / (double)line_len;
  return span >= lo && span <= hi;
}

Windows width_windows(const int* lengths, int n, const Format& fmt) {
  const double tol = fmt.fs_hz * 0.5e-6;
  const double loose_lo = fmt.hsync_width - 3.5 * tol, loose_hi = fmt.hsync_width + 4.0 * tol;
  double sum = 0.0;
  int cnt = 0;
  for (int i = 0; i < n; i++) {
    const double l = (double)lengths[i];
    if (l >= loose_lo && l <= loose_hi) {
      sum += l;
      cnt++;
    }
  }
  const double est = cnt > 0 ? (sum / cnt) : fmt.hsync_width;
  const double shift = est - fmt.hsync_width;
  Windows w;
  const double hnom = fmt.hsync_width + shift;
  w.h_lo = hnom - tol;
  w.h_hi = hnom + tol;
  w.e_lo = fmt.eq_pulse_width + shift - tol;
  w.e_hi = fmt.eq_pulse_width + shift + tol;
  w.v_lo = (fmt.vsync_width + shift) * 0.5;
  w.v_hi = fmt.vsync_width + shift + 2.0 * tol;
  return w;
}

// Vertical-blanking sequence recogniser over at most 26 pulses from `first`
// (pipeline.cu:519-609).  Appends to `seq`; true when the sequence closed.
bool blanking_sequence(const std::vector<SyncPulse>& raw, size_t first, const Windows& w, int eq_pulses, int line_len,
                       std::vector<ValidPulse>& seq) {
  bool done = false;
  const double half = eq_pulses / 2.0;
  int vsync_at = -1;
  double hold_until = 0.0, pending = -1.0;
  for (size_t i = first; i < raw.size() && i < first + 26; i++) {
    const SyncPulse& p = raw[i];
    const double len = (double)p.len;
    const int cur = seq.empty() ? -1 : seq.back().type;
    int type = -1;
    switch (cur) {
      case -1:
        if (within(len, w.h_lo, w.h_hi)) type = kHsync;
        break;
      case kHsync:
        if (within(len, w.h_lo, w.h_hi)) {
          type = kHsync;
        } else if (within(len, w.e_lo, w.e_hi)) {
          type = kEq1;
          pending = half;
        } else if (within(len, w.v_lo, w.v_hi)) {
          vsync_at = (int)seq.size() - 1;
          type = kVsync;
        }
        break;
      case kEq1:
        if (within(len, w.e_lo, w.e_hi)) {
          type = kEq1;
        } else if (within(len, w.v_lo, w.v_hi)) {
          vsync_at = (int)seq.size() - 1;
          type = kVsync;
          pending = half;
        } else if (within(len, w.h_lo, w.h_hi)) {
          type = kHsync;
        }
        break;
      case kVsync:
        if (within(len, w.e_lo, w.e_hi)) {
          type = kEq2;
          pending = half;
        } else if (within(len, w.v_lo, w.v_hi)) {
          type = kVsync;
        } else if ((double)p.start > hold_until && within(len, w.h_lo, w.h_hi)) {
          type = kHsync;
        }
        break;
      case kEq2:
        if (within(len, w.e_lo, w.e_hi)) {
          type = kEq2;
        } else if (within(len, w.h_lo, w.h_hi)) {
          type = kHsync;
          done = true;
        }
        break;
    }
    bool keep = type >= 0;
    if (keep && type != cur) {
      if ((double)p.start < hold_until) {
        keep = false;
      } else if (pending > 0.0) {
        hold_until = (double)p.start + ((pending - 0.1) * (double)line_len);
        pending = -1.0;
      }
    }
    if (keep) {
      const bool good = seq.empty() ? false : spacing_ok(seq.back().type, type, p.start - seq.back().p.start, line_len);
      seq.push_back({type, p, good});
    }
    if (done && vsync_at >= 0) return true;
  }
  return done;
}

// Pulse validation (pipeline.cu:611-648).
std::vector<ValidPulse> validate(const int* starts, const int* lengths, int n, const Format& fmt) {
  std::vector<ValidPulse> out;
  if (n <= 0) return out;
  const Windows w = width_windows(lengths, n, fmt);
  std::vector<SyncPulse> raw((size_t)n);
  for (int i = 0; i < n; i++) raw[i] = {starts[i], lengths[i]};
  int i = 0;
  while (i < n) {
    const SyncPulse cur = raw[i];
    if (within((double)cur.len, w.h_lo, w.h_hi)) {
      const bool good =
          !out.empty() && spacing_ok(out.back().type, kHsync, cur.start - out.back().p.start, fmt.samples_per_line);
      out.push_back({kHsync, cur, good});
      i++;
    } else if (i > 2 && within((double)cur.len, w.e_lo, w.e_hi) && !out.empty() && out.back().type == kHsync) {
      // The recogniser extends the list in place; an unfinished attempt is
      // rolled back (the reference runs it on a copy and keeps it on success).
      const size_t before = out.size();
      const bool done = blanking_sequence(raw, (size_t)(i - 2), w, fmt.num_eq_pulses, fmt.samples_per_line, out);
      if (done && out.size() > before) {
        // the reference measures the advance after replacing the list, so it is one
        i = std::min(i + 1, n);
      } else {
        out.resize(before);
        i++;
      }
    } else {
      i++;
    }
  }
  return out;
}

// Mean line length from the longest HSYNC run (pipeline.cu:479-517).
double mean_line(const std::vector<ValidPulse>& v, double nominal) {
  int best_start = -1, best_len = -1, run_start = -1, run_len = 0;
  for (int i = 0; i < (int)v.size(); i++) {
    if (v[i].type != kHsync) {
      if (run_start >= 0 && run_len > best_len) {
        best_start = run_start;
        best_len = run_len;
      }
      run_start = -1;
      run_len = 0;
    } else if (run_start < 0) {
      run_start = i;
      run_len = 0;
    } else {
      run_len++;
    }
  }
  if (run_start >= 0 && run_len > best_len) {
    best_start = run_start;
    best_len = run_len;
  }
  double sum = 0.0;
  int cnt = 0;
  if (best_start >= 1 && best_len >= 1) {
    for (int i = best_start + 1; i < best_start + best_len; i++) {
      const double l = (double)(v[i].p.start - v[i - 1].p.start);
      const double r = l / nominal;
      if (r >= 0.95 && r <= 1.05) {
        sum += l;
        cnt++;
      }
    }
  }
  return cnt == 0 ? nominal : sum / (double)cnt;
}

// Vertical-blanking anchor and field order (pipeline.cu:650-855), in three
// parts so that everything but a few scalar decisions can run before the
// carried state is known:
//   scan_blanking  the blanking pulses and the half-line pattern (no state);
//   decide_first   field order from the pattern and the previous field;
//   fit_anchor     first-hsync location for a given field order (state only
//                  through prev_loc, and the prediction when nothing fits).

// Vertical-blanking pulse positions and pattern agreement of one field.
BlankingScan scan_blanking(const std::vector<ValidPulse>& v, double mll, const Format& fmt) {
  BlankingScan s;
  for (int i = 0; i < 8; i++) s.vb_pulse[i] = -1;
  for (int i = 0; i < 4; i++) s.order_len[i] = -1;
  s.agree = s.seen = 0.0;
  if (v.empty() || mll <= 0.0) return s;
  const int lines0 = fmt.field_lines_first;
  int prev = -1, grp = 0, fgrp = 0;
  for (int i = 0; i < (int)v.size(); i++) {
    if (prev != -1 && v[i].good) {
      if (grp == 0 && v[i].p.start > v[0].p.start + lines0 * mll) {
        grp = 4;
        fgrp = 2;
      }
      const int pt = v[prev].type, t = v[i].type;
      if (pt == kHsync && t > kHsync) {
        s.vb_pulse[0 + grp] = v[i].p.start;
        s.order_len[0 + fgrp] = half_line_round((v[i].p.start - v[prev].p.start) / mll);
      } else if (pt == kEq1 && t == kVsync) {
        s.vb_pulse[1 + grp] = v[i].p.start;
      } else if (pt == kVsync && t == kEq2) {
        s.vb_pulse[2 + grp] = v[i].p.start;
      } else if (pt > kHsync && t == kHsync) {
        s.vb_pulse[3 + grp] = v[prev].p.start;
        s.order_len[1 + fgrp] = half_line_round((v[i].p.start - v[prev].p.start) / mll);
      }
    }
    prev = i;
  }
  const double* first_pat = field_pattern(fmt, true);
  const double* second_pat = field_pattern(fmt, false);
  for (int i = 0; i < 4; i++) {
    if (s.order_len[i] == first_pat[i]) {
      s.agree += 1.0;
      s.seen += 1.0;
    }
    if (s.order_len[i] == second_pat[i]) s.seen += 1.0;
  }
  return s;
}

// Field order: the pattern's vote when it reaches `confidence`, else the
// opposite of the previous field (the pattern alone for the first field).
bool decide_first(const BlankingScan& s, int prev_first, double prev_loc, int confidence) {
  bool first;
  if (prev_first == -1) first = s.seen == 0.0 || std::round(s.agree / std::max(1.0, s.seen)) == 1.0;
  else first = !prev_first;
  if (s.seen > 0.0) {
    if (prev_loc < 0.0) confidence = std::min(confidence, 50);
    const double weight = s.seen / 4.0;
    const int c_first = (int)std::llround((s.agree / s.seen) * weight * 100.0);
    const int c_second = (int)std::llround(((s.seen - s.agree) / s.seen) * weight * 100.0);
    if (c_first >= confidence && c_first > c_second) first = true;
    else if (c_second >= confidence && c_second > c_first) first = false;
  }
  return first;
}

// The field order the pattern fixes on its own at `confidence` whatever the
// carried state is (a vote that clears `confidence` also clears the lower
// threshold used after an invalid field), or -1.
int pattern_first(const BlankingScan& s, int confidence) {
  if (s.seen <= 0.0) return -1;
  const double weight = s.seen / 4.0;
  const int c_first = (int)std::llround((s.agree / s.seen) * weight * 100.0);
  const int c_second = (int)std::llround(((s.seen - s.agree) / s.seen) * weight * 100.0);
  if (c_first >= confidence && c_first > c_second) return 1;
  if (c_second >= confidence && c_second > c_first) return 0;
  return -1;
}

// First-hsync location for field order `first`.  loc_round is the estimate
// before the hsync refinement (the carried hsync_diff is taken from it).
AnchorFit fit_anchor(const BlankingScan& s, const std::vector<ValidPulse>& v, double mll, const Format& fmt,
                     bool first, double prev_off_lines, double prev_loc, double prev_diff) {
  AnchorFit out;
  if (v.empty() || mll <= 0.0) return out;
  const int lines[2] = {fmt.field_lines_first, fmt.field_lines_second};
  const double tol_lines = 0.5;
  const double section = fmt.num_eq_pulses / 2.0;
  const double cur_lines = first ? lines[0] : lines[1];
  const double pred_lines = predicted_field_lines(fmt, first);
  const double* pat = field_pattern(fmt, first);
  double vb_line[8];
  vb_line[0] = 0.0 + pat[0];
  vb_line[1] = vb_line[0] + section;
  vb_line[2] = vb_line[1] + section;
  vb_line[3] = vb_line[2] + section - 0.5;
  const double hsync_line = vb_line[3] + pat[1];
  vb_line[4] = cur_lines + pat[2];
  vb_line[5] = vb_line[4] + section;
  vb_line[6] = vb_line[5] + section;
  vb_line[7] = vb_line[6] + section - 0.5;
  auto pair_estimate = [&](int i1, int i2, double& loc, int& cnt, double& off) {
    const int p1 = s.vb_pulse[i1], p2 = s.vb_pulse[i2];
    if (p1 == -1 || p2 == -1 || mll == 0.0) return;
    const double actual = ((double)p1 - (double)p2) / mll;
    const double expect = vb_line[i1] - vb_line[i2];
    if (actual < expect + tol_lines && actual > expect - tol_lines) {
      off += actual - expect;
      loc += (double)p2 + mll * (hsync_line - vb_line[i2]);
      cnt += 1;
    }
  };
  double a_loc = 0.0, a_off = 0.0, b_loc = 0.0, b_off = 0.0;
  int a_cnt = 0, b_cnt = 0;
  for (int x = 0; x < 4; x++)
    for (int y = x + 1; y < 4; y++) pair_estimate(x, y, a_loc, a_cnt, a_off);
  for (int x = 0; x < 4; x++)
    for (int y = x + 1; y < 4; y++) pair_estimate(4 + x, 4 + y, b_loc, b_cnt, b_off);
  double loc = 0.0, off = 0.0;
  int cnt = 0;
  const double a_est = a_cnt ? a_loc / a_cnt : 0.0, b_est = b_cnt ? b_loc / b_cnt : 0.0;
  if (a_cnt && b_cnt && a_est < b_est + tol_lines * mll && a_est > b_est - tol_lines * mll) {
    loc = a_loc + b_loc;
    cnt = a_cnt + b_cnt;
    off = a_off + b_off;
    for (int x = 0; x < 4; x++)
      for (int y = 0; y < 4; y++) pair_estimate(x, 4 + y, loc, cnt, off);
  } else if (a_cnt == 6 || (prev_loc <= 0.0 && a_cnt > b_cnt)) {
    loc = a_loc;
    cnt = a_cnt;
    off = a_off;
  } else if (b_cnt == 6 || (prev_loc <= 0.0 && b_cnt > a_cnt)) {
    loc = b_loc;
    cnt = b_cnt;
    off = b_off;
  }
  const int predicted = (int)std::llround((prev_off_lines + pred_lines + prev_loc / mll) * mll);
  if (cnt == 0 && prev_loc > 0.0) {
    double p = (prev_diff <= 0.5 && prev_diff >= -0.5) ? predicted + mll * prev_diff : (double)predicted;
    if (p <= 0.0) p = (double)v.front().p.start;
    loc += p;
    cnt += 1;
    out.used_prediction = true;
  }
  out.cnt = cnt;
  if (cnt <= 0) return out;
  off /= cnt;
  loc = std::round((loc + off) / cnt);
  out.loc_round = loc;
  double hoff = 0.0;
  int hcnt = 0;
  for (const ValidPulse& p : v) {
    if (p.type != kHsync || !p.good) continue;
    const double line = ((double)p.p.start - loc) / mll + hsync_line;
    const int rl = (int)std::llround(line);
    if (rl > cur_lines) break;
    if (rl >= hsync_line) {
      hoff += loc + mll * ((double)rl - hsync_line) - (double)p.p.start;
      hcnt++;
    }
  }
  if (hcnt > 0) {
    hoff /= hcnt;
    loc -= hoff;
  }
  out.loc = loc;
  out.hsync_line = hsync_line;
  return out;
}

// The carried hsync_diff after a fit that used no prediction.
double hsync_diff_after(const AnchorFit& f, const Format& fmt, bool first, double mll, double prev_off_lines,
                        double prev_loc) {
  const int predicted = (int)std::llround((prev_off_lines + predicted_field_lines(fmt, first) + prev_loc / mll) * mll);
  return (f.loc_round - predicted) / mll;
}

// Nominal line grid snapped to the nearest pulse (pipeline.cu:857-893).
void snap_lines(const std::vector<ValidPulse>& v, double ref_pos, double ref_line, double mll, int nlines,
                double* locs) {
  thread_local std::vector<double> ps;
  ps.clear();
  ps.reserve(v.size());
  for (const ValidPulse& p : v) ps.push_back((double)p.p.start);
  // nearly sorted already (the recogniser revisits two pulses): insertion sort
  for (size_t a = 1; a < ps.size(); a++) {
    const double v = ps[a];
    size_t b = a;
    while (b > 0 && ps[b - 1] > v) {
      ps[b] = ps[b - 1];
      b--;
    }
    ps[b] = v;
  }
  const double max_dist = mll / 1.5;
  size_t cur = 0;
  for (int line = 0; line < nlines; line++) {
    locs[line] = ref_pos + mll * ((double)line - ref_line);
    if (cur >= ps.size()) continue;
    double d = std::fabs(ps[cur] - locs[line]);
    double best = max_dist, at = -1.0;
    size_t s = cur;
    while (s + 1 < ps.size()) {
      if (d <= best) {
        best = d;
        cur = s;
        at = ps[s];
      }
      const double nd = std::fabs(ps[s + 1] - locs[line]);
      if (nd > d) break;
      d = nd;
      s++;
    }
    if (at >= 0.0) {
      locs[line] = at;
      cur++;
    }
  }
}

}  // namespace

void prepare_lines(const Format& fmt, const int* pulse_starts, const int* pulse_lengths, int count, LinePrep& out,
                   double* spec_locs) {
  const int n = std::max(0, std::min(count, kMaxPulses));
  out.v = validate(pulse_starts, pulse_lengths, n, fmt);
  out.mll = mean_line(out.v, (double)fmt.samples_per_line);
  out.n_raw = n;
  out.raw0 = n > 0 ? (double)pulse_starts[0] : 0.0;
  out.scan = scan_blanking(out.v, out.mll, fmt);
  out.spec_first = -1;
  out.spec = AnchorFit();
  if (!spec_locs) return;
  // Ahead of the carried state: when the pattern fixes the field order and
  // the blanking pulses fit, the anchor and the snapped grid equal what the
  // in-order pass computes for any previous field with prev_loc > 0.
  const int pf = pattern_first(out.scan, kAnchorConfidence);
  if (pf < 0) return;
  const AnchorFit f = fit_anchor(out.scan, out.v, out.mll, fmt, pf == 1, 0.0, 1.0, 0.0);
  if (f.cnt <= 0 || f.used_prediction) return;
  snap_lines(out.v, f.loc, f.hsync_line, out.mll, fmt.lines_per_frame, spec_locs);
  out.spec_first = pf;
  out.spec = f;
}

void finish_lines(const Format& fmt, const LinePrep& prep, long long field_readloc, LineLocState& st, double* locs,
                  FieldLines* pulses, int* is_first) {
  const std::vector<ValidPulse>& v = prep.v;
  const double mll = prep.mll;
  double prev_off = 0.0;
  if (st.prev_first_hsync_readloc != -1 && mll > 0.0)
    prev_off = ((double)st.prev_first_hsync_readloc - (double)field_readloc) / mll;
  if (pulses) {
    const int kept = std::min((int)v.size(), kMaxPulses);
    pulses->starts.resize(kept);
    pulses->lengths.resize(kept);
    pulses->types.resize(kept);
    for (int i = 0; i < kept; i++) {
      pulses->starts[i] = v[i].p.start;
      pulses->lengths[i] = v[i].p.len;
      pulses->types[i] = v[i].type;
    }
  }
  const double prev_loc = st.prev_first_hsync_loc;
  bool valid = !v.empty() && mll > 0.0;
  bool first = false;
  AnchorFit f;
  if (valid) {
    first = decide_first(prep.scan, st.prev_first_field, prev_loc, kAnchorConfidence);
    if (prep.spec_first == (first ? 1 : 0) && prev_loc > 0.0) {
      f = prep.spec;  // locs already hold the snapped grid
    } else {
      f = fit_anchor(prep.scan, v, mll, fmt, first, prev_off, prev_loc, st.prev_first_hsync_diff);
      if (f.cnt > 0) snap_lines(v, f.loc, f.hsync_line, mll, fmt.lines_per_frame, locs);
    }
    valid = f.cnt > 0;
  }
  if (valid) {
    *is_first = first ? 1 : 0;
    st.prev_first_field = first ? 1 : 0;
    st.prev_progressive_field = 0;
    st.prev_first_hsync_readloc = field_readloc;
    st.prev_first_hsync_loc = f.loc;
    if (!f.used_prediction) st.prev_first_hsync_diff = hsync_diff_after(f, fmt, first, mll, prev_off, prev_loc);
  } else {
    for (int line = 0; line < fmt.lines_per_frame; line++) locs[line] = prep.raw0 + mll * (double)line;
    *is_first = st.prev_first_field >= 0 ? (1 - st.prev_first_field) : 1;
  }
}

void locate_lines(const Format& fmt, const int* pulse_starts, const int* pulse_lengths, int count,
                  long long field_readloc, LineLocState& st, FieldLines& out) {
  LinePrep prep;
  prepare_lines(fmt, pulse_starts, pulse_lengths, count, prep, nullptr);
  out.locs.assign((size_t)fmt.lines_per_frame, 0.0);
  finish_lines(fmt, prep, field_readloc, st, out.locs.data(), &out, &out.is_first);
}

}  // namespace cuvhs

namespace cuvhs {

// The single-pass line locator the reference runs when its host line
// location is switched off (CUVHS_K2B_DISABLE; src/pipeline/line_locs.cu:62-543,
// one GPU thread per field there, a host pool task here): width classes
// adapted to the field's mean hsync width, the blanking state machine for the
// reference pulse and the field parity, the mean line from the longest hsync
// run, then the nominal grid snapped to the nearest hsync marker.  No state
// is carried between fields.  Where the reference's device code evaluates
// a + b * c, the fused multiply-add its compiler forms is written out.
void nominal_pulse_types(const Format& fmt, const int* lengths, int count, int* types) {
  const double tol = 0.5e-6 * fmt.fs_hz;
  const double h_lo = fmt.hsync_width - tol, h_hi = fmt.hsync_width + tol;
  const double e_lo = fmt.eq_pulse_width - tol, e_hi = fmt.eq_pulse_width + tol;
  const double v_lo = fmt.vsync_width * 0.5, v_hi = fmt.vsync_width + 1.0e-6 * fmt.fs_hz;
  for (int i = 0; i < std::min(count, kMaxPulses); i++) {
    const double len = (double)lengths[i];
    if (len >= v_lo && len <= v_hi) types[i] = kVsync;
    else if (len >= h_lo && len <= h_hi) types[i] = kHsync;
    else if (len >= e_lo && len <= e_hi) types[i] = kEq1;
    else types[i] = kHsync;
  }
}

void single_pass_lines(const Format& fmt, const int* starts, const int* lengths, int count, double* locs,
                       int* parity) {
  const int n = std::max(0, std::min(count, kMaxPulses));
  const double tol = 0.5e-6 * fmt.fs_hz;
  const double inl = (double)fmt.samples_per_line;
  const double hnom = fmt.hsync_width, enom = fmt.eq_pulse_width, vnom = fmt.vsync_width;
  // width classes shifted by the field's mean hsync width (line_locs.cu:99-135)
  const double loose_lo = std::fma(-3.5, tol, hnom), loose_hi = std::fma(4.0, tol, hnom);
  double hsum = 0.0;
  int hcnt = 0;
  for (int i = 0; i < n; i++) {
    const double len = (double)lengths[i];
    if (len >= loose_lo && len <= loose_hi) {
      hsum += len;
      hcnt++;
    }
  }
  const double shift = (hcnt > 0 ? hsum / hcnt : hnom) - hnom;
  const double h_lo = hnom + shift - tol, h_hi = hnom + shift + tol;
  const double e_lo = enom + shift - tol, e_hi = enom + shift + tol;
  const double v_lo = (vnom + shift) * 0.5, v_hi = std::fma(2.0, tol, vnom + shift);
  thread_local std::vector<int> type;
  type.assign((size_t)n, kHsync);
  for (int i = 0; i < n; i++) {
    const double len = (double)lengths[i];
    if (len >= v_lo && len <= v_hi) type[i] = kVsync;
    else if (len >= h_lo && len <= h_hi) type[i] = kHsync;
    else if (len >= e_lo && len <= e_hi) type[i] = kEq1;
    else type[i] = kHsync;  // unclassified widths count as hsync
  }
  // blanking state machine: the first hsync after the vertical interval
  // (line_locs.cu:148-201)
  int ref = -1, last_h = -1, first_eq = -1, last_eq2 = -1, state = -1;
  for (int i = 0; i < n; i++) {
    const int t = type[i];
    if (state == -1) {
      if (t == kHsync) {
        state = kHsync;
        last_h = i;
      }
    } else if (state == kHsync) {
      if (t == kHsync) last_h = i;
      else if (t == kEq1) {
        state = kEq1;
        first_eq = i;
      } else if (t == kVsync) state = kVsync;
    } else if (state == kEq1) {
      if (t == kVsync) state = kVsync;
      else if (t == kHsync) {
        state = kHsync;
        last_h = i;
        first_eq = -1;
      }
    } else if (state == kVsync) {
      if (t == kEq1) {
        state = kEq2;
        last_eq2 = i;
      } else if (t == kHsync) {
        ref = i;
        break;
      }
    } else if (state == kEq2) {
      if (t == kEq1) last_eq2 = i;
      else if (t == kHsync) {
        if (last_eq2 < 0) last_eq2 = i - 1;
        ref = i;
        break;
      }
    }
  }
  // field parity from the half-line spacing entering or leaving the interval
  // (line_locs.cu:203-236)
  const bool ntsc = fmt.system == kNtsc;
  int par = -1;
  if (ref >= 0 && last_h >= 0 && first_eq >= 0) {
    const double lines = (double)(starts[first_eq] - starts[last_h]) / inl;
    par = ntsc ? (lines > 0.75 ? 1 : 0) : (lines > 0.75 ? 0 : 1);
  }
  if (par < 0 && ref >= 0 && last_eq2 >= 0) {
    const double lines = (double)(starts[ref] - starts[last_eq2]) / inl;
    par = ntsc ? (lines > 0.75 ? 1 : 0) : (lines > 0.75 ? 0 : 1);
  }
  *parity = par;
  // mean line length over the longest hsync run (line_locs.cu:246-284)
  int best_s = -1, best_n = 0, cur_s = -1, cur_n = 0;
  for (int i = 0; i < n; i++) {
    if (type[i] == kHsync) {
      if (cur_s == -1) {
        cur_s = i;
        cur_n = 1;
      } else {
        cur_n++;
      }
    } else {
      if (cur_n > best_n) {
        best_s = cur_s;
        best_n = cur_n;
      }
      cur_s = -1;
      cur_n = 0;
    }
  }
  if (cur_n > best_n) {
    best_s = cur_s;
    best_n = cur_n;
  }
  double mll = inl;
  if (best_n >= 2) {
    double sum = 0.0;
    int cnt = 0;
    for (int i = best_s + 1; i < best_s + best_n; i++) {
      const double sp = (double)(starts[i] - starts[i - 1]);
      if (sp >= inl * 0.95 && sp <= inl * 1.05) {
        sum += sp;
        cnt++;
      }
    }
    if (cnt > 0) mll = sum / cnt;
  }
  // reference position and line (line_locs.cu:295-337): a reference found in
  // the second half of the list belongs to the next field's interval
  double ref_pos, ref_line;
  if (ref >= 0) {
    ref_pos = (double)starts[ref];
    ref_line = 10.0;
    if (ref > n / 2) {
      const double back = ref_pos - (double)fmt.samples_per_field;
      if (back > 0.0) ref_pos = back;
    }
  } else {
    ref = 0;
    for (int i = 0; i < n; i++)
      if (type[i] == kHsync) {
        ref = i;
        break;
      }
    ref_pos = n > 0 ? (double)starts[ref] : 0.0;
    ref_line = 0.0;
  }
  // line markers: an EQ pulse followed closely by a tiny hsync fragment stands
  // for the line, and the fragment is dropped (line_locs.cu:365-399)
  thread_local std::vector<int> mk_s, mk_l, hs;
  mk_s.clear();
  mk_l.clear();
  const double tiny = hnom * 0.75, gap = inl * 0.25;
  for (int i = 0; i < n; i++) {
    const bool eq = type[i] == kEq1 || type[i] == kEq2;
    const bool surrogate = eq && i + 1 < n && type[i + 1] == kHsync && (double)lengths[i + 1] <= tiny &&
                           (double)(starts[i + 1] - starts[i]) <= gap;
    const bool fragment = type[i] == kHsync && (double)lengths[i] <= tiny && i > 0 &&
                          (type[i - 1] == kEq1 || type[i - 1] == kEq2) && (double)(starts[i] - starts[i - 1]) <= gap;
    if (surrogate || (type[i] == kHsync && !fragment)) {
      mk_s.push_back(starts[i]);
      mk_l.push_back(lengths[i]);
    }
  }
  // one marker per line interval: the one whose width is nearest the nominal
  // hsync (line_locs.cu:401-425)
  hs.clear();
  const double dup = inl * 0.75;
  const int nm = (int)mk_s.size();
  for (int c0 = 0; c0 < nm;) {
    int best = c0;
    double score = std::fabs((double)mk_l[c0] - hnom);
    int c1 = c0 + 1;
    while (c1 < nm && (double)(mk_s[c1] - mk_s[c0]) < dup) {
      const double sc = std::fabs((double)mk_l[c1] - hnom);
      if (sc < score || (sc == score && mk_s[c1] < mk_s[best])) {
        best = c1;
        score = sc;
      }
      c1++;
    }
    hs.push_back(mk_s[best]);
    c0 = c1;
  }
  // nominal grid snapped to the nearest marker ahead of a monotonic cursor
  // (line_locs.cu:429-470)
  const double max_d = mll / 1.5;
  const int nh = (int)hs.size();
  int cur = 0;
  for (int line = 0; line < fmt.lines_per_frame; line++) {
    const double expected = std::fma(mll, (double)line - ref_line, ref_pos);
    locs[line] = expected;
    if (cur >= nh) continue;
    double best_d = max_d;
    int best_pos = -1;
    for (int s = cur; s < nh; s++) {
      const double d = std::fabs((double)hs[s] - expected);
      if (d <= best_d) {
        best_d = d;
        best_pos = hs[s];
        cur = s;
      }
      if (s + 1 < nh) {
        if (std::fabs((double)hs[s + 1] - expected) > d) break;
      } else {
        break;
      }
    }
    if (best_pos >= 0) {
      locs[line] = (double)best_pos;
      cur++;
    }
  }
}

}  // namespace cuvhs
