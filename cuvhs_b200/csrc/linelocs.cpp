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

struct Anchor {
  bool valid = false;
  double first_hsync_loc = 0.0, first_hsync_line = 0.0;
  int first_field = -1, progressive_field = 0;
  double hsync_diff = -1.0;
};

// Vertical-blanking anchor and field order (pipeline.cu:650-855).
Anchor anchor_field(const std::vector<ValidPulse>& v, double mll, const Format& fmt, int prev_first, double prev_off_lines,
                    double prev_loc, double prev_diff, int confidence) {
  Anchor out;
  if (v.empty() || mll <= 0.0) return out;
  const int lines[2] = {fmt.field_lines_first, fmt.field_lines_second};
  const double tol_lines = 0.5;
  double order_len[4] = {-1, -1, -1, -1};
  int vb_pulse[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
  int prev = -1, grp = 0, fgrp = 0;
  for (int i = 0; i < (int)v.size(); i++) {
    if (prev != -1 && v[i].good) {
      if (grp == 0 && v[i].p.start > v[0].p.start + lines[0] * mll) {
        grp = 4;
        fgrp = 2;
      }
      const int pt = v[prev].type, t = v[i].type;
      if (pt == kHsync && t > kHsync) {
        vb_pulse[0 + grp] = v[i].p.start;
        order_len[0 + fgrp] = half_line_round((v[i].p.start - v[prev].p.start) / mll);
      } else if (pt == kEq1 && t == kVsync) {
        vb_pulse[1 + grp] = v[i].p.start;
      } else if (pt == kVsync && t == kEq2) {
        vb_pulse[2 + grp] = v[i].p.start;
      } else if (pt > kHsync && t == kHsync) {
        vb_pulse[3 + grp] = v[prev].p.start;
        order_len[1 + fgrp] = half_line_round((v[i].p.start - v[prev].p.start) / mll);
      }
    }
    prev = i;
  }
  double first_pat[4] = {1, 0.5, 0.5, 1};
  double second_pat[4] = {0.5, 1, 1, 0.5};
  double agree = 0.0, seen = 0.0;
  for (int i = 0; i < 4; i++) {
    if (order_len[i] == first_pat[i]) {
      agree += 1.0;
      seen += 1.0;
    }
    if (order_len[i] == second_pat[i]) seen += 1.0;
  }
  bool first;
  if (prev_first == -1) first = seen == 0.0 || std::round(agree / std::max(1.0, seen)) == 1.0;
  else first = !prev_first;
  if (seen > 0.0) {
    if (prev_loc < 0.0) confidence = std::min(confidence, 50);
    const double weight = seen / 4.0;
    const int c_first = (int)std::llround((agree / seen) * weight * 100.0);
    const int c_second = (int)std::llround(((seen - agree) / seen) * weight * 100.0);
    if (c_first >= confidence && c_first > c_second) first = true;
    else if (c_second >= confidence && c_second > c_first) first = false;
  }
  const double section = fmt.num_eq_pulses / 2.0;
  const double cur_lines = first ? lines[0] : lines[1];
  const double prev_lines = first ? lines[1] : lines[0];
  const double* pat = first ? first_pat : second_pat;
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
    const int p1 = vb_pulse[i1], p2 = vb_pulse[i2];
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
  const int predicted = (int)std::llround((prev_off_lines + prev_lines + prev_loc / mll) * mll);
  bool used_prediction = false;
  if (cnt == 0 && prev_loc > 0.0) {
    double p = (prev_diff <= 0.5 && prev_diff >= -0.5) ? predicted + mll * prev_diff : (double)predicted;
    if (p <= 0.0) p = (double)v.front().p.start;
    loc += p;
    cnt += 1;
    used_prediction = true;
  }
  if (cnt <= 0) return out;
  off /= cnt;
  loc = std::round((loc + off) / cnt);
  if (!used_prediction) prev_diff = (loc - predicted) / mll;
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
  out.valid = true;
  out.first_hsync_loc = loc;
  out.first_hsync_line = hsync_line;
  out.first_field = first ? 1 : 0;
  out.progressive_field = 0;
  out.hsync_diff = prev_diff;
  return out;
}

// Nominal line grid snapped to the nearest pulse (pipeline.cu:857-893).
void snap_lines(const std::vector<ValidPulse>& v, double ref_pos, double ref_line, double mll, int nlines,
                std::vector<double>& locs) {
  locs.assign((size_t)nlines, 0.0);
  std::vector<double> ps;
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

void prepare_lines(const Format& fmt, const int* pulse_starts, const int* pulse_lengths, int count,
                   LinePrep& out) {
  const int n = std::max(0, std::min(count, kMaxPulses));
  out.v = validate(pulse_starts, pulse_lengths, n, fmt);
  out.mll = mean_line(out.v, (double)fmt.samples_per_line);
  out.n_raw = n;
  out.raw0 = n > 0 ? (double)pulse_starts[0] : 0.0;
}

void finish_lines(const Format& fmt, const LinePrep& prep, long long field_readloc, LineLocState& st,
                  FieldLines& out) {
  const std::vector<ValidPulse>& v = prep.v;
  const double mll = prep.mll;
  double prev_off = 0.0;
  if (st.prev_first_hsync_readloc != -1 && mll > 0.0)
    prev_off = ((double)st.prev_first_hsync_readloc - (double)field_readloc) / mll;
  const Anchor an = anchor_field(v, mll, fmt, st.prev_first_field, prev_off, st.prev_first_hsync_loc,
                                 st.prev_first_hsync_diff, 75);
  const int kept = std::min((int)v.size(), kMaxPulses);
  out.starts.resize(kept);
  out.lengths.resize(kept);
  out.types.resize(kept);
  for (int i = 0; i < kept; i++) {
    out.starts[i] = v[i].p.start;
    out.lengths[i] = v[i].p.len;
    out.types[i] = v[i].type;
  }
  if (an.valid) {
    snap_lines(v, an.first_hsync_loc, an.first_hsync_line, mll, fmt.lines_per_frame, out.locs);
    out.is_first = an.first_field;
    st.prev_first_field = an.first_field;
    st.prev_progressive_field = an.progressive_field;
    st.prev_first_hsync_readloc = field_readloc;
    st.prev_first_hsync_loc = an.first_hsync_loc;
    st.prev_first_hsync_diff = an.hsync_diff;
  } else {
    out.locs.assign((size_t)fmt.lines_per_frame, 0.0);
    for (int line = 0; line < fmt.lines_per_frame; line++) out.locs[line] = prep.raw0 + mll * (double)line;
    out.is_first = st.prev_first_field >= 0 ? (1 - st.prev_first_field) : 1;
  }
}

void locate_lines(const Format& fmt, const int* pulse_starts, const int* pulse_lengths, int count,
                  long long field_readloc, LineLocState& st, FieldLines& out) {
  LinePrep prep;
  prepare_lines(fmt, pulse_starts, pulse_lengths, count, prep);
  finish_lines(fmt, prep, field_readloc, st, out);
}

}  // namespace cuvhs
