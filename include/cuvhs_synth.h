/* Seeded synthetic NTSC / PAL VHS RF test-signal generator (part of libcuvhs).
 *
 * No counterpart in the reference, which ships no test signal: it stands in for
 * the private tape captures the reference was developed on.  The parameters
 * follow the workload descriptions used to measure this decoder (sample rate,
 * field count, SNR, timebase jitter, dropouts, head switch, speed drift, and the
 * FM carrier/deviation perturbations used for parameter calibration).
 */
#ifndef CUVHS_SYNTH_H
#define CUVHS_SYNTH_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct cuvhs_synth_params {
  double sample_rate_hz;     /* capture rate, e.g. 28e6 */
  int n_fields;              /* fields of program material */
  int tail_lines;            /* extra lines appended after the last field */
  uint64_t seed;
  double snr_db;             /* RF SNR of the luma carrier against white noise */
  double jitter_bound;       /* per-line timebase random walk bound, samples */
  double jitter_step;        /* random walk step std-dev per line, samples */
  double dropout_line_rate;  /* probability that a line carries a dropout */
  int dropout_min, dropout_max;        /* dropout length range, samples */
  int headswitch_min, headswitch_max;  /* head-switch time jump range, samples (0 = off) */
  double speed_drift;        /* relative slow tape-speed drift amplitude */
  double start_line;         /* program line at sample 0; <0 picks a seeded start */
  double chroma_level;       /* colour-under amplitude relative to the luma carrier */
  double carrier_offset_hz;  /* FM carrier offset */
  double deviation_scale;    /* FM deviation scale (1 = nominal) */
  int first_track;           /* head track of the first field (0/1) */
  int threads;               /* 0 = all host cores */
  /* calibration perturbations (all 0 = the nominal tape) */
  double preemph_perturb[3]; /* relative changes of the pre-emphasis shelf's corner frequency, gain (dB)
                                and Q; the 2-pole filter stays stable */
  double line_offset_bound;  /* per-line delay of the picture and burst against the sync at the line's
                                start, uniform in +/- bound samples; within a line the delay runs
                                linearly to the next line's */
  double chroma_phase_bound; /* per-line colour-under phase offset, uniform in +/- bound radians */
  int system;                /* 0 = NTSC, 1 = PAL (timing, IRE map, colour-under carrier, V switch) */
} cuvhs_synth_params;

void cuvhs_synth_default_params(cuvhs_synth_params* p);
/* Number of u8 samples the parameters describe. */
long long cuvhs_synth_length(const cuvhs_synth_params* p);
/* Fill out[0..n) with the capture; returns 0 on success. */
int cuvhs_synth_ntsc(const cuvhs_synth_params* p, uint8_t* out, long long n);
/* The same capture of n samples generated front to back in pieces of any
 * size, with a few tens of MB of working memory however long the capture is
 * (a 10-minute 40 MHz capture is 2.4e10 samples): cuvhs_synth_next writes the
 * next `count` samples and returns how many it wrote (fewer at the end).
 * The pieces concatenate to cuvhs_synth_ntsc's bytes. */
typedef struct cuvhs_synth_stream cuvhs_synth_stream;
cuvhs_synth_stream* cuvhs_synth_open(const cuvhs_synth_params* p, long long n);
long long cuvhs_synth_next(cuvhs_synth_stream* s, uint8_t* out, long long count);
void cuvhs_synth_close(cuvhs_synth_stream* s);
/* The program-line table of the capture: for up to cap lines, the RF sample
 * where each line starts, its picture delay at the line start (samples) and
 * its colour-under phase offset (radians).  Returns the number of lines. */
long long cuvhs_synth_lines(const cuvhs_synth_params* p, long long n, double* start, double* offset, double* phase,
                            long long cap);
/* The pre-emphasis biquad the parameters use, normalised to a0 = 1:
 * b[0..2], a[0..2]. */
void cuvhs_synth_preemphasis(const cuvhs_synth_params* p, double b[3], double a[3]);

#ifdef __cplusplus
}
#endif
#endif
