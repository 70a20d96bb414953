// cuvhs-synth: write a seeded synthetic VHS RF capture (u8) to a file.
//
//   cuvhs-synth [name=value ...] out.u8
//
// Every name is a field of cuvhs_synth_params (include/cuvhs_synth.h); fields
// not given keep cuvhs_synth_default_params' values.  The tool links the
// synthesizer alone (no CUDA, no decoder), so a process that only needs an
// input file -- e.g. a benchmark of another decoder -- loads nothing else.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cuvhs_synth.h"

namespace {

bool set_param(cuvhs_synth_params& p, const std::string& name, const char* v) {
  struct D {
    const char* n;
    double* d;
  } doubles[] = {{"sample_rate_hz", &p.sample_rate_hz},
                 {"snr_db", &p.snr_db},
                 {"jitter_bound", &p.jitter_bound},
                 {"jitter_step", &p.jitter_step},
                 {"dropout_line_rate", &p.dropout_line_rate},
                 {"speed_drift", &p.speed_drift},
                 {"start_line", &p.start_line},
                 {"chroma_level", &p.chroma_level},
                 {"carrier_offset_hz", &p.carrier_offset_hz},
                 {"deviation_scale", &p.deviation_scale},
                 {"line_offset_bound", &p.line_offset_bound},
                 {"chroma_phase_bound", &p.chroma_phase_bound}};
  struct I {
    const char* n;
    int* i;
  } ints[] = {{"n_fields", &p.n_fields},         {"tail_lines", &p.tail_lines},
              {"dropout_min", &p.dropout_min},   {"dropout_max", &p.dropout_max},
              {"headswitch_min", &p.headswitch_min}, {"headswitch_max", &p.headswitch_max},
              {"first_track", &p.first_track},   {"threads", &p.threads},
              {"system", &p.system}};
  char* end = nullptr;
  for (const D& d : doubles)
    if (name == d.n) {
      *d.d = strtod(v, &end);
      return end && *end == 0;
    }
  for (const I& i : ints)
    if (name == i.n) {
      *i.i = (int)strtol(v, &end, 10);
      return end && *end == 0;
    }
  if (name == "seed") {
    p.seed = strtoull(v, &end, 10);
    return end && *end == 0;
  }
  return false;
}

}  // namespace

int main(int argc, char** argv) {
  cuvhs_synth_params p;
  cuvhs_synth_default_params(&p);
  const char* out = nullptr;
  for (int i = 1; i < argc; i++) {
    const char* eq = strchr(argv[i], '=');
    if (!eq) {
      out = argv[i];
      continue;
    }
    const std::string name(argv[i], eq - argv[i]);
    if (!set_param(p, name, eq + 1)) {
      fprintf(stderr, "cuvhs-synth: bad parameter %s\n", argv[i]);
      return 2;
    }
  }
  if (!out) {
    fprintf(stderr, "usage: cuvhs-synth [name=value ...] out.u8\n");
    return 2;
  }
  const long long n = cuvhs_synth_length(&p);
  if (n <= 0) {
    fprintf(stderr, "cuvhs-synth: empty capture\n");
    return 1;
  }
  std::vector<uint8_t> buf((size_t)n);
  if (cuvhs_synth_ntsc(&p, buf.data(), n) != 0) {
    fprintf(stderr, "cuvhs-synth: synthesis failed\n");
    return 1;
  }
  FILE* f = fopen(out, "wb");
  if (!f || fwrite(buf.data(), 1, buf.size(), f) != buf.size()) {
    perror(out);
    if (f) fclose(f);
    return 1;
  }
  fclose(f);
  return 0;
}
