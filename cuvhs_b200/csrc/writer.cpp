// .tbc.json writer: ld-tools field metadata in the exact text layout of the
// reference (src/io/tbc_writer.cpp:89-175), so files compare byte for byte.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "pipeline.h"

namespace cuvhs {

namespace {
void appendf(std::string& s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void appendf(std::string& s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  int n = vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (n > 0) s.append(buf, (size_t)std::min(n, (int)sizeof buf - 1));
}
void append_list(std::string& s, const int32_t* v, int n) {
  for (int j = 0; j < n; j++) appendf(s, j ? ", %d" : "%d", v[j]);
}
}  // namespace

std::string tbc_json(const Format& fmt, const cuvhs_field_info* fields, size_t n, const int32_t* dl,
                     const int32_t* ds, const int32_t* de) {
  std::string s;
  s.reserve(256 + n * 200);
  const double black = (0.0 - fmt.vsync_ire) * fmt.output_scale + fmt.output_zero;
  const double white = (100.0 - fmt.vsync_ire) * fmt.output_scale + fmt.output_zero;
  const bool pal = fmt.system == kPal;
  s += "{\n  \"videoParameters\": {\n";
  appendf(s, "    \"system\": \"%s\",\n    \"isSubcarrierLocked\": false,\n    \"isSourcePal\": %s,\n",
          pal ? "PAL" : "NTSC", pal ? "true" : "false");
  appendf(s, "    \"numberOfSequentialFields\": %d,\n", (int)n);
  appendf(s, "    \"black16bIre\": %.1f,\n", black);
  appendf(s, "    \"white16bIre\": %.1f,\n", white);
  appendf(s, "    \"sampleRate\": %.0f,\n", fmt.output_rate);
  appendf(s, "    \"fieldWidth\": %d,\n", fmt.output_line_len);
  appendf(s, "    \"fieldHeight\": %d,\n", fmt.output_field_lines);
  appendf(s, "    \"colourBurstStart\": %d,\n", fmt.burst_start);
  appendf(s, "    \"colourBurstEnd\": %d,\n", fmt.burst_end);
  appendf(s, "    \"activeVideoStart\": %d,\n    \"activeVideoEnd\": %d,\n", pal ? 185 : 134, pal ? 1107 : 894);
  s += "    \"tapeFormat\": \"VHS\",\n    \"isMapped\": false\n  },\n  \"fields\": [\n";
  for (size_t i = 0; i < n; i++) {
    const cuvhs_field_info& f = fields[i];
    s += "    {\n";
    appendf(s, "      \"isFirstField\": %s,\n", f.is_first_field ? "true" : "false");
    appendf(s, "      \"seqNo\": %d,\n", (int)i + 1);
    appendf(s, "      \"fileLoc\": %llu,\n", (unsigned long long)f.file_loc);
    if (f.field_phase_id > 0) appendf(s, "      \"fieldPhaseID\": %d,\n", f.field_phase_id);
    s += "      \"dropOuts\": {\n        \"fieldLine\": [";
    append_list(s, dl + f.dropout_offset, f.dropout_count);
    s += "],\n        \"startx\": [";
    append_list(s, ds + f.dropout_offset, f.dropout_count);
    s += "],\n        \"endx\": [";
    append_list(s, de + f.dropout_offset, f.dropout_count);
    s += "]\n      }\n";
    s += (i + 1 < n) ? "    },\n" : "    }\n";
  }
  s += "  ]\n}\n";
  return s;
}

}  // namespace cuvhs
