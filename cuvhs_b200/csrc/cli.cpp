// cuvhs command line: the reference's argument grammar (src/main.cpp:24-87) on
// top of libcuvhs.
//   cuvhs [--system NTSC|PAL] [-f MHz] [--format u8|s16|u16] [--dc-correct]
//         [--gpu id] [--overwrite] [--batch N] <input|-> <output_base>
// Exit status 0 with "Done." on success, 1 on any failure.
#include <strings.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/cuvhs.h"

namespace {

void usage(const char* prog) {
  fprintf(stderr,
          "cuvhs (B200) -- GPU VHS RF decoder\n"
          "\n"
          "Usage: %s [options] <input_file> <output_base>\n"
          "\n"
          "Arguments:\n"
          "  input_file       Raw RF capture (.u8, .s16, .u16, .raw), or - for stdin\n"
          "  output_base      Output prefix (creates .tbc, _chroma.tbc, .tbc.json)\n"
          "\n"
          "Options:\n"
          "  --system <NTSC|PAL>   Video system (default: NTSC)\n"
          "  -f <MHz>              Sample rate in MHz (default: 28)\n"
          "  --format <u8|s16|u16> Input sample format (default: auto from extension)\n"
          "  --dc-correct          Subtract per-read DC offset after normalization\n"
          "  --gpu <id>            GPU device ID, -1 for auto (default: 0)\n"
          "  --overwrite           Overwrite existing output files\n"
          "  --batch <fields>      Fields per chunk (default: from free GPU memory)\n"
          "  -h, --help            Show this help\n",
          prog);
}

}  // namespace

int main(int argc, char** argv) {
  cuvhs_config cfg;
  cuvhs_default_config(&cfg);
  std::string in, out, format = "";
  bool overwrite = false, dc_correct = false, pal = false;
  int pos = 0;
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "-h") || !strcmp(argv[i], "--help")) {
      usage(argv[0]);
      return 0;
    } else if (!strcmp(argv[i], "--system") && i + 1 < argc) {
      i++;
      if (!strcasecmp(argv[i], "NTSC")) pal = false;
      else if (!strcasecmp(argv[i], "PAL")) pal = true;
      else {
        fprintf(stderr, "Unknown system: %s\n", argv[i]);
        return 1;
      }
    } else if (!strcmp(argv[i], "-f") && i + 1 < argc) {
      cfg.sample_rate_mhz = atof(argv[++i]);
    } else if (!strcmp(argv[i], "--format") && i + 1 < argc) {
      format = argv[++i];
      if (format != "u8" && format != "s16" && format != "u16") {
        fprintf(stderr, "Unknown format: %s\n", format.c_str());
        return 1;
      }
    } else if (!strcmp(argv[i], "--dc-correct")) {
      dc_correct = true;
    } else if (!strcmp(argv[i], "--gpu") && i + 1 < argc) {
      cfg.device = atoi(argv[++i]);
    } else if (!strcmp(argv[i], "--batch") && i + 1 < argc) {
      cfg.batch_fields = atoi(argv[++i]);
    } else if (!strcmp(argv[i], "--overwrite")) {
      overwrite = true;
    } else if (argv[i][0] == '-' && strlen(argv[i]) > 1) {
      fprintf(stderr, "Unknown option: %s\n", argv[i]);
      return 1;
    } else {
      if (pos == 0) in = argv[i];
      else if (pos == 1) out = argv[i];
      else {
        fprintf(stderr, "Too many arguments\n");
        return 1;
      }
      pos++;
    }
  }
  if (pos < 2) {
    fprintf(stderr, "Error: input_file and output_base are required\n\n");
    usage(argv[0]);
    return 1;
  }
  if (format.empty()) {
    const size_t dot = in.find_last_of('.');
    const std::string ext = dot == std::string::npos ? in : in.substr(dot + 1);
    format = (ext == "s16") ? "s16" : (ext == "u16") ? "u16" : "u8";
  }
  cfg.system = pal ? 1 : 0;
  cfg.input_format = format == "s16" ? 1 : (format == "u16" ? 2 : 0);
  cfg.dc_correct = dc_correct ? 1 : 0;
  cuvhs_status s = cuvhs_decode_file(&cfg, in.c_str(), out.c_str(), overwrite ? 1 : 0);
  if (s != CUVHS_OK) {
    fprintf(stderr, "Pipeline failed: %s\n", cuvhs_status_string(s));
    return 1;
  }
  fprintf(stderr, "Done.\n");
  return 0;
}
