// `tetfit` command-line driver over the C ABI (include/tetfit.h), in place
// of the reference's src/DGA/main/dga_main.cpp:40-62: parse the script once,
// then run every simulation in label order, each writing its probe files
// (<name><label>_probe_E.dat / _probe_H.dat) and poynting.dat into the
// working directory.
//
//   tetfit [--fp32] [--device N] [--digits D] input_file
//
// --digits D writes the probe files with D significant digits (the reference
// writes 6).
//
// With no input file it prints the reference's "Input file missing!" text.
// Script errors print the reference's "Input file error at line N: ..." text.
// Every error exits with status 1 (the reference throws and aborts instead).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tetfit.h"

namespace {

int usage_error() {
  std::printf("Input file error at line 0: Input file missing! Correct use is: \"tetfit input_file\" \n");
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  std::printf("    TetFIT time-domain Maxwell solver, B200 build (sm_100a)\n\n");
  tf_opts o;
  tf_default_opts(&o);
  o.write_files = 1;
  o.verbose = 1;
  const char* input = nullptr;
  for (int k = 1; k < argc; k++) {
    if (std::strcmp(argv[k], "--fp32") == 0) {
      o.precision = TF_FP32;
    } else if (std::strcmp(argv[k], "--device") == 0 && k + 1 < argc) {
      o.device = std::atoi(argv[++k]);
    } else if (std::strcmp(argv[k], "--digits") == 0 && k + 1 < argc) {
      o.file_digits = std::atoi(argv[++k]);
    } else if (argv[k][0] == '-' && argv[k][1] == '-') {
      std::printf("unknown option %s\n", argv[k]);
      return 1;
    } else if (!input) {
      input = argv[k];
    } else {
      return usage_error();
    }
  }
  if (!input) return usage_error();
  tf_ctx* ctx = nullptr;
  if (tf_open(input, &ctx) != TF_OK) {
    std::printf("%s\n", tf_last_error(ctx));
    tf_close(ctx);
    return 1;
  }
  uint32_t n = 0;
  tf_simulations(ctx, nullptr, 0, &n);
  std::vector<uint32_t> labels(n);
  tf_simulations(ctx, labels.data(), n, &n);
  for (uint32_t label : labels) {
    if (tf_run(ctx, label, &o) != TF_OK) {
      std::printf("simulation %u: %s\n", label, tf_last_error(ctx));
      tf_close(ctx);
      return 1;
    }
  }
  tf_close(ctx);
  return 0;
}
