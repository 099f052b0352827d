// lbmc_run: the command-line program that replaces the reference's
// executable (LBM-C/index.cu:61-153): `lbmc_run <input file>` reads the
// input file, builds the model from the domain directory, runs the time
// loop with file output, screen messages and the steady-state test, and
// exits with 1 when the state becomes non-finite, as the reference does.
// Options (not in the reference): --storage f32|f16|f16sr|bf16|f64,
// --streaming shift|aa, --device N, --quiet.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "lbmc.h"

static void usage() {
  fprintf(stderr, "usage: lbmc_run <input file> [--storage f32|f16|f16sr|bf16|f64] [--streaming shift|aa] "
                  "[--device N] [--quiet]\n");
}

int main(int argc, char **argv) {
  if (argc < 2) {
    usage();
    return 2;
  }
  lbmc_config ov;
  lbmc_config_default(&ov, LBMC_D2Q9);
  ov.streaming = LBMC_STREAM_AA;
  int quiet = 0;
  for (int k = 2; k < argc; k++) {
    const char *a = argv[k];
    const char *v = k + 1 < argc ? argv[k + 1] : "";
    if (!strcmp(a, "--quiet")) {
      quiet = 1;
    } else if (!strcmp(a, "--storage")) {
      ov.storage = !strcmp(v, "f16")     ? LBMC_F16
                   : !strcmp(v, "f16sr") ? LBMC_F16_SR
                   : !strcmp(v, "bf16")  ? LBMC_BF16
                   : !strcmp(v, "f64")   ? LBMC_F64
                                         : LBMC_F32;
      k++;
    } else if (!strcmp(a, "--streaming")) {
      ov.streaming = !strcmp(v, "shift") ? LBMC_STREAM_SHIFT : LBMC_STREAM_AA;
      k++;
    } else if (!strcmp(a, "--device")) {
      ov.device = atoi(v);
      k++;
    } else {
      usage();
      return 2;
    }
  }
  lbmc_run_result r;
  const lbmc_status s = lbmc_run(argv[1], &ov, quiet, &r);
  if (s == LBMC_ERR_NAN) {
    fprintf(stderr, "non-finite state at step %lld\n", r.steps);
    return 1;
  }
  if (s != LBMC_OK) {
    fprintf(stderr, "lbmc_run: %s: %s\n", lbmc_status_string(s), lbmc_last_error());
    return 3;
  }
  if (!quiet)
    printf("steps %lld, %s, %d outputs, %.3f s\n", r.steps, r.steady ? "steady state reached" : "MaxT reached",
           r.outputs, r.seconds);
  return 0;
}
