// rnj_cli.cpp -- rnj-b200: rapidNJ's distance-matrix mode ("rapidnj <file> -o m")
// on the GPU, as a standalone program over the C ABI of librnjgpu.so.
//
// Options follow rapidNJ's (main.cpp:576-599) for the part of its CLI that
// computes a distance matrix:
//   <file>            alignment (single-line FASTA or Stockholm; picked by extension,
//                     or -i fa / -i sth)
//   -o m              the distance matrix (the only output of this program)
//   -a jc|kim         evolution model (default kim, main.cpp:253-274)
//   -t d|p            force DNA or protein (default: detected from the first sequence)
//   -f                naive estimator (no bit-string fast path)
//   -x <file>         write the matrix there instead of stdout
//   -c <n>            host threads for the row copy and text formatting
//   -g <n>            GPU device (default 0)
//   -v                timing of each stage on stderr
// Output: the "-o m" text of main.cpp:212-221.  Errors: a message on stderr and
// exit status 1.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <string>
#include <vector>

#include "rnj.h"

namespace {

void die(const std::string &what) {
  fprintf(stderr, "ERROR: %s%s%s\n", what.c_str(), *rnj_last_error() ? ": " : "", rnj_last_error());
  exit(1);
}

void usage() {
  fprintf(stderr,
          "usage: rnj-b200 <alignment> [-o m] [-a jc|kim] [-t d|p] [-f] [-i fa|sth] [-x outfile]\n"
          "                [-c threads] [-g device] [-v]\n");
  exit(1);
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char **argv) {
  const char *path = nullptr, *out = nullptr, *fmt = nullptr;
  int model = RNJ_KIMURA, type = RNJ_UNKNOWN, threads = 0, device = 0;
  bool fast = true, verbose = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&]() -> const char * {
      if (i + 1 >= argc) usage();
      return argv[++i];
    };
    if (a == "-a" || a == "--evolution-model") {
      const std::string m = val();
      if (m == "jc") model = RNJ_JC;
      else if (m == "kim") model = RNJ_KIMURA;
      else usage();
    } else if (a == "-t" || a == "--alignment-type") {
      const std::string t = val();
      if (t == "d") type = RNJ_DNA;
      else if (t == "p") type = RNJ_PROTEIN;
      else usage();
    } else if (a == "-o" || a == "--output-format") {
      if (std::string(val()) != "m") {
        fprintf(stderr, "ERROR: rnj-b200 writes distance matrices only (-o m)\n");
        exit(1);
      }
    } else if (a == "-f" || a == "--no-rapiddist") {
      fast = false;
    } else if (a == "-i" || a == "--input-format") {
      fmt = val();
    } else if (a == "-x" || a == "--outfile") {
      out = val();
    } else if (a == "-c" || a == "--cores") {
      threads = atoi(val());
    } else if (a == "-g" || a == "--gpu") {
      device = atoi(val());
    } else if (a == "-v" || a == "--verbose") {
      verbose = true;
    } else if (a == "-h" || a == "--help") {
      usage();
    } else if (!a.empty() && a[0] == '-') {
      usage();
    } else {
      path = argv[i];
    }
  }
  if (!path) usage();

  double t0 = now();
  rnj_ctx *ctx = nullptr;
  if (rnj_ctx_create(device, &ctx) != RNJ_OK) die("GPU context");
  // The alignment is parsed on the device, the matrix stays there and is
  // formatted there; only its text comes back.
  rnj_msa *msa = nullptr;
  if (rnj_msa_read_device(ctx, path, fmt, &msa) != RNJ_OK) die("could not read the alignment");
  int n = 0, L = 0, detected = RNJ_DNA;
  rnj_msa_info(msa, &n, &L, &detected);
  if (type == RNJ_UNKNOWN) type = detected;
  double t1 = now();

  std::vector<const char *> names(n);
  for (int i = 0; i < n; ++i) names[i] = rnj_msa_name(msa, i);
  float mx = 0.0f;
  double t2 = t1;
  if (n == 0) {
    if (rnj_write_matrix_text(out, names.data(), nullptr, 0, threads) != RNJ_OK)
      die("writing the matrix");
  } else {
    const void *d_chars = nullptr;
    size_t ld = 0;
    rnj_aln *aln = nullptr;
    rnj_mat *mat = nullptr;
    if (rnj_msa_device_chars(msa, &d_chars, &ld) != RNJ_OK ||
        rnj_aln_from_device(ctx, d_chars, n, L, ld, type, fast ? RNJ_FASTDIST : 0, &aln) != RNJ_OK ||
        rnj_distance(ctx, aln, model, &mat) != RNJ_OK)
      die("distance computation");
    float *d_m = nullptr;
    size_t ldm = 0;
    if (rnj_mat_device_ptr(mat, &d_m, &ldm) != RNJ_OK || rnj_mat_info(mat, nullptr, &mx) != RNJ_OK)
      die("distance computation");
    t2 = now();
    if (rnj_write_matrix_text_device(ctx, out, names.data(), d_m, ldm, n) != RNJ_OK)
      die("writing the matrix");
    rnj_mat_destroy(mat);
    rnj_aln_destroy(aln);
  }
  double t3 = now();
  if (verbose)
    fprintf(stderr, "read %.3f s, distances %.3f s (max %g), text %.3f s; %d sequences x %d columns\n",
            t1 - t0, t2 - t1, (double)mx, t3 - t2, n, L);
  rnj_ctx_destroy(ctx);
  rnj_msa_destroy(msa);
  return 0;
}
