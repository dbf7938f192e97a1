/*
 * Command-line front end of the reference build (test infrastructure only).
 *
 *   sbd_ref_cli sigma-sample <input.bin> <rows> <reps> <threads> [<row0>]
 *
 * Reads a problem written by sbdx.synth.write_problem_bin (header: L, nelec,
 * na, nb as int64; I0; h[L*L]; eri[packed]; alpha strings; beta strings), runs
 * the reference's own sigma (mult.h:376-632) restricted to bra alpha rows
 * [row0, row0 + rows) (row0 = 0 by default) `reps` times (helpers built once), and prints one JSON line per
 * run with the seconds and the number of off-diagonal det-pairs evaluated.
 */
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <string>
#include <omp.h>

extern "C" double ref_sigma_sample_range(int L, int nelec, double I0, const double* h,
                                         const double* eri, int bit_length, const uint64_t* astr,
                                         size_t na, const uint64_t* bstr, size_t nb, const double* C,
                                         double* S, size_t row0, size_t rows, int threads, int reps,
                                         double* seconds, double* pairs);

int main(int argc, char** argv) {
  if (argc < 6 || std::string(argv[1]) != "sigma-sample") {
    std::fprintf(stderr, "usage: %s sigma-sample <input.bin> <rows> <reps> <threads> [<row0>]\n", argv[0]);
    return 2;
  }
  FILE* f = std::fopen(argv[2], "rb");
  if (!f) { std::perror("open"); return 2; }
  int64_t hdr[4];
  if (std::fread(hdr, sizeof(int64_t), 4, f) != 4) return 3;
  int L = (int)hdr[0], nelec = (int)hdr[1];
  size_t na = (size_t)hdr[2], nb = (size_t)hdr[3];
  double I0;
  if (std::fread(&I0, sizeof(double), 1, f) != 1) return 3;
  size_t npair = (size_t)L * (L + 1) / 2, neri = npair * (npair + 1) / 2;
  std::vector<double> h((size_t)L * L), eri(neri);
  std::vector<uint64_t> a(na), b(nb);
  if (std::fread(h.data(), sizeof(double), h.size(), f) != h.size()) return 3;
  if (std::fread(eri.data(), sizeof(double), eri.size(), f) != eri.size()) return 3;
  if (std::fread(a.data(), sizeof(uint64_t), na, f) != na) return 3;
  if (std::fread(b.data(), sizeof(uint64_t), nb, f) != nb) return 3;
  std::fclose(f);
  size_t rows = (size_t)std::atoll(argv[3]);
  int reps = std::atoi(argv[4]);
  int threads = std::atoi(argv[5]);
  const size_t row0 = argc > 6 ? (size_t)std::atoll(argv[6]) : 0;
  if (threads <= 0) threads = omp_get_max_threads();
  std::vector<double> C(na * nb);
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (size_t i = 0; i < C.size(); ++i) {  // deterministic pseudo-random vector
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    C[i] = (double)(s >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
  std::vector<double> secs(reps > 0 ? reps : 1);
  double pairs = 0;
  ref_sigma_sample_range(L, nelec, I0, h.data(), eri.data(), 20, a.data(), na, b.data(), nb, C.data(),
                         nullptr, row0, rows, threads, reps, secs.data(), &pairs);
  for (int r = 0; r < reps; ++r)
    std::printf("{\"seconds\": %.6f, \"pairs\": %.0f, \"rows\": %zu, \"row0\": %zu, \"threads\": %d}\n",
                secs[r], pairs, rows, row0, threads);
  std::fflush(stdout);
  return 0;
}
