/*
 * C-callable driver around the UNMODIFIED reference sbd headers (walkup/sbd-ykt).
 *
 * TEST INFRASTRUCTURE ONLY. Built by oracle/Makefile into oracle/_ref/ from the
 * reference sources where they lie; used by tests/golden/make_golden.py to
 * produce golden fixtures, by the CPU test suite to pin the C restatement
 * (oracle/sbd_oracle.c), and by bench.py's CPU-baseline / reference arm.
 * Nothing in the product library links or calls this.
 *
 * Every entry point converts plain arrays (one uint64 per spin string, bit p =
 * orbital p; integrals as an L*L one-body matrix and an 8-fold packed ERI array)
 * into the reference's own types and calls the reference's own functions:
 *   - GenerateExcitation + MakeSmartHelper   chemistry/tpb/helper.h:132-197, 367-437
 *   - Hij                                     chemistry/basic/determinants.h:467-526
 *   - makeQChamDiagTerms                      chemistry/tpb/qcham.h:314-366
 *   - mult (on-the-fly sigma)                 chemistry/tpb/mult.h:376-632
 *   - Correlation (1-/2-RDM)                  chemistry/tpb/correlation.h:194-444
 *   - sbd::tpb::diag (struct and file paths)  chemistry/tpb/sbdiag.h:113-477, 493-586
 */
#include "ref_prelude.h"
#include "sbd/sbd.h"

#include <cstring>
#include <fstream>
#include <sstream>

namespace {

using Dets = std::vector<std::vector<size_t>>;

Dets to_words(const uint64_t* s, size_t n, int L, size_t bl) {
  size_t nw = ((size_t)L + bl - 1) / bl;
  Dets out(n, std::vector<size_t>(nw, 0));
  const uint64_t word_mask = (bl >= 64) ? ~0ull : ((1ull << bl) - 1ull);
  for (size_t i = 0; i < n; ++i)
    for (size_t w = 0; w < nw; ++w)
      out[i][w] = (size_t)((s[i] >> (w * bl)) & word_mask);
  return out;
}

uint64_t from_words(const std::vector<size_t>& v, size_t bl) {
  uint64_t x = 0;
  for (size_t w = 0; w < v.size(); ++w) x |= (uint64_t)v[w] << (w * bl);
  return x;
}

size_t eri_index(int p, int q, int r, int s) {
  size_t pq = p > q ? (size_t)p * (p + 1) / 2 + q : (size_t)q * (q + 1) / 2 + p;
  size_t rs = r > s ? (size_t)r * (r + 1) / 2 + s : (size_t)s * (s + 1) / 2 + r;
  return pq > rs ? pq * (pq + 1) / 2 + rs : rs * (rs + 1) / 2 + pq;
}

sbd::FCIDump make_fcidump(int L, int nelec, double I0, const double* h, const double* eri) {
  sbd::FCIDump fd;
  fd.header["NORB"] = std::to_string(L);
  fd.header["NELEC"] = std::to_string(nelec);
  fd.header["MS2"] = "0";
  // one line per 8-fold class: (pq|rs) with p>=q, r>=s, pair(pq) >= pair(rs)
  for (int p = 0; p < L; ++p)
    for (int q = 0; q <= p; ++q)
      for (int r = 0; r <= p; ++r)
        for (int s = 0; s <= r; ++s) {
          size_t pq = (size_t)p * (p + 1) / 2 + q, rs = (size_t)r * (r + 1) / 2 + s;
          if (rs > pq) continue;
          fd.integrals.emplace_back(eri[eri_index(p, q, r, s)], p + 1, q + 1, r + 1, s + 1);
        }
  for (int p = 0; p < L; ++p)
    for (int q = 0; q <= p; ++q) fd.integrals.emplace_back(h[(size_t)p * L + q], p + 1, q + 1, 0, 0);
  fd.integrals.emplace_back(I0, 0, 0, 0, 0);
  return fd;
}

struct Ham {
  int L = 0, N = 0;
  double I0 = 0;
  sbd::oneInt<double> I1;
  sbd::twoInt<double> I2;
};

Ham setup(int L, int nelec, double I0, const double* h, const double* eri) {
  Ham H;
  sbd::FCIDump fd = make_fcidump(L, nelec, I0, h, eri);
  sbd::SetupIntegrals(fd, H.L, H.N, H.I0, H.I1, H.I2);
  return H;
}

// World-size-1 task helpers exactly as MakeHelpers builds them (helper.h:447-589):
// three tasks with types 2,1,0 over the full bra/ket ranges.
void make_helpers(const Dets& a, const Dets& b, size_t bl, int L,
                  std::vector<sbd::TaskHelpers>& helper, std::vector<std::vector<size_t>>& shm) {
  MPI_Comm h_comm = 0, b_comm = 0, t_comm = 0;
  sbd::MakeHelpers(a, b, bl, (size_t)L, helper, shm, h_comm, b_comm, t_comm, 1, 1);
}

}  // namespace

extern "C" {

int ref_version() { return 1; }

/* Connectivity lists of the reference for one pair of string sets.
 * Output layout = MakeSmartHelper's shared memory (helper.h:367-437): for each
 * alpha bra: singles then doubles (ascending ket index); then for each beta bra
 * the same. Lengths returned per bra. `flat` may be NULL to query the size. */
long long ref_connectivity(const uint64_t* astr, size_t na, const uint64_t* bstr, size_t nb, int L,
                           int bit_length, uint64_t* a_slen, uint64_t* a_dlen, uint64_t* b_slen,
                           uint64_t* b_dlen, uint64_t* flat, long long flat_cap) {
  size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  sbd::TaskHelpers hp;
  hp.braAlphaStart = 0; hp.braAlphaEnd = na; hp.ketAlphaStart = 0; hp.ketAlphaEnd = na;
  hp.braBetaStart = 0; hp.braBetaEnd = nb; hp.ketBetaStart = 0; hp.ketBetaEnd = nb;
  hp.taskType = 0; hp.adetShift = 0; hp.bdetShift = 0;
  sbd::GenerateExcitation(a, b, bl, (size_t)L, hp);
  std::vector<size_t> shm;
  sbd::MakeSmartHelper(hp, shm);
  for (size_t i = 0; i < na; ++i) { a_slen[i] = hp.SinglesFromAlphaLen[i]; a_dlen[i] = hp.DoublesFromAlphaLen[i]; }
  for (size_t i = 0; i < nb; ++i) { b_slen[i] = hp.SinglesFromBetaLen[i]; b_dlen[i] = hp.DoublesFromBetaLen[i]; }
  long long n = (long long)shm.size();
  if (flat && flat_cap >= n)
    for (long long i = 0; i < n; ++i) flat[i] = shm[(size_t)i];
  sbd::FreeHelpers(hp);
  return n;
}

/* Matrix elements <bra|H|ket> by the reference Hij for n determinant pairs
 * (determinants.h:467-526; interleaved spin-orbital layout built by
 * DetFromAlphaBeta :97-119). orb_diff receives the reference's orbDiff code. */
void ref_hij(int L, int nelec, double I0, const double* h, const double* eri, int bit_length,
             size_t n, const uint64_t* bra_a, const uint64_t* bra_b, const uint64_t* ket_a,
             const uint64_t* ket_b, double* out, uint64_t* orb_diff) {
  Ham H = setup(L, nelec, I0, h, eri);
  size_t bl = (size_t)bit_length;
  for (size_t k = 0; k < n; ++k) {
    Dets ba = to_words(&bra_a[k], 1, L, bl), bb = to_words(&bra_b[k], 1, L, bl);
    Dets ka = to_words(&ket_a[k], 1, L, bl), kb = to_words(&ket_b[k], 1, L, bl);
    auto DI = sbd::DetFromAlphaBeta(ba[0], bb[0], bl, (size_t)L);
    auto DJ = sbd::DetFromAlphaBeta(ka[0], kb[0], bl, (size_t)L);
    size_t od = 0;
    size_t Ls = (size_t)L;
    out[k] = sbd::Hij(DI, DJ, bl, Ls, H.I0, H.I1, H.I2, od);
    if (orb_diff) orb_diff[k] = od;
  }
}

/* Diagonal terms hii (qcham.h:314-366), alpha-major index ia*nb+ib. */
void ref_diag_terms(int L, int nelec, double I0, const double* h, const double* eri, int bit_length,
                    const uint64_t* astr, size_t na, const uint64_t* bstr, size_t nb, double* hii) {
  Ham H = setup(L, nelec, I0, h, eri);
  size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  std::vector<sbd::TaskHelpers> helper;
  std::vector<std::vector<size_t>> shm;
  make_helpers(a, b, bl, L, helper, shm);
  std::vector<double> d;
  sbd::makeQChamDiagTerms(a, b, bl, (size_t)L, helper, H.I0, H.I1, H.I2, d, 0, 0, 0);
  std::memcpy(hii, d.data(), sizeof(double) * na * nb);
  sbd::FreeHelpers(helper);
}

/* One on-the-fly sigma S = H C (mult.h:376-632) at world size 1. */
void ref_sigma(int L, int nelec, double I0, const double* h, const double* eri, int bit_length,
               const uint64_t* astr, size_t na, const uint64_t* bstr, size_t nb, const double* C,
               double* S) {
  Ham H = setup(L, nelec, I0, h, eri);
  size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  std::vector<sbd::TaskHelpers> helper;
  std::vector<std::vector<size_t>> shm;
  make_helpers(a, b, bl, L, helper, shm);
  std::vector<double> hii;
  sbd::makeQChamDiagTerms(a, b, bl, (size_t)L, helper, H.I0, H.I1, H.I2, hii, 0, 0, 0);
  std::vector<double> Wk(C, C + na * nb), Wb(na * nb, 0.0);
  sbd::mult(hii, Wk, Wb, a, b, bl, (size_t)L, 1, 1, helper, H.I0, H.I1, H.I2, 0, 0, 0);
  std::memcpy(S, Wb.data(), sizeof(double) * na * nb);
  sbd::FreeHelpers(helper);
}

/* A bounded sample of the reference sigma for CPU-baseline timing: the
 * reference mult over helpers whose bra alpha range is restricted to
 * [row0, row0 + rows) (ket ranges stay full), exactly the per-task loops of
 * mult.h:453-610, which index the bra block relative to its start as an MPI
 * rank's block would be. The helpers are built once; mult runs `reps` times
 * and seconds[r] receives the duration of run r. *pairs receives the number
 * of off-diagonal det-pairs one run evaluates. Returns the mean seconds. */
double ref_sigma_sample_range(int L, int nelec, double I0, const double* h, const double* eri,
                              int bit_length, const uint64_t* astr, size_t na, const uint64_t* bstr,
                              size_t nb, const double* C, double* S, size_t row0, size_t rows, int threads,
                              int reps, double* seconds, double* pairs) {
  if (threads > 0) omp_set_num_threads(threads);
  Ham H = setup(L, nelec, I0, h, eri);
  size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  if (row0 >= na) row0 = na - 1;
  if (rows > na - row0) rows = na - row0;
  std::vector<sbd::TaskHelpers> helper(3);
  const size_t types[3] = {2, 1, 0};
  std::vector<std::vector<size_t>> shm(3);
  for (int t = 0; t < 3; ++t) {
    sbd::TaskHelpers& hp = helper[t];
    hp.braAlphaStart = row0; hp.braAlphaEnd = row0 + rows; hp.ketAlphaStart = 0; hp.ketAlphaEnd = na;
    hp.braBetaStart = 0; hp.braBetaEnd = nb; hp.ketBetaStart = 0; hp.ketBetaEnd = nb;
    hp.taskType = types[t]; hp.adetShift = 0; hp.bdetShift = 0;
    sbd::GenerateExcitation(a, b, bl, (size_t)L, hp);
    sbd::MakeSmartHelper(hp, shm[t]);
  }
  double np = 0;
  for (size_t ia = 0; ia < rows; ++ia) {
    double sa = (double)helper[0].SinglesFromAlphaLen[ia], da = (double)helper[0].DoublesFromAlphaLen[ia];
    np += (sa + da) * (double)nb;
    for (size_t ib = 0; ib < nb; ++ib)
      np += (double)(helper[0].SinglesFromBetaLen[ib] + helper[0].DoublesFromBetaLen[ib]) +
            sa * (double)helper[0].SinglesFromBetaLen[ib];
  }
  if (pairs) *pairs = np;
  // the diagonal loop of mult runs over T.size() == na*nb, so hii and Wb are full size
  std::vector<double> hii(na * nb, 0.0);
  std::vector<double> Wk(C, C + na * nb), Wb(na * nb, 0.0);
  double total = 0.0;
  for (int r = 0; r < reps; ++r) {
    std::fill(Wb.begin(), Wb.end(), 0.0);
    auto t0 = std::chrono::high_resolution_clock::now();
    sbd::mult(hii, Wk, Wb, a, b, bl, (size_t)L, 1, 1, helper, H.I0, H.I1, H.I2, 0, 0, 0);
    auto t1 = std::chrono::high_resolution_clock::now();
    double dt = std::chrono::duration<double>(t1 - t0).count();
    if (seconds) seconds[r] = dt;
    total += dt;
  }
  if (S) std::memcpy(S, Wb.data(), sizeof(double) * rows * nb);
  sbd::FreeHelpers(helper);
  return reps > 0 ? total / reps : 0.0;
}

double ref_sigma_sample_multi(int L, int nelec, double I0, const double* h, const double* eri,
                              int bit_length, const uint64_t* astr, size_t na, const uint64_t* bstr,
                              size_t nb, const double* C, double* S, size_t rows, int threads,
                              int reps, double* seconds, double* pairs) {
  return ref_sigma_sample_range(L, nelec, I0, h, eri, bit_length, astr, na, bstr, nb, C, S, 0, rows, threads,
                                reps, seconds, pairs);
}

double ref_sigma_sample(int L, int nelec, double I0, const double* h, const double* eri,
                        int bit_length, const uint64_t* astr, size_t na, const uint64_t* bstr,
                        size_t nb, const double* C, double* S, size_t rows, int threads,
                        double* pairs) {
  return ref_sigma_sample_multi(L, nelec, I0, h, eri, bit_length, astr, na, bstr, nb, C, S, rows,
                                threads, 1, nullptr, pairs);
}

/* 1-/2-RDM of a given vector W by the reference Correlation
 * (correlation.h:194-444). one: 2*L*L, two: 4*L^4 (reference index order). */
void ref_rdm(int L, const uint64_t* astr, size_t na, const uint64_t* bstr, size_t nb,
             int bit_length, const double* W, double* one, double* two) {
  size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  std::vector<sbd::TaskHelpers> helper;
  std::vector<std::vector<size_t>> shm;
  make_helpers(a, b, bl, L, helper, shm);
  std::vector<double> w(W, W + na * nb);
  std::vector<std::vector<double>> o, t;
  sbd::Correlation(w, a, b, bl, (size_t)L, 1, 1, helper, 0, 0, 0, o, t);
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  for (int s = 0; s < 2; ++s) std::memcpy(one + s * L2, o[s].data(), sizeof(double) * L2);
  for (int s = 0; s < 4; ++s) std::memcpy(two + s * L4, t[s].data(), sizeof(double) * L4);
  sbd::FreeHelpers(helper);
}

/* The reference Davidson driver sequence of tpb::diag (sbdiag.h:157-273) at
 * world size 1, returning the energy <W|HW> and the final vector W. */
double ref_davidson(int L, int nelec, double I0, const double* h, const double* eri,
                    int bit_length, const uint64_t* astr, size_t na, const uint64_t* bstr,
                    size_t nb, int max_it, int max_nb, double eps, double* W_out) {
  Ham H = setup(L, nelec, I0, h, eri);
  size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  std::vector<sbd::TaskHelpers> helper;
  std::vector<std::vector<size_t>> shm;
  make_helpers(a, b, bl, L, helper, shm);
  std::vector<double> W;
  sbd::BasisInitVector(W, a, b, 1, 1, 0, 0, 0, 0);
  std::vector<double> hii;
  sbd::makeQChamDiagTerms(a, b, bl, (size_t)L, helper, H.I0, H.I1, H.I2, hii, 0, 0, 0);
  sbd::Davidson(hii, W, a, b, bl, (size_t)L, 1, 1, helper, H.I0, H.I1, H.I2, 0, 0, 0, max_it,
                max_nb, eps, 86400.0);
  std::vector<double> C(W.size(), 0.0);
  sbd::mult(hii, W, C, a, b, bl, (size_t)L, 1, 1, helper, H.I0, H.I1, H.I2, 0, 0, 0);
  double E = 0.0;
  sbd::InnerProduct(W, C, E, 0);
  if (W_out) std::memcpy(W_out, W.data(), sizeof(double) * W.size());
  sbd::FreeHelpers(helper);
  return E;
}

/* sbd::tpb::diag, struct path (sbdiag.h:113-477), exact doubles in, outputs
 * copied out. carry: up to carry_cap strings (uint64), returns the count.
 * one/two may be NULL when do_rdm == 0. */
long long ref_tpb_diag(int L, int nelec, double I0, const double* h, const double* eri,
                       const uint64_t* astr, size_t na, const uint64_t* bstr, size_t nb,
                       int bit_length, int max_it, int max_nb, double eps, int do_rdm, double ratio,
                       double threshold, double* energy, double* density, uint64_t* carry,
                       long long carry_cap, double* one, double* two) {
  sbd::FCIDump fd = make_fcidump(L, nelec, I0, h, eri);
  size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  sbd::tpb::SBD p;
  p.max_it = max_it; p.max_nb = max_nb; p.eps = eps; p.do_rdm = do_rdm;
  p.ratio = ratio; p.threshold = threshold; p.bit_length = bl;
  double e = 0;
  std::vector<double> dens;
  Dets co;
  std::vector<std::vector<double>> o, t;
  sbd::tpb::diag(0, p, fd, a, b, std::string(""), std::string(""), e, dens, co, o, t);
  *energy = e;
  std::memcpy(density, dens.data(), sizeof(double) * dens.size());
  long long nco = (long long)co.size();
  for (long long k = 0; k < nco && k < carry_cap; ++k) carry[k] = from_words(co[(size_t)k], bl);
  if (do_rdm && one && two) {
    size_t L2 = (size_t)L * L, L4 = L2 * L2;
    for (int s = 0; s < 2; ++s) std::memcpy(one + s * L2, o[s].data(), sizeof(double) * L2);
    for (int s = 0; s < 4; ++s) std::memcpy(two + s * L4, t[s].data(), sizeof(double) * L4);
  }
  return nco;
}

/* sbd::tpb::diag, file-name path (sbdiag.h:493-586): FCIDUMP text file and
 * alpha-string .txt file (bdet = adet, shuffle 0). This path re-parses the
 * integrals through the broadcast text round trip (fcidump.h:156-169,251). */
long long ref_tpb_diag_files(const char* fcidump, const char* adetfile, int bit_length, int max_it,
                             int max_nb, double eps, int do_rdm, double ratio, double threshold,
                             double* energy, double* density, int density_cap, uint64_t* carry,
                             long long carry_cap, double* one, double* two) {
  sbd::tpb::SBD p;
  p.max_it = max_it; p.max_nb = max_nb; p.eps = eps; p.do_rdm = do_rdm;
  p.ratio = ratio; p.threshold = threshold; p.bit_length = (size_t)bit_length;
  double e = 0;
  std::vector<double> dens;
  Dets co;
  std::vector<std::vector<double>> o, t;
  sbd::tpb::diag(0, p, std::string(fcidump), std::string(adetfile), std::string(""),
                 std::string(""), e, dens, co, o, t);
  *energy = e;
  for (int i = 0; i < density_cap && i < (int)dens.size(); ++i) density[i] = dens[(size_t)i];
  long long nco = (long long)co.size();
  for (long long k = 0; k < nco && k < carry_cap; ++k)
    carry[k] = from_words(co[(size_t)k], (size_t)bit_length);
  if (do_rdm && one && two && !o.empty()) {
    size_t L = (size_t)std::sqrt((double)o[0].size());
    size_t L2 = L * L, L4 = L2 * L2;
    for (int s = 0; s < 2; ++s) std::memcpy(one + s * L2, o[s].data(), sizeof(double) * L2);
    for (int s = 0; s < 4; ++s) std::memcpy(two + s * L4, t[s].data(), sizeof(double) * L4);
  }
  return nco;
}

/* LoadAlphaDets (makedeterminants.h:160-185): parsed, sorted, deduped strings. */
long long ref_load_alpha_dets(const char* path, int L, int bit_length, uint64_t* out, long long cap) {
  Dets a;
  sbd::LoadAlphaDets(std::string(path), a, (size_t)bit_length, (size_t)L);
  long long n = (long long)a.size();
  for (long long k = 0; k < n && k < cap; ++k) out[k] = from_words(a[(size_t)k], (size_t)bit_length);
  return n;
}

/* The FCIDUMP after the reference's broadcast text round trip
 * (LoadFCIDump fcidump.h:27-139 -> MpiBcast :226-253 -> SetupIntegrals
 * makeintegrals.h:81-126): the integrals the file path actually solves with. */
int ref_fcidump_roundtrip(const char* path, int* L_out, int* nelec_out, double* I0_out, double* h,
                          double* eri, long long eri_cap) {
  sbd::FCIDump fd = sbd::LoadFCIDump(std::string(path));
  sbd::MpiBcast(fd, 0, 0);
  int L = 0, N = 0;
  double I0 = 0;
  sbd::oneInt<double> I1;
  sbd::twoInt<double> I2;
  sbd::SetupIntegrals(fd, L, N, I0, I1, I2);
  *L_out = L; *nelec_out = N; *I0_out = I0;
  if (h)
    for (int p = 0; p < L; ++p)
      for (int q = 0; q < L; ++q) h[(size_t)p * L + q] = I1.Value(2 * p, 2 * q);
  if (eri)
    for (long long k = 0; k < (long long)I2.store.size() && k < eri_cap; ++k) eri[k] = I2.store[(size_t)k];
  return (int)I2.store.size();
}

// Reference SaveWavefunction (chemistry/tpb/restart.h:20-67) at world size 1:
// writes file + "000000".
int ref_save_wavefunction(const char* file, const uint64_t* astr, size_t na, const uint64_t* bstr, size_t nb,
                          int L, int bit_length, const double* W) {
  const size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  std::vector<double> w(W, W + na * nb);
  MPI_Comm h_comm = 0, b_comm = 0, t_comm = 0;
  sbd::SaveWavefunction(std::string(file), a, b, 1, 1, h_comm, b_comm, t_comm, w);
  return 0;
}

// Reference LoadWavefunction (chemistry/tpb/restart.h:414-657) at world size 1
// onto the basis (astr, bstr): W receives na*nb doubles.
int ref_load_wavefunction(const char* file, const uint64_t* astr, size_t na, const uint64_t* bstr, size_t nb,
                          int L, int bit_length, double* W) {
  const size_t bl = (size_t)bit_length;
  Dets a = to_words(astr, na, L, bl), b = to_words(bstr, nb, L, bl);
  std::vector<double> w;
  MPI_Comm h_comm = 0, b_comm = 0, t_comm = 0;
  sbd::LoadWavefunction(std::string(file), a, b, 1, 1, h_comm, b_comm, t_comm, w);
  if (w.size() != na * nb) return 1;
  std::memcpy(W, w.data(), sizeof(double) * na * nb);
  return 0;
}

}  // extern "C"
