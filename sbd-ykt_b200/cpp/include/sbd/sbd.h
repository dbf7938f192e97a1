// sbd/sbd.h -- drop-in header API of the sbd tensor-product-basis path
// (walkup/sbd-ykt, namespace sbd / sbd::tpb) running on the B200 CUDA library
// through the C-ABI in sbdx.h.
//
// Include this header instead of the reference's sbd/sbd.h and link
// libsbdx.so. The names, argument meaning, output shapes and error behaviour
// of the entry points below follow the reference:
//   sbd::FCIDump, LoadFCIDump, MpiBcast(FCIDump)      framework/fcidump.h:18-253
//   sbd::from_string, makestring                        framework/bit_manipulation.h:135-172
//   sbd::LoadAlphaDets                                  chemistry/basic/makedeterminants.h:160-185
//   sbd::tpb::SBD, generate_sbd_data                    chemistry/tpb/sbdiag.h:12-96
//   sbd::tpb::diag (struct and file-name overloads)     chemistry/tpb/sbdiag.h:113-477, 493-586
//   sbd::SaveWavefunction / LoadWavefunction format     chemistry/tpb/restart.h:20-67, 414-657
//   sbd::SaveMatrixFormWF                               chemistry/tpb/restart.h:662-780
// The path runs at MPI world size 1 on one GPU: the communicator argument is
// accepted with any type (MPI_Comm or a placeholder) and is not used. The GPU
// is CUDA device SBDX_DEVICE (environment, default 0); SBDX_PRECISION=fp32
// selects the FP32-storage defect-correction solver, SBDX_AUTOTUNE=1 times the
// kernel shapes before solving. Errors throw std::runtime_error (the reference
// throws std::runtime_error / std::invalid_argument on bad input).
#ifndef SBD_B200_SBD_H
#define SBD_B200_SBD_H

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <numeric>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "sbdx.h"

namespace sbd {

// ---- FCIDUMP ---------------------------------------------------------------

struct FCIDump {
  std::map<std::string, std::string> header;
  std::vector<std::tuple<double, int, int, int, int>> integrals;
};

namespace detail {
inline std::string trim(const std::string& s) {
  const size_t b = s.find_first_not_of(" \t");
  if (b == std::string::npos) return "";
  const size_t e = s.find_last_not_of(" \t");
  return s.substr(b, e - b + 1);
}
inline void parse_header(const std::string& content, FCIDump& fd) {
  std::stringstream hs(content);
  std::string token;
  while (std::getline(hs, token, ',')) {
    const size_t eq = token.find('=');
    if (eq == std::string::npos) continue;
    fd.header[trim(token.substr(0, eq))] = trim(token.substr(eq + 1));
  }
}
inline void parse_integral_line(const std::string& line, FCIDump& fd) {
  std::stringstream ss(line);
  double v;
  int i, j, k, l;
  ss >> v >> i >> j >> k >> l;
  fd.integrals.emplace_back(v, i, j, k, l);
}
}  // namespace detail

// LoadFCIDump: header lines up to &END (with "&FCI" removed) joined and split
// at commas into KEY=VALUE; every later non-empty, non-'!' line is
// "value i j k l".
inline FCIDump LoadFCIDump(const std::string& filename) {
  std::ifstream in(filename);
  if (!in.is_open()) throw std::runtime_error("Failed to open FCIDUMP file.");
  FCIDump fd;
  std::string line, header;
  bool in_header = true;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '!') continue;
    if (in_header) {
      if (line.find("&END") != std::string::npos) { in_header = false; continue; }
      const size_t p = line.find("&FCI");
      if (p != std::string::npos) line.erase(p, 4);
      header += line;
    } else {
      detail::parse_integral_line(line, fd);
    }
  }
  detail::parse_header(header, fd);
  return fd;
}

// Text form used by the reference's broadcast: values at the default stream
// precision (6 significant digits).
inline std::string serializeFCIDump(const FCIDump& fd) {
  std::ostringstream os;
  for (const auto& kv : fd.header) os << kv.first << "=" << kv.second << ",\n";
  os << "&END\n";
  for (const auto& t : fd.integrals)
    os << std::get<0>(t) << " " << std::get<1>(t) << " " << std::get<2>(t) << " " << std::get<3>(t) << " "
       << std::get<4>(t) << "\n";
  return os.str();
}

inline FCIDump deserializeFCIDump(const std::string& data) {
  FCIDump fd;
  std::istringstream is(data);
  std::string line, header;
  bool in_header = true;
  while (std::getline(is, line)) {
    if (line.empty()) continue;
    if (in_header) {
      if (line.find("&END") != std::string::npos) { in_header = false; continue; }
      header += line + " ";
    } else {
      detail::parse_integral_line(line, fd);
    }
  }
  detail::parse_header(header, fd);
  return fd;
}

// At world size 1 the reference's broadcast is a serialise/parse round trip on
// the root itself, which rounds every integral to 6 significant digits.
template <typename Comm>
inline void MpiBcast(FCIDump& fd, int /*root*/, Comm /*comm*/) {
  fd = deserializeFCIDump(serializeFCIDump(fd));
}

// ---- bit strings -----------------------------------------------------------

inline std::vector<size_t> from_string(const std::string& s, size_t bit_length, size_t L) {
  std::vector<size_t> r((L + bit_length - 1) / bit_length, 0);
  for (size_t i = 0; i < L; ++i)
    if (s[L - 1 - i] == '1') r[i / bit_length] |= size_t(1) << (i % bit_length);
  return r;
}

inline std::string makestring(const std::vector<size_t>& c, size_t bit_length, size_t L) {
  std::string s;
  for (size_t i = L; i > 0; --i) s += (c[(i - 1) / bit_length] >> ((i - 1) % bit_length)) & 1 ? '1' : '0';
  return s;
}

namespace detail {
inline bool words_less(const std::vector<size_t>& a, const std::vector<size_t>& b) {
  for (size_t n = a.size(); n > 0; --n) {
    if (a[n - 1] < b[n - 1]) return true;
    if (a[n - 1] > b[n - 1]) return false;
  }
  return false;
}
inline uint64_t to_u64(const std::vector<size_t>& w, size_t bit_length) {
  uint64_t x = 0;
  for (size_t k = 0; k < w.size(); ++k) x |= (uint64_t)w[k] << (k * bit_length);
  return x;
}
inline std::vector<size_t> from_u64(uint64_t x, size_t bit_length, size_t L) {
  std::vector<size_t> w((L + bit_length - 1) / bit_length, 0);
  const uint64_t m = bit_length >= 64 ? ~0ull : ((1ull << bit_length) - 1);
  for (size_t k = 0; k < w.size(); ++k) w[k] = (size_t)((x >> (k * bit_length)) & m);
  return w;
}
inline std::string extension(const std::string& p) {
  const size_t d = p.rfind('.');
  std::string e = d == std::string::npos ? "" : p.substr(d + 1);
  for (auto& ch : e) ch = (char)std::tolower((unsigned char)ch);
  return e;
}
}  // namespace detail

// LoadAlphaDets: .txt (one '0'/'1' string per line, rightmost char = orbital
// 0) or .bin (ceil(L/8) bytes per string, high bit first); sorted ascending
// (highest word first) and deduplicated.
inline void LoadAlphaDets(const std::string& file, std::vector<std::vector<size_t>>& adet, size_t bit_length,
                          size_t L) {
  adet.clear();
  const std::string ext = detail::extension(file);
  if (ext == "txt") {
    std::ifstream in(file);
    if (!in.is_open()) throw std::runtime_error("Failed to open alpha det file.");
    std::string line;
    while (std::getline(in, line)) adet.push_back(from_string(line, bit_length, L));
  } else if (ext == "bin") {
    std::ifstream in(file, std::ios::binary);
    if (!in) throw std::runtime_error("Failed to open file");
    const size_t nbytes = (L + 7) / 8;
    std::vector<uint8_t> buf(nbytes);
    while (in.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)nbytes)) {
      std::vector<size_t> w((L + bit_length - 1) / bit_length, 0);
      size_t idx = 0, pos = 0;
      std::vector<int> bits;
      for (uint8_t byte : buf)
        for (int i = 7; i >= 0; --i, ++idx)
          if (8 * nbytes - L <= idx) bits.push_back((byte >> i) & 1);
      // bits[0] is orbital L-1 (highest), the reversed order gives orbital 0 first
      for (size_t p = 0; p < bits.size(); ++p, ++pos)
        if (bits[bits.size() - 1 - p]) w[pos / bit_length] |= size_t(1) << (pos % bit_length);
      adet.push_back(w);
    }
  }
  std::sort(adet.begin(), adet.end(), detail::words_less);
  adet.erase(std::unique(adet.begin(), adet.end()), adet.end());
}

// ShuffleDet: shuffle all but element 0 with std::mt19937(seed).
inline void ShuffleDet(std::vector<std::vector<size_t>>& det, unsigned int seed) {
  if (det.size() <= 1) return;
  std::mt19937 g(seed);
  std::shuffle(det.begin() + 1, det.end(), g);
}

// ---- wavefunction files ----------------------------------------------------

inline std::string to_padded_string(size_t n, size_t d) {
  std::ostringstream os;
  os << std::setw((int)d) << std::setfill('0') << n;
  return os.str();
}

// One binary file `file + "000000"`: na, nb, det_length (size_t), the alpha
// and beta strings in bit_length-bit words, then W (double, alpha-major).
inline void SaveWavefunction(const std::string& file, const std::vector<std::vector<size_t>>& adet,
                             const std::vector<std::vector<size_t>>& bdet, const std::vector<double>& W) {
  std::ofstream of(file + to_padded_string(0, 6), std::ios::binary);
  if (!of) throw std::runtime_error("SaveWavefunction: cannot open " + file);
  size_t na = adet.size(), nb = bdet.size(), len = adet.empty() ? 0 : adet[0].size();
  of.write(reinterpret_cast<const char*>(&na), sizeof(size_t));
  of.write(reinterpret_cast<const char*>(&nb), sizeof(size_t));
  of.write(reinterpret_cast<const char*>(&len), sizeof(size_t));
  for (const auto& d : adet) of.write(reinterpret_cast<const char*>(d.data()), (std::streamsize)(sizeof(size_t) * len));
  for (const auto& d : bdet) of.write(reinterpret_cast<const char*>(d.data()), (std::streamsize)(sizeof(size_t) * len));
  of.write(reinterpret_cast<const char*>(W.data()), (std::streamsize)(sizeof(double) * W.size()));
}

// Loads a saved wavefunction onto the current basis: every saved (alpha, beta)
// pair whose strings are both present is copied to its new position, the rest
// is dropped, and the result is normalised.
inline void LoadWavefunction(const std::string& file, const std::vector<std::vector<size_t>>& adet,
                             const std::vector<std::vector<size_t>>& bdet, std::vector<double>& W) {
  std::ifstream in(file + to_padded_string(0, 6), std::ios::binary);
  if (!in.is_open()) throw std::runtime_error("failed to open input file " + file + to_padded_string(0, 6));
  const std::string name = file + to_padded_string(0, 6);
  auto need = [&](bool ok, const char* what) {
    if (!ok) throw std::runtime_error("LoadWavefunction: " + name + ": " + what);
  };
  size_t na = 0, nb = 0, len = 0;
  in.read(reinterpret_cast<char*>(&na), sizeof(size_t));
  in.read(reinterpret_cast<char*>(&nb), sizeof(size_t));
  in.read(reinterpret_cast<char*>(&len), sizeof(size_t));
  need((bool)in, "file shorter than its 3-word header");
  // the header must describe exactly the bytes that follow
  in.seekg(0, std::ios::end);
  const std::streamoff total = in.tellg();
  in.seekg((std::streamoff)(3 * sizeof(size_t)), std::ios::beg);
  const long double body = (long double)(na + nb) * len * sizeof(size_t) + (long double)na * nb * sizeof(double);
  need(len >= 1 && len <= 64 && body == (long double)(total - (std::streamoff)(3 * sizeof(size_t))),
       "header (alpha count, beta count, words per string) does not match the file size");
  std::vector<std::vector<size_t>> la(na, std::vector<size_t>(len)), lb(nb, std::vector<size_t>(len));
  for (auto& d : la) in.read(reinterpret_cast<char*>(d.data()), (std::streamsize)(sizeof(size_t) * len));
  for (auto& d : lb) in.read(reinterpret_cast<char*>(d.data()), (std::streamsize)(sizeof(size_t) * len));
  need((bool)in, "short read of the strings");
  std::vector<double> lw(na * nb);
  in.read(reinterpret_cast<char*>(lw.data()), (std::streamsize)(sizeof(double) * lw.size()));
  need((bool)in, "short read of the wavefunction");
  W.assign(adet.size() * bdet.size(), 0.0);
  std::vector<long long> ma(na, -1), mb(nb, -1);
  for (size_t i = 0; i < na; ++i) {
    auto it = std::find(adet.begin(), adet.end(), la[i]);
    if (it != adet.end()) ma[i] = it - adet.begin();
  }
  for (size_t i = 0; i < nb; ++i) {
    auto it = std::find(bdet.begin(), bdet.end(), lb[i]);
    if (it != bdet.end()) mb[i] = it - bdet.begin();
  }
  for (size_t i = 0; i < na; ++i)
    if (ma[i] >= 0)
      for (size_t j = 0; j < nb; ++j)
        if (mb[j] >= 0) W[(size_t)ma[i] * bdet.size() + (size_t)mb[j]] += lw[i * nb + j];
  double s = 0.0;
  for (double x : W) s += x * x;
  if (!(s > 0.0)) throw std::runtime_error("LoadWavefunction: no saved determinant is in the current basis");
  const double f = 1.0 / std::sqrt(s);
  for (double& x : W) x *= f;
}

// Dense alpha x beta dump: .bin = raw doubles, .txt/.dat = one line per
// determinant "value # ia: string ib: string".
inline void SaveMatrixFormWF(const std::string& filename, size_t bit_length, size_t L,
                             const std::vector<std::vector<size_t>>& adet,
                             const std::vector<std::vector<size_t>>& bdet, const std::vector<double>& W) {
  const std::string ext = detail::extension(filename);
  if (ext == "bin") {
    std::ofstream of(filename, std::ios::binary);
    of.write(reinterpret_cast<const char*>(W.data()), (std::streamsize)(sizeof(double) * W.size()));
  } else if (ext == "dat" || ext == "txt") {
    std::ofstream of(filename);
    of.precision(6);
    for (size_t ia = 0; ia < adet.size(); ++ia)
      for (size_t ib = 0; ib < bdet.size(); ++ib)
        of << W[ia * bdet.size() + ib] << " # " << ia << ": " << makestring(adet[ia], bit_length, L) << " " << ib
           << ": " << makestring(bdet[ib], bit_length, L) << "\n";
  }
}

namespace tpb {

struct SBD {
  int task_comm_size = 1;
  int adet_comm_size = 1;
  int bdet_comm_size = 1;
  int h_comm_size = 1;
  int method = 0;
  int max_it = 1;
  int max_nb = 10;
  double eps = 1.0e-4;
  double max_time = 86400.0;
  int init = 0;
  int do_shuffle = 0;
  int do_rdm = 0;
  double ratio = 0.0;
  double threshold = 0.01;
  size_t bit_length = 20;
  std::string dump_matrix_form_wf;
};

inline SBD generate_sbd_data(int argc, char* argv[]) {
  SBD d;
  for (int i = 0; i + 1 < argc; ++i) {
    const std::string a(argv[i]);
    const char* v = argv[i + 1];
    if (a == "--adet_comm_size") { d.adet_comm_size = std::atoi(v); ++i; }
    else if (a == "--bdet_comm_size") { d.bdet_comm_size = std::atoi(v); ++i; }
    else if (a == "--task_comm_size") { d.task_comm_size = std::atoi(v); ++i; }
    else if (a == "--method") { d.method = std::atoi(v); ++i; }
    else if (a == "--iteration") { d.max_it = std::atoi(v); ++i; }
    else if (a == "--block") { d.max_nb = std::atoi(v); ++i; }
    else if (a == "--tolerance") { d.eps = std::atof(v); ++i; }
    else if (a == "--carryover_ratio") { d.ratio = std::atof(v); ++i; }
    else if (a == "--carryover_threshold") { d.threshold = std::atof(v); ++i; }
    else if (a == "--max_time") { d.max_time = std::atof(v); ++i; }
    else if (a == "--shuffle") { d.do_shuffle = std::atoi(v); ++i; }
    else if (a == "--rdm") { d.do_rdm = std::atoi(v); ++i; }
    else if (a == "--bit_length") { d.bit_length = (size_t)std::atoi(v); ++i; }
    else if (a == "--dump_matrix_form_wf") { d.dump_matrix_form_wf = std::string(v); ++i; }
  }
  return d;
}

namespace detail {

struct Ctx {
  sbdx_ctx* h = nullptr;
  explicit Ctx(int device) {
    if (sbdx_ctx_create(&h, device) != SBDX_OK) throw std::runtime_error("sbdx: cannot create a context on the GPU");
  }
  ~Ctx() { sbdx_ctx_destroy(h); }
  void check(int rc) const {
    if (rc != SBDX_OK) throw std::runtime_error(std::string("sbdx: ") + sbdx_last_error(h));
  }
};

inline int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  return v ? std::atoi(v) : dflt;
}

// SetupIntegrals (makeintegrals.h:81-126): NORB/NELEC from the header; lines
// in file order, last one wins; i=j=k=l=0 is I0, k=l=0 is h_ij = h_ji,
// anything else an 8-fold ERI class.
inline void setup_integrals(const FCIDump& fd, int& L, int& N, double& I0, std::vector<double>& h,
                            std::vector<double>& eri) {
  L = 0;
  N = 0;
  for (const auto& kv : fd.header) {
    if (kv.first == "NORB") L = std::atoi(kv.second.c_str());
    if (kv.first == "NELEC") N = std::atoi(kv.second.c_str());
  }
  if (L < 1 || L > 64) throw std::invalid_argument("FCIDUMP: NORB must be in [1, 64] for the GPU path");
  const size_t P = (size_t)L * (L + 1) / 2;
  h.assign((size_t)L * L, 0.0);
  eri.assign(P * (P + 1) / 2, 0.0);
  I0 = 0.0;
  auto pair = [](size_t p, size_t q) { return p > q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p; };
  for (const auto& t : fd.integrals) {
    const double v = std::get<0>(t);
    const int i = std::get<1>(t), j = std::get<2>(t), k = std::get<3>(t), l = std::get<4>(t);
    if (i == 0 && j == 0 && k == 0 && l == 0) {
      I0 = v;
    } else if (k == 0 && l == 0) {
      if (i < 1 || j < 1 || i > L || j > L) throw std::out_of_range("FCIDUMP: one-electron index out of range");
      h[(size_t)(i - 1) * L + (j - 1)] = v;
      h[(size_t)(j - 1) * L + (i - 1)] = v;
    } else {
      if (i < 1 || j < 1 || k < 1 || l < 1 || i > L || j > L || k > L || l > L)
        throw std::out_of_range("FCIDUMP: two-electron index out of range");
      eri[pair(pair(i - 1, j - 1), pair(k - 1, l - 1))] = v;
    }
  }
}

// CarryOverAlphaDet (rdmat.h:60-132) from the alpha-string weights.
inline void carry_over(const std::vector<double>& D, const std::vector<std::vector<size_t>>& adet, double ratio,
                       double threshold, std::vector<std::vector<size_t>>& rdet, double& truncated) {
  std::vector<size_t> idx(D.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](size_t i, size_t j) { return D[i] > D[j]; });
  size_t kept = 0;
  truncated = 0.0;
  if (ratio == 0.0) {
    std::vector<double> S(D.size());
    double s = 0.0;
    for (size_t i = 0; i < D.size(); ++i) { s += D[idx[i]]; S[i] = s; }
    kept = (size_t)(std::upper_bound(S.begin(), S.end(), 1.0 - threshold) - S.begin()) + 1;
    kept = std::min(kept, D.size());
  } else {
    kept = std::min((size_t)(ratio * (double)adet.size()), D.size());
    double s = 0.0;
    for (size_t i = 0; i < kept; ++i) s += D[idx[i]];
    truncated = 1.0 - s;
  }
  rdet.assign(kept, std::vector<size_t>());
  for (size_t k = 0; k < kept; ++k) rdet[k] = adet[idx[k]];
}

}  // namespace detail

// diag, struct path (sbdiag.h:113-477): integrals as given (exact doubles).
template <typename Comm>
void diag(const Comm& /*comm*/, const SBD& sbd_data, const FCIDump& fcidump,
          const std::vector<std::vector<size_t>>& adet, const std::vector<std::vector<size_t>>& bdet,
          const std::string& loadname, const std::string& savename, double& energy, std::vector<double>& density,
          std::vector<std::vector<size_t>>& carryover_bitstrings, std::vector<std::vector<double>>& one_p_rdm,
          std::vector<std::vector<double>>& two_p_rdm) {
  if (sbd_data.adet_comm_size * sbd_data.bdet_comm_size * sbd_data.task_comm_size != 1)
    throw std::invalid_argument("sbd::tpb::diag (GPU): the basis runs at world size 1 on one GPU");
  if (sbd_data.method != 0 && sbd_data.method != 1)
    throw std::invalid_argument("sbd::tpb::diag (GPU): method must be 0 (on-the-fly sigma) or 1 (stored Hamiltonian)");
  if (adet.empty() || bdet.empty()) throw std::invalid_argument("sbd::tpb::diag: empty string set");
  int L = 0, N = 0;
  double I0 = 0.0;
  std::vector<double> h, eri;
  detail::setup_integrals(fcidump, L, N, I0, h, eri);
  const size_t bl = sbd_data.bit_length;
  std::vector<uint64_t> a(adet.size()), b(bdet.size());
  for (size_t i = 0; i < adet.size(); ++i) a[i] = sbd::detail::to_u64(adet[i], bl);
  for (size_t i = 0; i < bdet.size(); ++i) b[i] = sbd::detail::to_u64(bdet[i], bl);

  detail::Ctx ctx(detail::env_int("SBDX_DEVICE", 0));
  ctx.check(sbdx_set_integrals(ctx.h, L, I0, h.data(), eri.data(), eri.size()));
  ctx.check(sbdx_set_strings(ctx.h, a.data(), a.size(), b.data(), b.size()));
  ctx.check(sbdx_build_connectivity(ctx.h));
  if (detail::env_int("SBDX_AUTOTUNE", 0)) ctx.check(sbdx_autotune(ctx.h, nullptr, nullptr));
  if (sbd_data.method == 1) {  // method 1 (sbdiag.h:275-300): store H, then the same Davidson
    const auto t0 = std::chrono::high_resolution_clock::now();
    uint64_t nnz = 0;
    ctx.check(sbdx_build_hamiltonian(ctx.h, &nnz));
    const double sec = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
    std::cout << " Elapsed time for make Hamiltonian " << sec << " (sec) " << std::endl;
  }

  const size_t D = a.size() * b.size();
  std::vector<double> W;
  int init_from_W = 0;
  if (!loadname.empty()) {
    LoadWavefunction(loadname, adet, bdet, W);
    init_from_W = 1;
  }
  const char* prec = std::getenv("SBDX_PRECISION");
  sbdx_davidson_params p{};
  p.max_it = sbd_data.max_it;
  p.max_nb = sbd_data.max_nb;
  p.eps = sbd_data.eps;
  p.max_time = sbd_data.max_time;
  p.precision = (prec && std::string(prec) == "fp32") ? SBDX_FP32 : SBDX_FP64;
  p.defect_every = 0;
  p.verbose = detail::env_int("SBDX_VERBOSE", 1);
  sbdx_davidson_info info{};
  // the converged vector stays on the device: the density, the RDMs and the
  // carry-over weights reduce it there (occupation.h:10-95, rdmat.h:10-58 act
  // on the distributed vector in place); it comes to the host only when a file
  // has to be written
  ctx.check(sbdx_davidson(ctx.h, &p, init_from_W, init_from_W ? W.data() : nullptr, &info));
  const double* dW = nullptr;
  ctx.check(sbdx_wavefunction_device(ctx.h, 0, &dW));
  energy = info.energy;
  std::cout.precision(16);
  std::cout << " Energy = " << energy << std::endl;

  const size_t Lz = (size_t)L;
  if (sbd_data.do_rdm == 0) {
    density.assign(2 * Lz, 0.0);
    ctx.check(sbdx_occupation_device(ctx.h, dW, density.data()));
  } else {
    std::vector<double> one(2 * Lz * Lz), two(4 * Lz * Lz * Lz * Lz);
    ctx.check(sbdx_rdm_device(ctx.h, dW, one.data(), two.data()));
    one_p_rdm.assign(2, std::vector<double>());
    two_p_rdm.assign(4, std::vector<double>());
    for (int s = 0; s < 2; ++s) one_p_rdm[s].assign(one.begin() + s * Lz * Lz, one.begin() + (s + 1) * Lz * Lz);
    const size_t L4 = Lz * Lz * Lz * Lz;
    for (int s = 0; s < 4; ++s) two_p_rdm[s].assign(two.begin() + s * L4, two.begin() + (s + 1) * L4);
    density.assign(2 * Lz, 0.0);
    for (size_t io = 0; io < Lz; ++io) {
      density[2 * io] = one_p_rdm[0][io + Lz * io];
      density[2 * io + 1] = one_p_rdm[1][io + Lz * io];
    }
  }

  std::vector<double> wa(a.size());
  ctx.check(sbdx_alpha_weights_device(ctx.h, dW, wa.data()));
  double truncated = 0.0;
  detail::carry_over(wa, adet, sbd_data.ratio, sbd_data.threshold, carryover_bitstrings, truncated);
  if (sbd_data.ratio != 0.0) std::cout << " truncated weight in carry-over = " << truncated << std::endl;

  if (!savename.empty() || !sbd_data.dump_matrix_form_wf.empty()) {
    W.resize(D);
    ctx.check(sbdx_get_wavefunction(ctx.h, 0, W.data()));
  }
  if (!savename.empty()) SaveWavefunction(savename, adet, bdet, W);
  if (!sbd_data.dump_matrix_form_wf.empty())
    SaveMatrixFormWF(sbd_data.dump_matrix_form_wf, bl, Lz, adet, bdet, W);
}

// diag, file-name path (sbdiag.h:493-586): FCIDUMP through the broadcast text
// round trip, alpha strings from file, beta strings from the shuffle rule.
template <typename Comm>
void diag(const Comm& comm, const SBD& sbd_data, const std::string& fcidumpfile, const std::string& adetfile,
          const std::string& loadname, const std::string& savename, double& energy, std::vector<double>& density,
          std::vector<std::vector<size_t>>& carryover_bitstrings, std::vector<std::vector<double>>& one_p_rdm,
          std::vector<std::vector<double>>& two_p_rdm) {
  FCIDump fcidump = LoadFCIDump(fcidumpfile);
  MpiBcast(fcidump, 0, comm);
  size_t L = 0;
  for (const auto& kv : fcidump.header)
    if (kv.first == "NORB") L = (size_t)std::atoi(kv.second.c_str());
  std::vector<std::vector<size_t>> adet, bdet;
  LoadAlphaDets(adetfile, adet, sbd_data.bit_length, L);
  const auto now = []() {
    return static_cast<unsigned int>(std::chrono::high_resolution_clock::now().time_since_epoch().count());
  };
  switch (sbd_data.do_shuffle) {
    case 1: ShuffleDet(adet, now()); bdet = adet; break;
    case 2: bdet = adet; ShuffleDet(adet, now()); ShuffleDet(bdet, now()); break;
    case 3: ShuffleDet(adet, 42u); bdet = adet; break;
    case 4: bdet = adet; ShuffleDet(adet, 1729u); ShuffleDet(bdet, 137u); break;
    default: bdet = adet; break;
  }
  diag(comm, sbd_data, fcidump, adet, bdet, loadname, savename, energy, density, carryover_bitstrings, one_p_rdm,
       two_p_rdm);
}

}  // namespace tpb
}  // namespace sbd

#endif
