// sbd_diag: command-line driver of the GPU drop-in, with the flags of the
// reference's sample (samples/selected_basis_diagonalization/main.cc:35-56
// and chemistry/tpb/sbdiag.h:35-96):
//   --fcidump F --adetfile A [--bdetfile B] [--loadname L] [--savename S]
//   [--carryoverfile C] [--iteration N] [--block N] [--tolerance x] [--rdm 0|1]
//   [--carryover_ratio r] [--carryover_threshold t] [--shuffle k] [--bit_length b]
//   [--max_time s] [--dump_matrix_form_wf file]
// Without --bdetfile it calls the file-name overload of sbd::tpb::diag (beta
// strings = alpha strings, FCIDUMP text round trip); with --bdetfile it loads
// both string files and calls the struct overload with the FCIDUMP as parsed.
// Prints the energy, the orbital occupations and the first carry-over strings;
// with --rdm 1 writes 1pRDM.txt / 2pRDM.txt and checks E1 + E2 + I0 against
// the energy, as the sample does (main.cc:166-216).
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "sbd/sbd.h"

int main(int argc, char* argv[]) {
  std::string adetfile("alphadets.txt"), bdetfile, fcidumpfile("fcidump.txt"), loadname, savename, carryoverfile;
  for (int i = 0; i + 1 < argc; ++i) {
    const std::string a(argv[i]);
    if (a == "--adetfile") adetfile = argv[++i];
    else if (a == "--bdetfile") bdetfile = argv[++i];
    else if (a == "--fcidump") fcidumpfile = argv[++i];
    else if (a == "--loadname") loadname = argv[++i];
    else if (a == "--savename") savename = argv[++i];
    else if (a == "--carryoverfile") carryoverfile = argv[++i];
  }
  const auto sbd_data = sbd::tpb::generate_sbd_data(argc, argv);
  const int comm = 0;  // world size 1
  double energy = 0.0;
  std::vector<double> density;
  std::vector<std::vector<size_t>> cobits;
  std::vector<std::vector<double>> one, two;
  sbd::FCIDump fcidump;
  int L = 0;
  try {
    if (bdetfile.empty()) {
      sbd::tpb::diag(comm, sbd_data, fcidumpfile, adetfile, loadname, savename, energy, density, cobits, one, two);
      fcidump = sbd::LoadFCIDump(fcidumpfile);
      sbd::MpiBcast(fcidump, 0, comm);
    } else {
      fcidump = sbd::LoadFCIDump(fcidumpfile);
      for (const auto& kv : fcidump.header)
        if (kv.first == "NORB") L = std::atoi(kv.second.c_str());
      std::vector<std::vector<size_t>> adet, bdet;
      sbd::LoadAlphaDets(adetfile, adet, sbd_data.bit_length, (size_t)L);
      sbd::LoadAlphaDets(bdetfile, bdet, sbd_data.bit_length, (size_t)L);
      sbd::tpb::diag(comm, sbd_data, fcidump, adet, bdet, loadname, savename, energy, density, cobits, one, two);
    }
  } catch (const std::exception& e) {
    std::cerr << "sbd_diag: " << e.what() << std::endl;
    return 1;
  }
  for (const auto& kv : fcidump.header)
    if (kv.first == "NORB") L = std::atoi(kv.second.c_str());
  std::cout.precision(16);
  std::cout << " Sample-based diagonalization: Energy = " << energy << std::endl;
  std::cout << " Sample-based diagonalization: density = ";
  for (size_t i = 0; i < density.size() / 2; ++i) std::cout << (i == 0 ? "[" : ",") << density[2 * i] + density[2 * i + 1];
  std::cout << "]" << std::endl;
  std::cout << " Sample-based diagonalization: carryover bitstrings =";
  for (size_t i = 0; i < cobits.size() && i < 6; ++i) std::cout << " " << sbd::makestring(cobits[i], sbd_data.bit_length, L);
  if (cobits.size() > 6) std::cout << " ... " << sbd::makestring(cobits.back(), sbd_data.bit_length, L);
  std::cout << std::endl;
  if (!carryoverfile.empty()) {
    std::ofstream of(carryoverfile);
    for (const auto& c : cobits) of << sbd::makestring(c, sbd_data.bit_length, L) << "\n";
  }
  if (!one.empty()) {
    int Lr = 0, N = 0;
    double I0 = 0.0;
    std::vector<double> h, eri;
    sbd::tpb::detail::setup_integrals(fcidump, Lr, N, I0, h, eri);
    const size_t Lz = (size_t)L;
    auto pair = [](size_t p, size_t q) { return p > q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p; };
    double e1 = 0.0, e2 = 0.0;
    std::ofstream o1("1pRDM.txt"), o2("2pRDM.txt");
    o1.precision(16);
    o2.precision(16);
    for (size_t io = 0; io < Lz; ++io)
      for (size_t jo = 0; jo < Lz; ++jo) {
        const double g = one[0][io + Lz * jo] + one[1][io + Lz * jo];
        o1 << io << " " << jo << " " << g << "\n";
        e1 += h[io * Lz + jo] * g;
      }
    for (size_t io = 0; io < Lz; ++io)
      for (size_t jo = 0; jo < Lz; ++jo)
        for (size_t ia = 0; ia < Lz; ++ia)
          for (size_t ja = 0; ja < Lz; ++ja) {
            const size_t k = io + Lz * jo + Lz * Lz * (ia + Lz * ja);
            const double G = two[0][k] + two[1][k] + two[2][k] + two[3][k];
            o2 << io << " " << jo << " " << ia << " " << ja << " " << G << "\n";
            e2 += 0.5 * eri[pair(pair(io, ia), pair(jo, ja))] * G;
          }
    std::cout << " One-Body energy = " << e1 << std::endl;
    std::cout << " Two-Body energy = " << e2 << std::endl;
    std::cout << " One-Body + Two-Body energy = " << e1 + e2 << std::endl;
    std::cout << " One-Body + Two-Body energy + I0 = " << e1 + e2 + I0 << std::endl;
  }
  return 0;
}
