// Test helper: the drop-in header's wavefunction file I/O (sbd/sbd.h,
// SaveWavefunction / LoadWavefunction in the layout of the reference's
// chemistry/tpb/restart.h:20-67, 414-657), driven from the CPU test suite.
//
//   restart_io load <file> <basis> <out>   LoadWavefunction(file) onto the basis,
//                                          W written to <out> as raw doubles
//   restart_io save <file> <basis> <in>    SaveWavefunction(file) of the basis
//                                          with W read from <in>
// <basis>: text "L bit_length na nb" then na alpha and nb beta strings as
// unsigned 64-bit integers (bit p = orbital p). Exit status 1 with the
// exception text on stderr when the header API throws.
#include <cstdint>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "sbd/sbd.h"

namespace {

using Dets = std::vector<std::vector<size_t>>;

void read_basis(const std::string& path, Dets& a, Dets& b) {
  std::ifstream in(path);
  size_t L = 0, bl = 0, na = 0, nb = 0;
  if (!(in >> L >> bl >> na >> nb)) throw std::runtime_error("bad basis file " + path);
  a.clear();
  b.clear();
  for (size_t i = 0; i < na + nb; ++i) {
    uint64_t x = 0;
    if (!(in >> x)) throw std::runtime_error("short basis file " + path);
    (i < na ? a : b).push_back(sbd::detail::from_u64(x, bl, L));
  }
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 5) {
    std::cerr << "usage: restart_io load|save <file> <basis> <vector>\n";
    return 2;
  }
  try {
    const std::string mode = argv[1];
    Dets a, b;
    read_basis(argv[3], a, b);
    std::vector<double> W;
    if (mode == "load") {
      sbd::LoadWavefunction(argv[2], a, b, W);
      std::ofstream out(argv[4], std::ios::binary);
      out.write(reinterpret_cast<const char*>(W.data()), (std::streamsize)(sizeof(double) * W.size()));
    } else if (mode == "save") {
      W.resize(a.size() * b.size());
      std::ifstream in(argv[4], std::ios::binary);
      in.read(reinterpret_cast<char*>(W.data()), (std::streamsize)(sizeof(double) * W.size()));
      if (!in) throw std::runtime_error("short vector file");
      sbd::SaveWavefunction(argv[2], a, b, W);
    } else {
      std::cerr << "unknown mode " << mode << "\n";
      return 2;
    }
  } catch (const std::exception& e) {
    std::cerr << e.what() << "\n";
    return 1;
  }
  return 0;
}
