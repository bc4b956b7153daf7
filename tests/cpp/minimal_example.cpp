// A C++ caller of the engine through include/xatu_bse.hpp (the header-only host API over the C ABI), in
// the shape of the reference's main/minimal_example.cpp:13-19: read a .model file, build the exciton,
// mesh, initializeHamiltonian, BShamiltonian, diagonalize.
//
//   minimal_example <model> <ncell> <nbands> <eps_m> <eps_s> <r0> <Qx> <Qy> <Qz> <exchange 0|1>
//                   <precision fp64|mixed> <method diag|davidson> <nstates>
//
// Prints "dim N" and then one line per state, "E <index> <energy in eV>".
//
//   minimal_example parse <model>
//
// only reads the model and prints what the reader found (no device needed).
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>

#include "xatu_bse.hpp"

int main(int argc, char** argv) {
  if (argc == 3 && std::string(argv[1]) == "parse") {
    try {
      const xatu::SystemConfiguration config(argv[2]);
      const xatu::SystemInfo& s = config.systemInfo;
      double habs = 0;
      for (const auto& m : s.hamiltonian)
        for (const auto& z : m) habs += std::abs(z);
      std::printf("ndim %d natoms %zu species %zu norb %d ncells %zu filling %d sum|H| %.10f overlap %zu\n", s.ndim,
                  s.motif.size(), s.norbitals.size(), s.norb, s.hamiltonian.size(), s.filling, habs, s.overlap.size());
      return 0;
    } catch (const std::exception& e) {
      std::fprintf(stderr, "error: %s\n", e.what());
      return 1;
    }
  }
  if (argc != 14) {
    std::fprintf(stderr, "usage: %s model ncell nbands eps_m eps_s r0 Qx Qy Qz exchange precision method nstates\n",
                 argv[0]);
    return 2;
  }
  try {
    const int ncell = std::atoi(argv[2]), nbands = std::atoi(argv[3]);
    const std::array<double, 3> params = {std::atof(argv[4]), std::atof(argv[5]), std::atof(argv[6])};
    const std::array<double, 3> Q = {std::atof(argv[7]), std::atof(argv[8]), std::atof(argv[9])};
    const bool exchange = std::atoi(argv[10]) != 0;
    const std::string precision = argv[11], method = argv[12];
    const int nstates = std::atoi(argv[13]);

    xatu::SystemConfiguration config(argv[1]);
    xatu::ExcitonTB exciton(config, ncell, nbands, 0, params, Q);
    exciton.setExchange(exchange);
    exciton.brillouinZoneMesh(ncell);
    exciton.initializeHamiltonian();
    exciton.BShamiltonian(precision == "mixed" ? XATU_PREC_MIXED : XATU_PREC_FP64);
    xatu::Result r = exciton.diagonalize(method, nstates);
    std::printf("dim %lld\n", (long long)r.dim);
    for (int s = 0; s < nstates; s++) std::printf("E %d %.12f\n", s, r.eigval[s]);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
