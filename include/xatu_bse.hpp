/*
 * xatu_bse.hpp -- C++ host API of the B200 BSE engine, header-only, over the C ABI of xatu_bse.h.
 *
 * It mirrors the part of Xatu's C++ interface that drives the exciton hot path, with the same class and
 * method names and argument meanings, on standard-library types instead of Armadillo:
 *
 *   xatu::SystemConfiguration(file)            src/SystemConfiguration.cpp:20-258 (.model reader),
 *                                              src/ConfigurationBase.cpp:43-150 (block format)
 *   xatu::ExcitonTB(config, ncell, nbands, nrmbands, {eps_m, eps_s, r0}, Q)
 *                                              include/xatu/ExcitonTB.hpp:72-73, src/ExcitonTB.cpp:128-150
 *   brillouinZoneMesh(n)                       src/Lattice.cpp:140-162
 *   initializeHamiltonian()                    include/xatu/ExcitonTB.hpp:140, src/ExcitonTB.cpp:794-815
 *   BShamiltonian()                            include/xatu/ExcitonTB.hpp:141, src/ExcitonTB.cpp:822-921
 *   diagonalize(method, nstates)               include/xatu/ExcitonTB.hpp:143, src/ExcitonTB.cpp:930-972
 *   setExchange, setMode, setReciprocalVectors, setGauge, selectPotential, selectExchangePotential,
 *   setScissor, setCutoff, setRegularization, setQ
 *                                              src/ExcitonTB.cpp:227-300, src/Exciton.tpp:16-117
 *
 * Errors follow the reference's convention: std::invalid_argument for bad input (the engine's status
 * message as text), std::runtime_error for device failures.  Every computation runs on the GPU through
 * libxatu_bse.so; this header holds host arrays and fills the ABI's descriptors.
 */
#ifndef XATU_BSE_HPP
#define XATU_BSE_HPP

#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "xatu_bse.h"

namespace xatu {

using cplx = std::complex<double>;

// ------------------------------------------------------------------ .model reader
struct SystemInfo {
  int ndim = 0;
  int filling = 0;
  std::vector<std::array<double, 3>> bravaisLattice;
  std::vector<std::array<double, 4>> motif;              // x, y, z, species
  std::vector<int> norbitals;                            // per species
  std::vector<std::array<double, 3>> bravaisVectors;     // cells of H(R)
  std::vector<std::vector<cplx>> hamiltonian;            // per cell, row-major norb x norb
  std::vector<std::vector<cplx>> overlap;                // empty, or like hamiltonian
  int norb = 0;
};

class SystemConfiguration {
 public:
  SystemInfo systemInfo;

  explicit SystemConfiguration(const std::string& file) {
    if (file.empty()) throw std::invalid_argument("ConfigurationBase: file must not be empty");
    read_blocks(file);
    parse();
    for (const char* a : {"dimension", "bravaislattice", "motif", "norbitals", "filling", "bravaisvectors",
                          "hamiltonian"})
      if (std::find(found_.begin(), found_.end(), a) == found_.end())
        throw std::invalid_argument(std::string("Missing arguments in config. file: missing ") + a);
    check();
  }

 private:
  std::vector<std::string> found_;
  std::map<std::string, std::vector<std::string>> contents_;

  static std::string key_of(const std::string& line) {   // ConfigurationBase::parseArgument
    std::string k;
    for (char c : line.substr(line.find('#') + 1))
      if (!std::isspace(static_cast<unsigned char>(c))) k += static_cast<char>(std::tolower(c));
    return k;
  }

  void read_blocks(const std::string& file) {   // ConfigurationBase::extractArguments / extractRawContent
    std::ifstream in(file);
    if (!in) throw std::invalid_argument("ConfigurationBase: file does not exist: " + file);
    std::vector<std::string> lines;
    for (std::string l; std::getline(in, l);) lines.push_back(l);
    std::string arg;
    std::vector<std::string> content;
    for (size_t i = 0; i < lines.size(); i++) {
      const std::string& line = lines[i];
      if (line.find('#') != std::string::npos) {
        if (i + 1 != lines.size()) found_.push_back(key_of(line));   // keys on the last line are not recorded
        if (!content.empty()) {
          contents_[arg] = content;
          content.clear();
        }
        arg = key_of(line);
      } else if (line.empty() || line.find('!') != std::string::npos) {
        continue;
      } else {
        std::string s = line;
        std::replace(s.begin(), s.end(), ',', ' ');
        std::replace(s.begin(), s.end(), ';', ' ');
        content.push_back(s);
      }
    }
    contents_[arg] = content;
  }

  static std::vector<std::string> tokens(const std::string& line) {
    std::istringstream is(line);
    std::vector<std::string> t;
    for (std::string w; is >> w;) t.push_back(w);
    return t;
  }

  // istream >> double on a token: the longest numeric prefix ("+0.5j" -> 0.5)
  static double number(const std::string& tok) {
    char* end = nullptr;
    const double v = std::strtod(tok.c_str(), &end);
    if (end == tok.c_str()) throw std::invalid_argument("cannot parse number from '" + tok + "'");
    return v;
  }

  static std::vector<double> numbers(const std::string& line) {
    std::vector<double> v;
    for (const auto& t : tokens(line)) v.push_back(number(t));
    return v;
  }

  template <size_t D>
  static std::vector<std::array<double, D>> rows(const std::vector<std::string>& content, const char* what) {
    std::vector<std::array<double, D>> out;
    for (const auto& line : content) {
      const auto v = numbers(line);
      if (v.size() < D) throw std::invalid_argument(what);
      std::array<double, D> r{};
      for (size_t j = 0; j < D; j++) r[j] = v[j];
      out.push_back(r);
    }
    return out;
  }

  // SystemConfiguration::parseMatrices (SystemConfiguration.cpp:159-228): matrices separated by '&' lines
  static std::vector<std::vector<cplx>> matrices(const std::vector<std::string>& content, int* dim) {
    const std::string& first = content.at(0);
    const bool is_complex = first.find('i') != std::string::npos || first.find('j') != std::string::npos;
    int n = 0;
    for (const auto& line : content) {
      if (line.find('&') != std::string::npos) break;
      n++;
    }
    std::vector<std::vector<cplx>> mats;
    std::vector<cplx> m((size_t)n * n);
    int r = 0;
    for (const auto& line : content) {
      if (line.find('&') != std::string::npos) {
        mats.push_back(m);
        std::fill(m.begin(), m.end(), cplx(0, 0));
        r = 0;
        continue;
      }
      const auto t = tokens(line);
      int j = 0;
      for (size_t q = 0; q < t.size() && j < n; q++, j++) {
        const double re = number(t[q]);
        double im = 0;
        if (is_complex && ++q < t.size()) im = number(t[q]);
        m[(size_t)r * n + j] = cplx(re, im);
      }
      r++;
    }
    *dim = n;
    return mats;
  }

  void parse() {
    SystemInfo& s = systemInfo;
    for (const auto& arg : found_) {
      const auto& c = contents_[arg];
      if (arg == "dimension") {
        if (c.size() != 1) throw std::invalid_argument("Expected only one line for 'Dimension'");
        s.ndim = (int)number(tokens(c[0]).at(0));
      } else if (arg == "bravaislattice") {
        s.bravaisLattice = rows<3>(c, "Bravais vectors must have three components");
      } else if (arg == "motif") {
        s.motif = rows<4>(c, "Motif must be of shape (x,y,z,'species')");
      } else if (arg == "norbitals") {
        if (c.size() != 1) throw std::invalid_argument("Error: Orbital information must be one line only");
        for (double v : numbers(c[0])) s.norbitals.push_back((int)v);
      } else if (arg == "filling") {
        if (c.size() != 1) throw std::invalid_argument("Expected only one line in 'filling' field");
        const double f = number(tokens(c[0]).at(0));
        if (f != std::floor(f)) throw std::invalid_argument("Filling must be a positive integer.");
        s.filling = (int)f;
      } else if (arg == "bravaisvectors") {
        s.bravaisVectors = rows<3>(c, "Bravais vectors must have three components");
      } else if (arg == "hamiltonian") {
        s.hamiltonian = matrices(c, &s.norb);
      } else if (arg == "overlap") {
        int n = 0;
        s.overlap = matrices(c, &n);
      }
    }
  }

  void check() const {   // SystemConfiguration::checkContentCoherence (SystemConfiguration.cpp:235-258)
    const SystemInfo& s = systemInfo;
    if (s.ndim != (int)s.bravaisLattice.size())
      throw std::invalid_argument("Error: Dimensions must match number of Bravais basis");
    if (s.hamiltonian.size() != s.bravaisVectors.size())
      throw std::invalid_argument("Error: Number of H matrices must match number of Bravais vectors");
    if (!s.overlap.empty() && s.overlap.size() != s.hamiltonian.size())
      throw std::invalid_argument("Error: Number of overlap matrices must match number of H matrices");
    std::set<int> species;
    for (const auto& m : s.motif) species.insert((int)m[3]);
    if (species.size() != s.norbitals.size())
      throw std::invalid_argument(
          "Error: Number of different species must match be consistent in motif and orbitals");
  }
};

// ------------------------------------------------------------------ results
struct Result {
  std::vector<double> eigval;   // ascending; all N for "diag", nstates otherwise
  std::vector<cplx> eigvec;     // N x nstates, column-major (column s = state s), the reference's layout
  int64_t dim = 0;
  int nstates = 0;
  cplx coefficient(int64_t row, int state) const { return eigvec[(size_t)state * dim + row]; }
};

// ------------------------------------------------------------------ exciton
class ExcitonTB {
 public:
  ExcitonTB(const SystemConfiguration& config, int ncell = 20, int nbands = 1, int nrmbands = 0,
            std::array<double, 3> parameters = {1, 5, 1}, std::array<double, 3> Q = {0, 0, 0}, int device = 0)
      : info_(config.systemInfo), ncell_(ncell), Q_(Q) {
    eps_m_ = parameters[0];
    eps_s_ = parameters[1];
    r0_ = parameters[2];
    if (r0_ == 0) throw std::invalid_argument("Error: r0 must be non-zero");
    cutoff_ = ncell / 2.5;
    int basisdim = 0;
    for (const auto& m : info_.motif) basisdim += info_.norbitals.at((size_t)m[3]);
    if (2 * nbands > basisdim)
      throw std::invalid_argument("Error: Number of bands cannot be higher than actual material bands");
    const int fl = info_.filling - 1;
    for (int b = fl - nbands - nrmbands + 1; b <= fl - nrmbands; b++) valence_.push_back(b);
    for (int b = fl + 1 + nrmbands; b <= fl + nbands + nrmbands; b++) conduction_.push_back(b);
    status(xatu_ctx_create(&ctx_, device), "xatu_ctx_create");
  }
  ExcitonTB(const ExcitonTB&) = delete;
  ExcitonTB& operator=(const ExcitonTB&) = delete;
  ~ExcitonTB() {
    if (ctx_) xatu_ctx_destroy(ctx_);
  }

  // setters with the reference's checks
  void setExchange(bool on) { exchange_ = on; }
  void setMode(const std::string& mode) {
    if (mode != "realspace" && mode != "reciprocalspace")
      throw std::invalid_argument("setMode(): mode must be either realspace or reciprocalspace");
    mode_ = mode;
  }
  void setReciprocalVectors(int n) {
    if (n < 0) throw std::invalid_argument("setReciprocalVectors(): given number must be positive");
    nReciprocalVectors_ = n;
  }
  void setGauge(const std::string& gauge) {
    if (gauge != "lattice" && gauge != "atomic")
      throw std::invalid_argument("setGauge(): gauge must be either lattice or atomic");
    gauge_ = gauge;
  }
  void selectPotential(const std::string& p) { potential_ = potential_kind(p); }
  void selectExchangePotential(const std::string& p) { exchangePotential_ = potential_kind(p); }
  void setScissor(double s) { scissor_ = s; }
  void setCutoff(double c) {
    if (c > 0) cutoff_ = c;
  }
  void setRegularization(double r) { regularization_ = r; }
  void setQ(std::array<double, 3> Q) { Q_ = Q; }

  // Lattice::brillouinZoneMesh
  void brillouinZoneMesh(int n) {
    std::vector<double> brav = flat(info_.bravaisLattice), recip((size_t)info_.ndim * 3);
    status(xatu_reciprocal_lattice(info_.ndim, brav.data(), recip.data()), "xatu_reciprocal_lattice");
    size_t nk = 1;
    for (int d = 0; d < info_.ndim; d++) nk *= (size_t)n;
    kpoints_.assign(nk * 3, 0.0);
    status(xatu_mesh_mp(info_.ndim, recip.data(), n, kpoints_.data()), "xatu_mesh_mp");
  }

  // ExcitonTB::initializeHamiltonian: system and parameters to the device, band solve, interaction tables
  void initializeHamiltonian() {
    if (valence_.empty() && conduction_.empty()) throw std::invalid_argument("Error: Exciton object must have some bands");
    if (kpoints_.empty()) throw std::invalid_argument("Error: BZ mesh must be initialized first");
    const double a = std::sqrt(info_.bravaisLattice[0][0] * info_.bravaisLattice[0][0] +
                               info_.bravaisLattice[0][1] * info_.bravaisLattice[0][1] +
                               info_.bravaisLattice[0][2] * info_.bravaisLattice[0][2]);
    if (regularization_ < 1e-10) regularization_ = a;
    std::vector<double> brav = flat(info_.bravaisLattice), motif = flat(info_.motif),
                        cells = flat(info_.bravaisVectors);
    std::vector<cplx> ham, ovl;
    for (const auto& m : info_.hamiltonian) ham.insert(ham.end(), m.begin(), m.end());
    for (const auto& m : info_.overlap) ovl.insert(ovl.end(), m.begin(), m.end());
    xatu_system_desc sd{info_.ndim, brav.data(), (int)info_.motif.size(), motif.data(), (int)info_.norbitals.size(),
                        info_.norbitals.data(), (int)info_.bravaisVectors.size(), cells.data(),
                        reinterpret_cast<const double*>(ham.data()),
                        ovl.empty() ? nullptr : reinterpret_cast<const double*>(ovl.data()), info_.filling, -1, 0};
    check(xatu_system_upload(ctx_, &sd));
    xatu_exciton_desc ed{};
    ed.ncell = ncell_;
    ed.factor = 1;
    ed.nk = (int)(kpoints_.size() / 3);
    ed.kpoints = kpoints_.data();
    ed.nmesh = ed.nk;
    ed.mesh = kpoints_.data();
    ed.nvalence = (int)valence_.size();
    ed.nconduction = (int)conduction_.size();
    ed.valence_bands = valence_.data();
    ed.conduction_bands = conduction_.data();
    ed.eps_m = eps_m_;
    ed.eps_s = eps_s_;
    ed.r0 = r0_;
    ed.regularization = regularization_;
    ed.cutoff = cutoff_;
    for (int i = 0; i < 3; i++) ed.Q[i] = Q_[i];
    ed.scissor = scissor_;
    ed.exchange = exchange_ ? 1 : 0;
    ed.mode = mode_ == "realspace" ? XATU_MODE_REALSPACE : XATU_MODE_RECIPROCAL;
    ed.n_reciprocal = nReciprocalVectors_;
    ed.potential = potential_;
    ed.exchange_potential = exchangePotential_;
    ed.gauge = gauge_ == "lattice" ? XATU_GAUGE_LATTICE : XATU_GAUGE_ATOMIC;
    check(xatu_exciton_set(ctx_, &ed));
    check(xatu_bands_compute(ctx_));
    check(xatu_interaction_build(ctx_));
  }

  // ExcitonTB::BShamiltonian: XATU_PREC_FP64 (the reference's complex128 HBS_) or XATU_PREC_MIXED
  void BShamiltonian(int precision = XATU_PREC_FP64) { check(xatu_bse_build(ctx_, precision)); }

  // ExcitonTB::diagonalize: "diag" -> all eigenvalues (FP64 dense), "davidson" / "sparse" -> lowest nstates
  Result diagonalize(const std::string& method = "diag", int nstates = 8) {
    Result r;
    check(xatu_bse_dim(ctx_, &r.dim));
    int solver;
    if (method == "diag") {
      solver = XATU_SOLVER_DENSE_FP64;
      r.eigval.assign((size_t)r.dim, 0.0);
    } else if (method == "davidson" || method == "sparse") {
      solver = XATU_SOLVER_DAVIDSON;
      r.eigval.assign((size_t)nstates, 0.0);
    } else {
      throw std::invalid_argument("Method for diagonalization must be either diag, davidson or sparse");
    }
    r.nstates = nstates;
    r.eigvec.assign((size_t)r.dim * nstates, cplx(0, 0));
    check(xatu_bse_solve(ctx_, solver, nstates, r.eigval.data(), reinterpret_cast<double*>(r.eigvec.data())));
    return r;
  }

  int64_t excitonbasisdim() const {
    return (int64_t)(kpoints_.size() / 3) * (int64_t)valence_.size() * (int64_t)conduction_.size();
  }
  xatu_ctx* context() const { return ctx_; }

 private:
  static int potential_kind(const std::string& p) {
    if (p == "keldysh") return XATU_POT_KELDYSH;
    if (p == "coulomb") return XATU_POT_COULOMB;
    throw std::invalid_argument("Potential must be either keldysh or coulomb");
  }
  template <size_t D>
  static std::vector<double> flat(const std::vector<std::array<double, D>>& rows) {
    std::vector<double> v;
    for (const auto& r : rows) v.insert(v.end(), r.begin(), r.end());
    return v;
  }
  static void status(xatu_status st, const char* what) {
    if (st != XATU_OK) throw std::runtime_error(std::string(what) + " failed with status " + std::to_string(st));
  }
  void check(xatu_status st) const {
    if (st == XATU_OK) return;
    const std::string msg = xatu_last_error(ctx_) ? xatu_last_error(ctx_) : "engine error";
    if (st == XATU_ERR_INVALID || st == XATU_ERR_STATE || st == XATU_ERR_UNSUPPORTED) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
  }

  SystemInfo info_;
  xatu_ctx* ctx_ = nullptr;
  int ncell_;
  std::array<double, 3> Q_;
  double eps_m_ = 1, eps_s_ = 5, r0_ = 1, regularization_ = 0, cutoff_ = 0, scissor_ = 0;
  bool exchange_ = false;
  std::string mode_ = "realspace", gauge_ = "lattice";
  int nReciprocalVectors_ = 1;
  int potential_ = XATU_POT_KELDYSH, exchangePotential_ = XATU_POT_KELDYSH;
  std::vector<int> valence_, conduction_;
  std::vector<double> kpoints_;
};

}  // namespace xatu

#endif /* XATU_BSE_HPP */
