// BK1-BK6 / BP1-BP6 drivers behind bp_driver_main(): the reference
// executables' command-line keys, settings semantics and result lines, running
// on the C ABI.
//
// Settings semantics follow libs/core/settings.cpp:
//   * every setting has a short key, long key, name, default, description and
//     an optional list of allowed values (updateVal rejects anything else);
//   * "-v"/"--verbose" and "-a"/"--affine" take no value;
//   * a setting given twice on the command line is an error;
//   * compareSetting is a substring test; "-h"/"--help" prints the usage.
// Keys come from libs/core/platformSettings.cpp:31-50,
// libs/mesh/meshSettings.cpp:31-62 and BP/BP5/src/bp5Settings.cpp:30-46.
// Keys marked "extension" select the modes the reference does not have.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/bp_b200.h"

namespace {

struct Setting {
  std::string shortkey, longkey, name, val, description;
  std::vector<std::string> options;
  bool set_on_cmdline = false;
};

class Settings {
 public:
  void add(const std::string& sk, const std::string& lk, const std::string& name, const std::string& val,
           const std::string& desc, const std::vector<std::string>& options = {}) {
    for (auto& it : map_)
      if (it.second.shortkey == sk || it.second.longkey == lk)
        throw std::runtime_error("Setting with key: [" + sk + "] already exists.");
    if (map_.count(name)) throw std::runtime_error("Setting with name: [" + name + "] already exists.");
    map_[name] = Setting{sk, lk, name, val, desc, options, false};
    order_.push_back(name);
  }
  void change(const std::string& name, const std::string& v) {
    auto it = map_.find(name);
    if (it == map_.end()) throw std::runtime_error("Setting with name: [" + name + "] does not exist.");
    Setting& s = it->second;
    if (!s.options.empty()) {
      bool ok = false;
      for (auto& o : s.options) ok = ok || (o == v);
      if (!ok) {
        std::ostringstream ss;
        ss << "Value: \"" << v << "\" not valid for setting " << name << "\nPossible values are: { ";
        for (size_t i = 0; i < s.options.size(); ++i) ss << s.options[i] << (i + 1 < s.options.size() ? ", " : " }");
        throw std::runtime_error(ss.str());
      }
    }
    s.val = v;
  }
  // returns false when -h was given (usage printed)
  bool parse(int argc, char** argv) {
    for (int i = 1; i < argc;) {
      if (!std::strcmp(argv[i], "-h") || !std::strcmp(argv[i], "--help")) {
        usage();
        return false;
      }
      bool matched = false;
      for (auto& it : map_) {
        Setting& s = it.second;
        if (s.shortkey != argv[i] && s.longkey != argv[i]) continue;
        matched = true;
        if (s.set_on_cmdline)
          throw std::runtime_error("Cannot set setting [" + s.name + "] twice in run command.");
        if (!std::strcmp(argv[i], "-v") || !std::strcmp(argv[i], "--verbose")) {
          change("VERBOSE", "TRUE");
          i += 1;
        } else if (!std::strcmp(argv[i], "-a") || !std::strcmp(argv[i], "--affine")) {
          change("AFFINE MESH", "TRUE");
          i += 1;
        } else {
          if (i + 1 >= argc) throw std::runtime_error(std::string("Missing value for option ") + argv[i]);
          change(s.name, argv[i + 1]);
          i += 2;
        }
        s.set_on_cmdline = true;
        break;
      }
      if (!matched) throw std::runtime_error(std::string("Unknown option ") + argv[i] + " (see -h)");
    }
    return true;
  }
  std::string get(const std::string& name) const {
    auto it = map_.find(name);
    if (it == map_.end()) throw std::runtime_error("Unable to find setting: [" + name + "]");
    return it->second.val;
  }
  bool compare(const std::string& name, const std::string& token) const {
    return get(name).find(token) != std::string::npos;
  }
  void usage() const {
    std::cout << "Usage:\n\n";
    for (auto& n : order_) {
      const Setting& s = map_.at(n);
      std::cout << "Name:     [" << s.name << "]\n";
      std::cout << "CL keys:  [" << s.shortkey << ", " << s.longkey << "]\n";
      if (!s.description.empty()) std::cout << "Description: " << s.description << "\n";
      if (!s.options.empty()) {
        std::cout << "Possible values: { ";
        for (size_t i = 0; i < s.options.size(); ++i) std::cout << s.options[i] << (i + 1 < s.options.size() ? ", " : " }");
        std::cout << "\n";
      }
      std::cout << "\n";
    }
    std::cout << "Name:     [HELP]\nCL keys:  [-h, --help]\nDescription: Print this help message\n";
  }
  void report() const {
    std::cout << "Settings:\n\n";
    for (auto& n : order_) {
      const Setting& s = map_.at(n);
      std::cout << "Name:     [" << s.name << "]\nCL keys:  [" << s.shortkey << ", " << s.longkey << "]\nValue:    "
                << s.val << "\n\n";
    }
  }

 private:
  std::map<std::string, Setting> map_;
  std::vector<std::string> order_;
};

void add_common(Settings& S, bool bp) {
  // platform (libs/core/platformSettings.cpp:31-50)
  S.add("-m", "--mode", "THREAD MODEL", "CUDA", "OCCA's Parallel execution platform",
        {"Serial", "OpenMP", "CUDA", "HIP", "OpenCL"});
  S.add("-pl", "--platform", "PLATFORM NUMBER", "0", "Parallel platform number (used in OpenCL mode)");
  S.add("-d", "--device", "DEVICE NUMBER", "0", "Parallel device number");
  // mesh (libs/mesh/meshSettings.cpp:31-62)
  S.add("-e", "--elements", "ELEMENT TYPE", "Hex", "Type of mesh elements", {"Tri", "Quad", "Tet", "Hex"});
  S.add("-nx", "--dimx", "BOX NX", "10", "Number of elements in X-dimension per rank");
  S.add("-ny", "--dimy", "BOX NY", "10", "Number of elements in Y-dimension per rank");
  S.add("-nz", "--dimz", "BOX NZ", "10", "Number of elements in Z-dimension per rank");
  S.add("-p", "--degree", "POLYNOMIAL DEGREE", "4", "Degree of polynomial finite element space",
        {"1", "2", "3", "4", "5", "6", "7", "8", "9", "10", "11", "12", "13", "14", "15"});
  S.add("-a", "--affine", "AFFINE MESH", "FALSE", "Assume elements are affine images of reference element",
        {"TRUE", "FALSE"});
  if (bp) S.add("-o", "--output", "OUTPUT FILE NAME", "", "Write the solution to <name>_0000.vtu");
  S.add("-v", "--verbose", "VERBOSE", "FALSE", "Enable verbose output", {"TRUE", "FALSE"});
  // extensions
  S.add("-pc", "--precon", "PRECONDITIONER", "NONE", "CG preconditioner (extension)", {"NONE", "JACOBI"});
  S.add("-fp", "--precision", "PRECISION", "FP64",
        "FP64, or MIXED: FP32 CG with FP64 reliable updates, needs -tol (extension)", {"FP64", "MIXED"});
  S.add("-f", "--forcing", "FORCING", "ANALYTIC",
        "Right-hand side: analytic sin forcing, or f=2u-1 per gathered node from the seeded LCG (extension)",
        {"ANALYTIC", "RANDOM"});
  S.add("-s", "--seed", "FORCING SEED", "0", "LCG seed of the RANDOM forcing (extension)");
  S.add("-pt", "--perturb", "VERTEX PERTURBATION", "0", "Interior vertex perturbation, fraction of h (extension)");
  S.add("-ps", "--perturb-seed", "PERTURBATION SEED", "1", "LCG seed of the vertex perturbation (extension)");
  if (!bp)
    S.add("-nr", "--rhs", "RIGHT-HAND SIDES", "1",
          "With -fp MIXED: apply the FP32 operator to 1, 2 or 4 interleaved right-hand sides at once (extension)",
          {"1", "2", "4"});
  if (bp) {
    S.add("-nr", "--rhs", "RIGHT-HAND SIDES", "1",
          "Solve this many RANDOM right-hand sides (seeds s, s+1, ...) together with the batched solver (extension)");
    S.add("-it", "--iterations", "CG ITERATIONS", "100", "Maximum CG iterations of the timed solve (extension)");
    S.add("-wi", "--warmup-iterations", "WARMUP ITERATIONS", "1000", "CG iterations of the warmup solve (extension)");
    S.add("-tol", "--tolerance", "CG TOLERANCE", "0", "CG stop tolerance of the timed solve (extension)");
  }
}

void check(int rc) {
  if (rc != BP_SUCCESS) throw std::runtime_error(bp_last_error());
}

double now_after_finish() {
  check(bp_finish(nullptr));
  return std::chrono::duration<double>(std::chrono::high_resolution_clock::now().time_since_epoch()).count();
}

struct Problem {
  bp_mesh_t mesh = nullptr;
  bp_solver_t solver = nullptr;
  bp_mesh_view_t view{};
  bp_cubature_view_t cub{};   // BP1-BP4
  ~Problem() {
    if (solver) bp_solver_destroy(solver);
    if (mesh) bp_mesh_destroy(mesh);
  }
};

void setup(const Settings& S, Problem& P, int Nfields, int bp) {
  if (!S.compare("THREAD MODEL", "CUDA"))
    throw std::runtime_error("THREAD MODEL " + S.get("THREAD MODEL") +
                             " is not available: this build runs the CUDA (sm_100a) path only");
  const bool tri = S.compare("ELEMENT TYPE", "Tri");
  const bool tet = S.compare("ELEMENT TYPE", "Tet");
  const bool quad = S.compare("ELEMENT TYPE", "Quad");
  if (quad && bp <= 4)
    throw std::runtime_error("ELEMENT TYPE Quad is available for BK5/BK6 and BP5/BP6 (BP1-BP4: Hex only)");
  if ((tri || tet) && (bp != 5 || !S.compare("AFFINE MESH", "TRUE")))
    throw std::runtime_error("ELEMENT TYPE " + S.get("ELEMENT TYPE") + " is available for BK5 and BP5 with -a");
  check(bp_platform_init(std::atoi(S.get("DEVICE NUMBER").c_str())));
  bp_box_desc_t d{};
  d.dim = quad || tri ? 2 : 3;
  d.simplex = tri || tet ? 1 : 0;
  d.nx = std::atoi(S.get("BOX NX").c_str());
  d.ny = std::atoi(S.get("BOX NY").c_str());
  d.nz = quad || tri ? 1 : std::atoi(S.get("BOX NZ").c_str());
  d.N = std::atoi(S.get("POLYNOMIAL DEGREE").c_str());
  d.affine = S.compare("AFFINE MESH", "TRUE") ? 1 : 0;
  d.Nfields = quad && Nfields > 1 ? 2 : Nfields;   // BP6 has Nfields = dim
  d.pert = std::atof(S.get("VERTEX PERTURBATION").c_str());
  d.pert_seed = std::strtoull(S.get("PERTURBATION SEED").c_str(), nullptr, 10);
  check(bp_mesh_create(&d, &P.mesh));
  check(bp_mesh_view(P.mesh, &P.view));
  bp_solver_desc_t sd{};
  sd.bp = bp;
  sd.lambda = 1.0;   // BP/BP5/bp5Main.cpp:47
  sd.precon = S.compare("PRECONDITIONER", "JACOBI") ? BP_PRECON_JACOBI : BP_PRECON_NONE;
  sd.precision = S.compare("PRECISION", "MIXED") ? BP_PRECISION_MIXED : BP_PRECISION_FP64;
  check(bp_solver_create(P.mesh, &sd, &P.solver));
  if (bp <= 4) check(bp_mesh_cubature_view(P.mesh, &P.cub));
}

struct DevVec {
  double* p = nullptr;
  explicit DevVec(size_t n) { check(bp_malloc(reinterpret_cast<void**>(&p), n * sizeof(double))); }
  ~DevVec() { bp_free(p); }
};
struct DevVec32 {
  float* p = nullptr;
  explicit DevVec32(size_t n) {
    if (n) check(bp_malloc(reinterpret_cast<void**>(&p), n * sizeof(float)));
  }
  ~DevVec32() {
    if (p) bp_free(p);
  }
};

// reference byte model for one Ax application: BP5/BP6 bp5Run.cpp:106-142,
// bk5Run.cpp:97-125; BP3/BP4 bp3Run.cpp:107-122; BP1/BP2 bp1Run.cpp and
// bk1Run.cpp (one factor per point, J or JW).  sv: bytes per value (8 as the
// reference; 4 for the FP32 operator of the mixed-precision solver).
double ax_bytes(int bp, const bp_mesh_view_t& v, long long Ndofs, double sv = 8.0) {
  const double E = v.Nelements, Np = v.Np, Nf = v.Nfields;
  const double cNq = v.N + 2, cNp = cNq * cNq * cNq;
  const double per_point = bp <= 2 ? 1.0 : (v.dim == 2 ? 4.0 : 7.0);   // J, or ggeo + wJ (mesh.dim==3 ? 7 : 4)
  const double points = v.affine ? 1.0 : (bp <= 4 ? cNp : Np);
  return Ndofs * sv + (points * per_point * sv + 4.0 + Np * Nf * 4.0 + Np * Nf * sv) * E;
}
// reference flop model for one Ax application (the same files, Hex branches)
double ax_flops(int bp, const bp_mesh_view_t& v) {
  const double Nq = v.Nq, E = v.Nelements, Nf = v.Nfields;
  if (v.simplex)   // affine TRIANGLES and TETRAHEDRA branches of bp5Run.cpp:145-155
    return (v.dim == 2 ? 8.0 * v.Np * v.Np + 8.0 * v.Np : 14.0 * v.Np * v.Np + 14.0 * v.Np) * Nf * E;
  if (v.dim == 2)   // QUADRILATERALS branches of bp5Run.cpp:144-187
    return (v.affine ? 8 * Nq * Nq * Nq + 12 * Nq * Nq : 8 * Nq * Nq * Nq + 8 * Nq * Nq) * Nf * E;
  const double cNq = v.N + 2, Nq3 = Nq * Nq * Nq, cNq3 = cNq * cNq * cNq;
  const double interp = 4 * cNq * Nq3 + 4 * cNq * cNq * Nq * Nq + 4 * cNq3 * Nq;
  double f;
  if (bp <= 2) f = v.affine ? 6 * Nq * Nq3 + Nq3 : interp + cNq3;
  else if (bp <= 4) f = v.affine ? 24 * Nq * Nq3 + 17 * Nq3 : interp + 12 * cNq * cNq3 + 17 * cNq3;
  else f = v.affine ? 12 * Nq * Nq3 + 21 * Nq3 : 12 * Nq * Nq3 + 18 * Nq3;
  return f * Nf * E;
}

// CG model bytes and flops of one system (bpNRun.cpp: first iteration + Niter iterations)
void cg_model(int bp, const bp_mesh_view_t& v, long long Ndofs, int Niter, double& Nbytes, double& Nflops) {
  const double NGlobal = (double)v.Nlocal;
  const double NbytesAx = ax_bytes(bp, v, Ndofs);
  const double NbytesGather = (Ndofs + 1) * 4.0 + NGlobal * 4.0 + NGlobal * 8.0 + Ndofs * 8.0;
  Nbytes = (4 * Ndofs * 8.0 + NbytesAx + NbytesGather) + (11 * Ndofs * 8.0 + NbytesAx + NbytesGather) * Niter;
  const double NflopsAx = ax_flops(bp, v);
  Nflops = (5.0 * Ndofs + NflopsAx + NGlobal) + (11.0 * Ndofs + NflopsAx + NGlobal) * Niter;
}

// -nr K: K right-hand sides of the same problem solved together by the batched
// solver (packed lanes in a mixed-precision BP5 solve); the result line counts
// every system's unknowns x iterations
int run_bp_batch(const char* name, int bp, Settings& S, int nr) {
  if (bp % 2 == 0) throw std::runtime_error("-nr is available for BP1, BP3 and BP5");
  if (!S.compare("ELEMENT TYPE", "Hex")) throw std::runtime_error("-nr is available for Hex meshes");
  if (!S.compare("FORCING", "RANDOM")) throw std::runtime_error("-nr needs -f RANDOM");
  if (!S.compare("THREAD MODEL", "CUDA"))
    throw std::runtime_error("THREAD MODEL " + S.get("THREAD MODEL") +
                             " is not available: this build runs the CUDA (sm_100a) path only");
  check(bp_platform_init(std::atoi(S.get("DEVICE NUMBER").c_str())));
  bp_batch_problem_t pr{};
  pr.nx = std::atoi(S.get("BOX NX").c_str());
  pr.ny = std::atoi(S.get("BOX NY").c_str());
  pr.nz = std::atoi(S.get("BOX NZ").c_str());
  pr.N = std::atoi(S.get("POLYNOMIAL DEGREE").c_str());
  pr.pert = std::atof(S.get("VERTEX PERTURBATION").c_str());
  pr.pert_seed = std::strtoull(S.get("PERTURBATION SEED").c_str(), nullptr, 10);
  pr.nrhs = nr;
  pr.rhs_seed = std::strtoull(S.get("FORCING SEED").c_str(), nullptr, 10);
  pr.affine = S.compare("AFFINE MESH", "TRUE") ? 1 : 0;
  bp_solver_desc_t sd{};
  sd.bp = bp;
  sd.lambda = 1.0;
  sd.precon = S.compare("PRECONDITIONER", "JACOBI") ? BP_PRECON_JACOBI : BP_PRECON_NONE;
  sd.precision = S.compare("PRECISION", "MIXED") ? BP_PRECISION_MIXED : BP_PRECISION_FP64;
  bp_batch_t B = nullptr;
  check(bp_batch_create(&pr, 1, &sd, &B));
  struct Guard {
    bp_batch_t b;
    ~Guard() { bp_batch_destroy(b); }
  } guard{B};
  const int maxIter = std::atoi(S.get("CG ITERATIONS").c_str());
  const double tol = std::atof(S.get("CG TOLERANCE").c_str());
  std::vector<bp_solve_stats_t> st(nr);
  double ms = 0.0;
  check(bp_batch_solve(B, tol, maxIter, st.data(), &ms));   // warmup (graph capture)
  const double t0 = now_after_finish();
  check(bp_batch_solve(B, tol, maxIter, st.data(), &ms));
  const double t1 = now_after_finish();
  const double elapsed = t1 - t0;
  int32_t Nd = 0;
  check(bp_batch_system_info(B, 0, nullptr, &Nd));
  // the sizes the byte/flop model needs
  bp_mesh_view_t v{};
  v.N = pr.N; v.Nq = pr.N + 1; v.Np = v.Nq * v.Nq * v.Nq; v.Nelements = pr.nx * pr.ny * pr.nz; v.Nfields = 1;
  v.affine = pr.affine; v.Ngather = Nd; v.Nlocal = (int64_t)v.Nelements * v.Np;
  double Nbytes = 0, Nflops = 0, dofit = 0;
  int itmax = 0;
  for (int k = 0; k < nr; ++k) {
    double nb, nf;
    cg_model(bp, v, Nd, st[k].iterations, nb, nf);
    Nbytes += nb;
    Nflops += nf;
    dofit += (double)Nd * st[k].iterations;
    itmax = std::max(itmax, (int)st[k].iterations);
  }
  std::printf(
      "%s: N=%2d, DOFs=%lld, elapsed=%4.4f, iterations=%d, time per DOF=%1.2e, avg BW (GB/s)=%6.1f, avg GFLOPs=%6.1f, "
      "DOFs*iterations/ranks*time=%1.2e, %s \n",
      name, pr.N, (long long)Nd, elapsed, itmax, elapsed / ((double)Nd * nr), Nbytes / (1.0e9 * elapsed),
      Nflops / (1.0e9 * elapsed), dofit / elapsed, pr.affine ? "Element=Hex, Affine" : "Element=Hex");
  std::printf("%s extra: right-hand sides=%d solved together, precision=%s, precon=%s, iterations per system:", name,
              nr, S.get("PRECISION").c_str(), S.get("PRECONDITIONER").c_str());
  for (int k = 0; k < nr; ++k) std::printf(" %d", st[k].iterations);
  std::printf(", relative residuals:");
  for (int k = 0; k < nr; ++k) std::printf(" %.3e", std::sqrt(st[k].rdotr / (st[k].rdotr0 > 0 ? st[k].rdotr0 : 1.0)));
  std::printf(", device ms=%.4f\n", ms);
  std::fflush(stdout);
  return BP_SUCCESS;
}

int run_bp(const char* name, int bp, Settings& S) {
  const int nr = std::atoi(S.get("RIGHT-HAND SIDES").c_str());
  if (nr < 1 || nr > 64) throw std::runtime_error("-nr must be 1..64");
  if (nr > 1) return run_bp_batch(name, bp, S, nr);
  const int Nfields = (bp == 6 || bp == 4 || bp == 2) ? 3 : 1;
  Problem P;
  setup(S, P, Nfields, bp);
  if (S.compare("VERBOSE", "TRUE")) S.report();
  const int32_t N = P.view.Ngather;
  DevVec x(N), r(N), b(N);
  const bool random = S.compare("FORCING", "RANDOM");
  const uint64_t seed = std::strtoull(S.get("FORCING SEED").c_str(), nullptr, 10);
  check(bp_solver_rhs(P.solver, random ? BP_RHS_RANDOM : BP_RHS_ANALYTIC, seed, b.p, nullptr));
  const int maxIter = std::atoi(S.get("CG ITERATIONS").c_str());
  const int warmIter = std::atoi(S.get("WARMUP ITERATIONS").c_str());
  const double tol = std::atof(S.get("CG TOLERANCE").c_str());
  const int verbose = S.compare("VERBOSE", "TRUE") ? 1 : 0;
  bp_solve_stats_t st{};
  // warmup solve (bp5Run.cpp:66-69)
  check(bp_linalg_set(N, 0.0, x.p, nullptr));
  check(bp_memcpy_dtod(r.p, b.p, sizeof(double) * N, nullptr));
  const bool mixed = S.compare("PRECISION", "MIXED");
  check(bp_solver_solve(P.solver, x.p, r.p, mixed ? 1e-30 : 0.0, warmIter, nullptr, nullptr, &st));
  // timed solve (bp5Run.cpp:71-95)
  check(bp_linalg_set(N, 0.0, x.p, nullptr));
  check(bp_memcpy_dtod(r.p, b.p, sizeof(double) * N, nullptr));
  std::vector<double> hr(maxIter > 0 ? maxIter : 1), ha(maxIter > 0 ? maxIter : 1);
  const double t0 = now_after_finish();
  check(bp_solver_solve(P.solver, x.p, r.p, tol, maxIter, hr.data(), ha.data(), &st));
  const double t1 = now_after_finish();
  const double elapsed = t1 - t0;
  const int Niter = st.iterations;
  if (verbose) {
    std::printf("CG: initial res norm %12.12f \n", std::sqrt(st.rdotr0));
    for (int k = 0; k < Niter; ++k) std::printf("CG: it %d, r norm %12.12le, alpha = %le \n", k + 1, hr[k], ha[k]);
  }
  const long long Ndofs = N;
  const double NGlobal = (double)P.view.Nlocal;
  const double NbytesAx = ax_bytes(bp, P.view, Ndofs);
  const double NbytesGather = (Ndofs + 1) * 4.0 + NGlobal * 4.0 + NGlobal * 8.0 + Ndofs * 8.0;
  const double Nbytes = (4 * Ndofs * 8.0 + NbytesAx + NbytesGather) + (11 * Ndofs * 8.0 + NbytesAx + NbytesGather) * Niter;
  const double NflopsAx = ax_flops(bp, P.view);
  const double Nflops = (5.0 * Ndofs + NflopsAx + NGlobal) + (11.0 * Ndofs + NflopsAx + NGlobal) * Niter;
  std::string suffix = P.view.simplex ? (P.view.dim == 2 ? "Element=Tri" : "Element=Tet")
                                       : P.view.dim == 2 ? "Element=Quad" : "Element=Hex";
  if (P.view.affine) suffix += ", Affine";
  std::printf(
      "%s: N=%2d, DOFs=%lld, elapsed=%4.4f, iterations=%d, time per DOF=%1.2e, avg BW (GB/s)=%6.1f, avg GFLOPs=%6.1f, "
      "DOFs*iterations/ranks*time=%1.2e, %s \n",
      name, P.view.N, Ndofs, elapsed, Niter, elapsed / Ndofs, Nbytes / (1.0e9 * elapsed), Nflops / (1.0e9 * elapsed),
      Ndofs * ((double)Niter / (1 * elapsed)), suffix.c_str());
  const double rel = std::sqrt(st.rdotr / (st.rdotr0 > 0 ? st.rdotr0 : 1.0));
  std::printf("%s extra: precision=%s, precon=%s, forcing=%s, final r norm=%.6e, relative residual=%.6e, "
              "reliable updates=%d, device ms=%.4f\n",
              name, S.get("PRECISION").c_str(), S.get("PRECONDITIONER").c_str(), S.get("FORCING").c_str(),
              std::sqrt(st.rdotr), rel, st.updates, st.elapsed_ms);
  std::fflush(stdout);
  // "-o name": the solution scattered to the local nodes, name_0000.vtu (bp5Run.cpp:220-238)
  const std::string out = S.get("OUTPUT FILE NAME");
  if (!out.empty()) {
    const size_t NL = (size_t)P.view.Nlocal;
    DevVec xL(NL);
    check(bp_memset(xL.p, 0, sizeof(double) * NL, nullptr));
    check(bp_ogs_scatter(N, P.view.rowStarts, P.view.colIds, x.p, xL.p, nullptr));
    std::vector<double> h(NL);
    check(bp_memcpy_dtoh(h.data(), xL.p, sizeof(double) * NL, nullptr));
    check(bp_finish(nullptr));
    char fname[4096];
    std::snprintf(fname, sizeof(fname), "%s_%04d.vtu", out.c_str(), 0);
    check(bp_mesh_write_vtu(P.mesh, h.data(), fname));
  }
  return BP_SUCCESS;
}

int run_bk(const char* name, int bk, Settings& S) {
  const int Nfields = (bk == 6 || bk == 4 || bk == 2) ? 3 : 1;
  Problem P;
  setup(S, P, Nfields, bk);
  if (S.compare("VERBOSE", "TRUE")) S.report();
  const int32_t Ngather = P.view.Ngather;
  DevVec q(Ngather), Aq((size_t)P.view.Nlocal);
  const bool random = S.compare("FORCING", "RANDOM");
  const uint64_t seed = std::strtoull(S.get("FORCING SEED").c_str(), nullptr, 10);
  if (random) {
    // BK input q = 2u-1 per gathered node (the forcing's f)
    DevVec b(Ngather);
    check(bp_solver_rhs(P.solver, BP_RHS_RANDOM, seed, b.p, q.p));
  } else {
    // gathered analytic forcing (bk5Run.cpp:38-50)
    check(bp_solver_rhs(P.solver, BP_RHS_ANALYTIC, 0, q.p, nullptr));
  }
  bp_ax_desc_t d{};
  d.bp = bk;
  d.N = P.view.N;
  d.affine = P.view.affine;
  d.Nfields = P.view.Nfields;
  d.dim = P.view.dim;
  // -fp MIXED times the FP32 operator of the mixed-precision solver (BK5/BK6)
  const bool fp32 = S.compare("PRECISION", "MIXED");
  if (fp32 && P.view.simplex) throw std::runtime_error("BK5 -e Tri/Tet times the FP64 operator only");
  const size_t ng = P.view.affine ? (size_t)P.view.Nelements : (size_t)P.view.Nelements * P.view.Np;
  const int nr = std::atoi(S.get("RIGHT-HAND SIDES").c_str());
  if (nr > 1 && (!fp32 || bk != 5)) throw std::runtime_error("-nr is available for BK5 with -fp MIXED");
  const size_t nggeo = P.view.dim == 2 ? 3 : 6;
  if (nr > 1 && P.view.dim == 2) throw std::runtime_error("-nr is available for Hex meshes");
  DevVec32 wJ32(fp32 ? ng : 0), ggeo32(fp32 ? nggeo * ng : 0), gllw32(fp32 ? P.view.Nq : 0),
      D32(fp32 ? (size_t)P.view.Nq * P.view.Nq : 0), q32(fp32 ? (size_t)Ngather * nr : 0),
      Aq32(fp32 ? (size_t)P.view.Nlocal * nr : 0);
  if (fp32) {
    check(bp_convert_f64_f32(ng, P.view.wJ, wJ32.p, nullptr));
    check(bp_convert_f64_f32(nggeo * ng, P.view.ggeo, ggeo32.p, nullptr));
    check(bp_convert_f64_f32(P.view.Nq, P.view.gllw, gllw32.p, nullptr));
    check(bp_convert_f64_f32((size_t)P.view.Nq * P.view.Nq, P.view.D, D32.p, nullptr));
    // every right-hand side gets the same input (the timing does not depend on the values)
    DevVec32 q1(Ngather);
    check(bp_convert_f64_f32(Ngather, q.p, q1.p, nullptr));
    for (int k = 0; k < nr; ++k)
      check(bp_memcpy_dtod(q32.p + (size_t)Ngather * k, q1.p, sizeof(float) * Ngather, nullptr));
    if (nr > 1) {   // interleave: q32[row*nr + k]
      std::vector<float> h((size_t)Ngather * nr), t((size_t)Ngather * nr);
      check(bp_memcpy_dtoh(h.data(), q32.p, sizeof(float) * h.size(), nullptr));
      check(bp_finish(nullptr));
      for (int k = 0; k < nr; ++k)
        for (int32_t r = 0; r < Ngather; ++r) t[(size_t)r * nr + k] = h[(size_t)k * Ngather + r];
      check(bp_memcpy_htod(q32.p, t.data(), sizeof(float) * t.size(), nullptr));
      check(bp_finish(nullptr));
    }
  }
  // BK1-BK4 in FP32: FP32 copies of the cubature operands
  const bool cub32 = fp32 && bk <= 4;
  const size_t nc = !cub32 ? 0 : P.view.affine ? (size_t)P.view.Nelements : (size_t)P.view.Nelements * P.cub.cubNp;
  const size_t Nq2 = (size_t)P.view.Nq * P.view.Nq, nD = P.view.affine ? Nq2 : (size_t)P.cub.cubNq * P.cub.cubNq;
  const size_t nI = (size_t)P.cub.cubNq * P.view.Nq;
  DevVec32 cwJ(nc), cgeo(6 * nc), cD(cub32 ? nD : 0), cI(cub32 ? nI : 0), cV(cub32 ? Nq2 : 0), cM(cub32 ? Nq2 : 0);
  if (cub32) {
    check(bp_convert_f64_f32(nc, P.cub.cubwJ, cwJ.p, nullptr));
    check(bp_convert_f64_f32(6 * nc, P.cub.cubggeo, cgeo.p, nullptr));
    check(bp_convert_f64_f32(nD, P.cub.cubD, cD.p, nullptr));
    check(bp_convert_f64_f32(nI, P.cub.cubInterp, cI.p, nullptr));
    check(bp_convert_f64_f32(Nq2, P.cub.invV, cV.p, nullptr));
    check(bp_convert_f64_f32(Nq2, P.cub.MM, cM.p, nullptr));
  }
  auto apply = [&]() {
    if (cub32)
      check(bp_ax_cub_hex3d_f32(&d, P.view.Nelements, P.view.elementList, P.view.GlobalToLocal, cwJ.p, cgeo.p, cD.p,
                                cI.p, cV.p, cM.p, 1.0f, q32.p, Aq32.p, nullptr));
    else if (fp32)
      check(bp_ax_hex3d_f32_multi(&d, nr, P.view.Nelements, P.view.elementList, P.view.GlobalToLocal, wJ32.p,
                                  ggeo32.p, gllw32.p, D32.p, 1.0f, q32.p, Aq32.p, nullptr));
    else if (P.view.simplex && P.view.dim == 3)
      check(bp_ax_tet3d(&d, P.view.Nelements, P.view.elementList, P.view.GlobalToLocal, P.view.wJ, P.view.ggeo,
                        P.view.S, P.view.MM, 1.0, q.p, Aq.p, nullptr));
    else if (P.view.simplex)
      check(bp_ax_tri2d(&d, P.view.Nelements, P.view.elementList, P.view.GlobalToLocal, P.view.wJ, P.view.ggeo,
                        P.view.S, P.view.MM, 1.0, q.p, Aq.p, nullptr));
    else if (bk >= 5)
      check(bp_ax_hex3d(&d, P.view.Nelements, P.view.elementList, P.view.GlobalToLocal, P.view.wJ, P.view.ggeo,
                        P.view.gllw, P.view.D, 1.0, q.p, Aq.p, nullptr));
    else
      check(bp_ax_cub_hex3d(&d, P.view.Nelements, P.view.elementList, P.view.GlobalToLocal, P.cub.cubwJ,
                            P.cub.cubggeo, P.cub.cubD, P.cub.cubInterp, P.cub.invV, P.cub.MM, 1.0, q.p, Aq.p,
                            nullptr));
  };
  for (int n = 0; n < 5; ++n) apply();
  const int Ntests = 50;
  const double t0 = now_after_finish();
  for (int n = 0; n < Ntests; ++n) apply();
  const double t1 = now_after_finish();
  const double elapsed = (t1 - t0) / Ntests;
  const long long Ndofs = Ngather;
  // per apply: the model's bytes with 4-byte values, the q/Aq terms once per right-hand side
  double Nbytes = ax_bytes(bk, P.view, Ndofs, fp32 ? 4.0 : 8.0);
  if (nr > 1) Nbytes += (nr - 1) * (Ndofs * 4.0 + (double)P.view.Nlocal * 4.0);
  const double Nflops = ax_flops(bk, P.view) * nr;
  std::string suffix = P.view.simplex ? (P.view.dim == 2 ? "Element=Tri" : "Element=Tet")
                                       : P.view.dim == 2 ? "Element=Quad" : "Element=Hex";
  if (P.view.affine) suffix += ", Affine";
  std::printf(
      "%s: N=%2d, DOFs=%lld, elapsed=%4.4f, time per DOF=%1.2e, avg BW (GB/s)=%6.1f, avg GFLOPs=%6.1f, "
      "DOFs/ranks*time=%1.2e, %s \n",
      name, P.view.N, Ndofs, elapsed, elapsed / Ndofs, Nbytes / (1.0e9 * elapsed), Nflops / (1.0e9 * elapsed),
      Ndofs * (double)nr / (1 * elapsed), suffix.c_str());
  std::fflush(stdout);
  return BP_SUCCESS;
}

}  // namespace

extern "C" int bp_driver_main(const char* name, int argc, char** argv) {
  try {
    std::string n = name ? name : "";
    const bool bp = n.size() == 3 && n[0] == 'B' && n[1] == 'P';
    const bool bk = n.size() == 3 && n[0] == 'B' && n[1] == 'K';
    const int which = (bp || bk) ? n[2] - '0' : 0;
    if (!(bp || bk) || which < 1 || which > 6)
      throw std::runtime_error("bp_driver_main: available drivers are BP1-BP6 and BK1-BK6");
    Settings S;
    add_common(S, bp);
    if (!S.parse(argc, argv)) return BP_SUCCESS;
    return bp ? run_bp(n.c_str(), which, S) : run_bk(n.c_str(), which, S);
  } catch (const std::exception& e) {
    std::string banner = "---[ Error ]";
    std::fprintf(stderr, "\n%s%s\n    Message  : %s\n%s\n", banner.c_str(), std::string(80 - banner.size(), '-').c_str(),
                 e.what(), std::string(80, '=').c_str());
    return BP_ERROR;
  }
}
