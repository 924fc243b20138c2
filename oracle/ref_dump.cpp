// Golden-data dump from the reference's OWN host code (TEST INFRASTRUCTURE).
//
//   oracle/_ref/ref_dump OUT.bin NFIELDS SEED [reference command line: -nx 3 -ny 3 -nz 2 -p 5 [-a] ...]
//
// Compiled against the reference's sources (libs/core, libs/mesh, libs/ogs,
// libs/primitives) with the host-only shims of oracle/ref_shim/ (one-rank MPI,
// host-memory OCCA, LAPACK stand-ins); see oracle/Makefile, target `ref`.  It
// follows the set-up sequence of the reference's BP drivers
// (BP/BP5/bp5Main.cpp:30-57, BP/BP5/src/bp5Setup.cpp:29-52):
// settings from the command line, platform_t, mesh_t (box, connectivity,
// global numbering, physical nodes, geometric factors), the masked ogs of
// mesh_t::MaskedGatherScatterSetup (libs/mesh/meshMaskedGatherScatterSetup.cpp)
// with NFIELDS fields, ogs_t::SetupGlobalToLocalMapping, and
// mesh_t::CubatureSetup (libs/mesh/meshCubatureSetupHex3D.cpp); then it applies
// the reference's host ogs Gather (Add, Trans) and Scatter (NoTrans)
// (libs/ogs/ogsOperator.cpp:61-98,207-239) to vectors drawn with the
// reference's prim::random after prim::seedRNG(SEED).
//
// Output: a sequence of records  u32 name length, name, u8 type ('i' int32,
// 'l' int64, 'd' float64), u64 count, count values (little endian).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mesh.hpp"
#include "ogs.hpp"
#include "ogs/ogsOperator.hpp"
#include "primitives.hpp"

using namespace libp;

namespace libp {
void meshAddSettings(settings_t& settings);
}

namespace {

FILE* g_out = nullptr;

void put(const std::string& name, char type, const void* data, uint64_t count) {
  const uint32_t len = (uint32_t)name.size();
  const size_t bytes = type == 'i' ? 4 : 8;
  std::fwrite(&len, 4, 1, g_out);
  std::fwrite(name.data(), 1, len, g_out);
  std::fwrite(&type, 1, 1, g_out);
  std::fwrite(&count, 8, 1, g_out);
  if (count) std::fwrite(data, bytes, count, g_out);
}
void put(const std::string& name, const memory<int>& m) { put(name, 'i', m.ptr(), m.length()); }
void put(const std::string& name, const memory<long long int>& m) { put(name, 'l', m.ptr(), m.length()); }
void put(const std::string& name, const memory<double>& m) { put(name, 'd', m.ptr(), m.length()); }
void put_int(const std::string& name, long long v) { put(name, 'l', &v, 1); }

// The gather operators are protected members of ogs_t; a derived view reads them.
struct OgsView : public ogs::ogs_t {
  explicit OgsView(const ogs::ogs_t& o) : ogs::ogs_t(o) {}
  const ogs::ogsOperator_t& local() const { return *gatherLocal; }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s OUT.bin NFIELDS SEED [reference options]\n", argv[0]);
    return 2;
  }
  const std::string out = argv[1];
  const int Nfields = std::atoi(argv[2]);
  const uint64_t seed = std::strtoull(argv[3], nullptr, 10);
  // the reference's own command line, after argv[0]
  std::vector<char*> args{argv[0]};
  for (int i = 4; i < argc; ++i) args.push_back(argv[i]);
  int rargc = (int)args.size();
  char** rargv = args.data();

  comm_t::Init(rargc, rargv);
  int rc = 0;
  try {
    comm_t comm(comm_t::world().Dup());
    settings_t settings(comm);
    platformAddSettings(settings);
    meshAddSettings(settings);
    settings.newSetting("-v", "--verbose", "VERBOSE", "FALSE", "Enable verbose output", {"TRUE", "FALSE"});
    settings.parseSettings(rargc, rargv);

    platform_t platform(settings);
    mesh_t mesh(platform, settings, comm);

    ogs::InitializeKernels(platform, ogs::Dfloat, ogs::Add);
    ogs::ogs_t ogs = mesh.MaskedGatherScatterSetup(Nfields);
    memory<dlong> GlobalToLocal(mesh.Nelements * mesh.Np * Nfields);
    ogs.SetupGlobalToLocalMapping(GlobalToLocal);
    mesh.CubatureSetup();

    g_out = std::fopen(out.c_str(), "wb");
    if (!g_out) {
      std::fprintf(stderr, "cannot write %s\n", out.c_str());
      return 1;
    }
    put_int("N", mesh.N);
    put_int("Nq", mesh.Nq);
    put_int("Np", mesh.Np);
    put_int("Nelements", mesh.Nelements);
    put_int("Nfields", Nfields);
    put_int("Ngather", ogs.Ngather);
    put_int("NgatherGlobal", ogs.NgatherGlobal);
    put_int("cubNq", mesh.cubNq);
    put("EToV", mesh.EToV);
    put("EX", mesh.EX);
    put("EY", mesh.EY);
    put("EZ", mesh.EZ);
    put("globalIds", mesh.globalIds);
    put("GlobalToLocal", GlobalToLocal);
    OgsView view(ogs);
    put("rowStartsT", view.local().rowStartsT);
    put("colIdsT", view.local().colIdsT);
    put("rowStartsN", view.local().rowStartsN);
    put("colIdsN", view.local().colIdsN);
    put("gllz", mesh.gllz);
    put("gllw", mesh.gllw);
    put("D", mesh.D);
    put("MM", mesh.MM);
    if (mesh.S.length()) put("S", mesh.S);   // Tri2D: Srr, Srs, Sss
    put("x", mesh.x);
    put("y", mesh.y);
    put("z", mesh.z);
    put("wJ", mesh.wJ);
    put("ggeo", mesh.ggeo);
    put("cubr", mesh.cubr);
    put("cubw", mesh.cubw);
    put("cubInterp", mesh.cubInterp);
    put("cubD", mesh.cubD);
    if (mesh.invV.length()) put("invV", mesh.invV);
    if (!settings.compareSetting("AFFINE MESH", "TRUE")) {
      put("cubwJ", mesh.cubwJ);
      put("cubggeo", mesh.cubggeo);
    }

    // the reference's host gather (Add, Trans) of a seeded E-vector and host
    // scatter (NoTrans) of a seeded gathered vector
    const dlong NL = mesh.Nelements * mesh.Np * Nfields;
    memory<double> v(NL), gv(ogs.Ngather), sv(NL), g(ogs.Ngather);
    prim::seedRNG(seed);
    prim::random(NL, v);
    for (dlong n = 0; n < NL; ++n) v[n] = 2.0 * v[n] - 1.0;
    ogs.Gather(gv, v, 1, ogs::Add, ogs::Trans);
    prim::seedRNG(seed + 1);
    prim::random(ogs.Ngather, g);
    for (dlong n = 0; n < ogs.Ngather; ++n) g[n] = 2.0 * g[n] - 1.0;
    for (dlong n = 0; n < NL; ++n) sv[n] = 0.0;
    ogs.Scatter(sv, g, 1, ogs::NoTrans);
    put("gather_in", v);
    put("gather_out", gv);
    put("scatter_in", g);
    put("scatter_out", sv);
    std::fclose(g_out);
  } catch (std::exception& e) {
    std::fprintf(stderr, "reference set-up failed: %s\n", e.what());
    rc = 1;
  }
  comm_t::Finalize();
  return rc;
}
