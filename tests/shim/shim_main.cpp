// A reference-style caller written against include/segpu.hpp, the C++ shim
// with the reference's class names. Built and run by tests/test_shim.py.
//
//   shim_main cpu   options parsing and a Mesh (host tables), then a Field,
//                   which must fail loudly without a CUDA device (no CPU
//                   fallback)
//   shim_main gpu <fields>   (lap - 1) u = f on an 8x8, p=6 doubly periodic
//                   mesh through Mesh, BCs, Field, Advector and
//                   HelmholtzEqn, with the tracer and the velocity read from
//                   <fields> (raw doubles: nVertsTotal tracer values, then
//                   nVertsTotal velocity pairs); prints the iteration count
//                   and the solution values
#include <cstdio>
#include <cstring>

#include "segpu.hpp"

static int cpu_case() {
  se_solver_opts o = se_options("helm_", "-helm_ksp_rtol 1e-9 -helm_ksp_max_it 77 -helm_pc_type fdm");
  std::printf("version %s\n", se_version());
  std::printf("opts rtol %.3g max_it %d method %d\n", o.rtol, o.max_it, o.method);
  int nEls[2] = {4, 4};
  double lo[2] = {0.0, 0.0}, hi[2] = {1.0, 1.0};
  bool per[2] = {true, true};
  Mesh m("m", nEls, "legendre", 6, lo, hi, per);  // host tables only
  std::printf("mesh %d vertices\n", m.nVertsTotal);
  try {
    Field f("f", &m, 1, nullptr);  // device memory
    std::printf("field created\n");
  } catch (const std::runtime_error& e) {
    std::printf("field refused: %s\n", e.what());
  }
  return 0;
}

static int gpu_case(const char* fields) {
  int nEls[2] = {8, 8};
  double lo[2] = {0.0, 0.0}, hi[2] = {1.0, 1.0};
  bool per[2] = {true, true};
  Mesh m("m", nEls, "legendre", 6, lo, hi, per);
  BCs bcs(false, false, false, false, &m);
  Field phi("phi", &m, 1, &bcs), vel("vel", &m, 2, nullptr), u("u", &m, 1, &bcs);
  std::FILE* fp = std::fopen(fields, "rb");
  if (!fp) return 2;
  const size_t nv = (size_t)m.nVertsTotal;
  const bool got = std::fread(phi.host.data(), sizeof(double), nv, fp) == nv &&
                   std::fread(vel.host.data(), sizeof(double), 2 * nv, fp) == 2 * nv;
  std::fclose(fp);
  if (!got) return 3;
  phi.Upload();
  vel.Upload();
  Advector adv(&phi, &vel);
  adv.Advect(0.01);
  se_ok(se_field_copy(phi.h, adv.fieldSL));
  HelmholtzEqn helm(&u, &phi, -1.0, -1.0, 1.0, 0);
  helm.Assemble();
  helm.Solve("helm_", false, "-helm_ksp_rtol 1e-10");
  u.Download();
  std::printf("its %d reason %d\n", helm.last().its, helm.last().reason);
  for (int i = 0; i < m.nVertsTotal; i++) std::printf("%.17g\n", u.vals[i][0]);
  return 0;
}

int main(int argc, char** argv) {
  if (argc > 2 && std::strcmp(argv[1], "gpu") == 0) return gpu_case(argv[2]);
  return cpu_case();
}
