// Test driver of the MatShell binding (include/dendro_b200_matshell.hpp),
// compiled against the project's single-rank PETSc stand-ins
// (oracle/ref_build/shim) -- test infrastructure.  It builds a mesh through
// the C ABI, wraps the operator in a MatShell the way CreateJacobian2 /
// CreateElasticityMat do (examples/src/backend/omgNeumann.C:643-745,
// elasticityJac.C), and drives it through PETSc's MatMult and
// MatGetDiagonal:
//
//   matshell_driver lapmass <octs.u32> <maxDepth> <x.f64> <coef.f64|none> <y.f64> <d.f64>
//   matshell_driver elastic <octs.u32> <maxDepth> <x.f64> <mu> <lambda> <y.f64> <d.f64>
//   matshell_driver transfer <octs.u32> <maxDepth> <nlevels> <level> <xf.f64> <xc.f64> <out>
//
// The transfer mode builds the hierarchy, wraps R from `level` to level + 1
// in a MatShell as DAMGSetUp does (src/omg/omg.C:2278-2283) and writes
// MatMult (R xf), MatMultTranspose (P xc), MatMultAdd (1 + R xf) and
// MatMultTransposeAdd (1 + P xc) to <out>.R / .P / .RA / .PA.
//
// Octant files hold 4 x uint32 per octant (x, y, z, level).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "petsc.h"
#include "petscmat.h"
#include "petscvec.h"
#include "dendro_b200_matshell.hpp"

namespace {

template <class T>
std::vector<T> read_raw(const char* path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  const size_t n = size_t(f.tellg()) / sizeof(T);
  std::vector<T> v(n);
  f.seekg(0);
  f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(T)));
  return v;
}
void write_raw(const char* path, const double* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), std::streamsize(n * sizeof(double)));
}
int fail(const char* where, dg_status st) {
  char msg[512];
  dg_last_error(msg, sizeof msg);
  std::fprintf(stderr, "%s: %s (%s)\n", where, dg_status_string(st), msg);
  return 1;
}

}  // namespace

int run_transfer(int argc, char** argv) {
  if (argc < 9) return 2;
  PetscInitialize(&argc, &argv, nullptr, nullptr);
  std::vector<uint32_t> raw = read_raw<uint32_t>(argv[2]);
  const uint32_t depth = uint32_t(std::atoi(argv[3]));
  const int nlevels = std::atoi(argv[4]), level = std::atoi(argv[5]);
  std::vector<dg_octant> octs(raw.size() / 4);
  for (size_t i = 0; i < octs.size(); ++i)
    octs[i] = dg_octant{raw[4 * i], raw[4 * i + 1], raw[4 * i + 2], raw[4 * i + 3]};
  dg_octree* tree = nullptr;
  dg_damg* m = nullptr;
  dg_status st = dg_octree_from_octants(octs.data(), int64_t(octs.size()), 0, depth, &tree);
  if (st) return fail("octree", st);
  dg_damg_config cfg;
  dg_damg_default_config(&cfg);
  cfg.nlevels = nlevels;
  if ((st = dg_damg_create(tree, &cfg, &m))) return fail("damg", st);
  Mat R;
  if (dendro_b200::DgCreateRestrictionShell(PETSC_COMM_WORLD, m, level, 1, &R)) return 1;
  const std::vector<double> xf = read_raw<double>(argv[6]), xc = read_raw<double>(argv[7]);
  Vec vf, vc, rf, pc, one_c, one_f, ra, pa;
  auto make = [](const std::vector<double>& v, Vec* out) {
    VecCreateSeq(PETSC_COMM_WORLD, PetscInt(v.size()), out);
    PetscScalar* p = nullptr;
    VecGetArray(*out, &p);
    std::memcpy(p, v.data(), sizeof(double) * v.size());
    VecRestoreArray(*out, &p);
  };
  make(xf, &vf);
  make(xc, &vc);
  VecDuplicate(vc, &rf);
  VecDuplicate(vf, &pc);
  VecDuplicate(vc, &one_c);
  VecDuplicate(vf, &one_f);
  VecSet(one_c, 1.0);
  VecSet(one_f, 1.0);
  VecDuplicate(vc, &ra);
  VecDuplicate(vf, &pa);
  VecSet(pc, 7.0);  // overwritten by MatMultTranspose
  if (MatMult(R, vf, rf) || MatMultTranspose(R, vc, pc) || MatMultAdd(R, vf, one_c, ra) ||
      MatMultTransposeAdd(R, vc, one_f, pa))
    return 1;
  const std::string out = argv[8];
  const std::pair<const char*, Vec> outs[] = {{".R", rf}, {".P", pc}, {".RA", ra}, {".PA", pa}};
  for (const auto& o : outs) {
    PetscScalar* p = nullptr;
    VecGetArray(o.second, &p);
    write_raw((out + o.first).c_str(), p, o.second->a.size());
  }
  ((PetscErrorCode(*)(Mat))R->op[MATOP_DESTROY])(R);
  MatDestroy(&R);
  for (Vec v : {vf, vc, rf, pc, one_c, one_f, ra, pa}) VecDestroy(&v);
  dg_damg_destroy(m);
  dg_octree_destroy(tree);
  PetscFinalize();
  return 0;
}

int main(int argc, char** argv) {
  if (argc > 1 && !std::strcmp(argv[1], "transfer")) return run_transfer(argc, argv);
  if (argc < 8) {
    std::fprintf(stderr, "bad arguments\n");
    return 2;
  }
  const std::string mode = argv[1];
  const bool elastic = mode == "elastic";
  if (elastic && argc < 9) return 2;
  PetscInitialize(&argc, &argv, nullptr, nullptr);
  std::vector<uint32_t> raw = read_raw<uint32_t>(argv[2]);
  const uint32_t depth = uint32_t(std::atoi(argv[3]));
  std::vector<dg_octant> octs(raw.size() / 4);
  for (size_t i = 0; i < octs.size(); ++i)
    octs[i] = dg_octant{raw[4 * i], raw[4 * i + 1], raw[4 * i + 2], raw[4 * i + 3]};
  dg_octree* tree = nullptr;
  dg_da* da = nullptr;
  dg_mat* J = nullptr;
  dg_status st = dg_octree_from_octants(octs.data(), int64_t(octs.size()), 0, depth, &tree);
  if (st) return fail("octree", st);
  if ((st = dg_da_create(tree, &da))) return fail("da", st);
  if (elastic) {
    st = dg_mat_create_elasticity(da, std::atof(argv[5]), std::atof(argv[6]), nullptr, &J);
  } else {
    std::vector<double> coef;
    if (std::strcmp(argv[5], "none")) coef = read_raw<double>(argv[5]);
    st = dg_mat_create_lapmass(da, coef.empty() ? nullptr : coef.data(), &J);
  }
  if (st) return fail("operator", st);
  Mat A;
  if (dendro_b200::DgCreateMatShell(PETSC_COMM_WORLD, J, &A)) return 1;
  std::vector<double> xin = read_raw<double>(argv[4]);
  Vec x, y, d;
  VecCreateSeq(PETSC_COMM_WORLD, PetscInt(xin.size()), &x);
  PetscScalar* px = nullptr;
  VecGetArray(x, &px);
  std::memcpy(px, xin.data(), sizeof(double) * xin.size());
  VecRestoreArray(x, &px);
  VecDuplicate(x, &y);
  VecDuplicate(x, &d);
  if (MatMult(A, x, y)) return 1;
  if (MatGetDiagonal(A, d)) return 1;
  const char* out_y = argv[elastic ? 7 : 6];
  const char* out_d = argv[elastic ? 8 : 7];
  PetscScalar* py = nullptr;
  VecGetArray(y, &py);
  write_raw(out_y, py, xin.size());
  PetscScalar* pd = nullptr;
  VecGetArray(d, &pd);
  write_raw(out_d, pd, xin.size());
  // the shell's MATOP_DESTROY frees the operator, as PETSc's MatDestroy calls it
  ((PetscErrorCode(*)(Mat))A->op[MATOP_DESTROY])(A);
  MatDestroy(&A);
  VecDestroy(&x);
  VecDestroy(&y);
  VecDestroy(&d);
  dg_da_destroy(da);
  dg_octree_destroy(tree);
  PetscFinalize();
  return 0;
}
