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

int main(int argc, char** argv) {
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
