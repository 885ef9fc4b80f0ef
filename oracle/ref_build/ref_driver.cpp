// Driver of the reference build (oracle/_ref/dendro_ref) -- test
// infrastructure.  It calls the reference's own functions, compiled from its
// sources by oracle/ref_build/build_ref.py, and writes their results as raw
// binary files so that the CPU oracle can be checked against them:
//
//   dendro_ref octree  <pts.f64> <maxDepth> <maxNumPts> <outdir>
//       ot::points2Octree, ot::balanceOctree (incCorner), ot::coarsenOctree
//   dendro_ref balance <octs.u32> <maxDepth> <outdir>
//       ot::balanceOctree (incCorner) and ot::coarsenOctree of a linear octree
//   dendro_ref timings <lin.u32> <maxDepth>
//       seconds of ot::balanceOctree and of the DA construction (stderr:
//       balanced octants, elements, balance s, DA s)
//   dendro_ref mesh    <octs.u32> <maxDepth> <outdir>
//       ot::DA maps: per element anchor, level, child number, hanging mask and
//       the 8 node ids (Vec order), plus the node anchors
//   dendro_ref matvec  <octs.u32> <maxDepth> <x.f64> <coef.f64|none> <out.f64> [reps]
//       Jacobian2MatMult (examples/src/backend/omgJac.C:1775); with reps > 0
//       prints the seconds per application on stderr
//   dendro_ref elastic <octs.u32> <maxDepth> <x.f64> <out.f64>
//       ElasticityMatMult with Dirichlet nodes on the domain boundary
//   dendro_ref transfer <octs.u32> <maxDepth> <nlevels> <outdir>
//       DAMGCreateAndSetDA + DAMGSetUp; per level the node anchors, and the
//       restriction / prolongation of the vectors level<l>_in.f64 /
//       coarse<l>_in.f64 found in outdir
//   dendro_ref elastic_transfer <octs.u32> <maxDepth> <nlevels> <outdir>
//       the elasticity solver's hierarchy (dof 3, suppressed DOFs, elasticity
//       contexts); per level the boundary flags, and the restriction /
//       prolongation of 3-dof vectors level<l>_in.f64 / coarse<l>_in.f64
//   dendro_ref jac3 <octs.u32> <maxDepth> <nlevels> <outdir>
//       DAMGCreateAndSetDA + DAMGSetUp, then per coarse level l (1 = next to
//       the finest) Jacobian3MatMult (examples/src/backend/omgJac.C:2235) with
//       the Jacobian-3 context of that level: the next finer level's DA and
//       its coefficients coef<l-1>.f64 (a, b per element), applied to
//       jin<l>.f64 -> jout<l>.f64 (files in outdir)
//   dendro_ref dirichlet <octs.u32> <maxDepth> <x.f64> <outdir>
//       assignBoundaryFlags (src/oda/odaUtils.C:1054) -> bdy.u8 (nodal Vec),
//       DirichletLaplacianMatMult / DirichletJacobianMatMult and their
//       GetDiagonal (examples/src/backend/omgJac.C:859-1160) -> yL.f64, yJ.f64,
//       dL.f64, dJ.f64
//   dendro_ref io <octs.u32> <maxDepth> <pts.f64> <vals.f64> <outdir>
//       the reference's file writers (src/oct/OctFunctions.C:313-440):
//       writeNodesToFile -> octs.ot, writePtsToFile -> pts.pts,
//       writeDataPtsToFile -> data.pts; then its readers on those files:
//       octs_rt.u32, pts_rt.f64, data_pts_rt.f64, data_vals_rt.f64
//
// Octant files hold 4 x uint32 per octant (x, y, z, level); run from a
// directory that holds the reference's Stencils/*.inp (they are read from the
// working directory).
#include <execinfo.h>
#include <signal.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "petsc.h"
#include "petscmat.h"
#include "petscvec.h"
#include "TreeNode.h"
#include "oda.h"
#include "omg.h"
#include "omgJac.h"
#include "elasticityJac.h"
#include "handleStencils.h"
#include "parUtils.h"
#include "externVars.h"
#include "rotation.h"

// Operator stencil tables (the reference's drivers define these globals).
double**** LaplacianType2Stencil = NULL;
double**** MassType2Stencil = NULL;
double**** GradDivType2Stencil = NULL;
double***** LaplacianType1Stencil = NULL;
double***** MassType1Stencil = NULL;

namespace {

template <class T>
std::vector<T> read_raw(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    fprintf(stderr, "cannot read %s\n", path.c_str());
    exit(2);
  }
  std::streamsize n = f.tellg();
  f.seekg(0);
  std::vector<T> v(size_t(n) / sizeof(T));
  f.read(reinterpret_cast<char*>(v.data()), n);
  return v;
}

template <class T>
void write_raw(const std::string& path, const T* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), std::streamsize(n * sizeof(T)));
}

std::vector<ot::TreeNode> read_octs(const std::string& path, unsigned maxDepth) {
  std::vector<uint32_t> a = read_raw<uint32_t>(path);
  std::vector<ot::TreeNode> v;
  v.reserve(a.size() / 4);
  for (size_t i = 0; i + 3 < a.size(); i += 4) v.push_back(ot::TreeNode(a[i], a[i + 1], a[i + 2], a[i + 3], 3, maxDepth));
  return v;
}

void write_octs(const std::string& path, const std::vector<ot::TreeNode>& v) {
  std::vector<uint32_t> a;
  a.reserve(4 * v.size());
  for (const ot::TreeNode& t : v) {
    a.push_back(t.getX());
    a.push_back(t.getY());
    a.push_back(t.getZ());
    a.push_back(t.getLevel());
  }
  write_raw(path, a.data(), a.size());
}

// Per element: anchor, level, child number, hanging mask, Vec ids of the 8
// nodes; node anchors indexed by Vec id.
void dump_mesh(ot::DA& da, const std::string& dir, const std::string& tag) {
  const unsigned nvec = da.getNodeSize();  // includes the boundary nodes (oda.txx:141)
  std::vector<double> ids(nvec);
  for (unsigned i = 0; i < nvec; ++i) ids[i] = i;
  double* buf = NULL;
  da.vecGetBuffer<double>(ids, buf, false, false, true, 1);
  std::vector<uint32_t> elem, node_xyz(3 * size_t(nvec), 0xffffffffu);
  const unsigned D = da.getMaxDepth();
  if (da.iAmActive()) {
    for (da.init<ot::DA_FLAGS::ALL>(); da.curr() < da.end<ot::DA_FLAGS::ALL>(); da.next<ot::DA_FLAGS::ALL>()) {
      unsigned idx = da.curr();
      Point p = da.getCurrentOffset();
      unsigned lev = da.getLevel(idx);
      unsigned s = 1u << (D - lev);
      unsigned c = da.getChildNumber();
      unsigned mask = da.getHangingNodeIndex(idx);
      unsigned nodes[8];
      da.getNodeIndices(nodes);
      unsigned px = p.xint(), py = p.yint(), pz = p.zint();
      unsigned qx = px & ~(2 * s - 1), qy = py & ~(2 * s - 1), qz = pz & ~(2 * s - 1);
      elem.push_back(px);
      elem.push_back(py);
      elem.push_back(pz);
      elem.push_back(lev);
      elem.push_back(c);
      elem.push_back(mask);
      for (int v = 0; v < 8; ++v) {
        unsigned id = unsigned(buf[nodes[v]]);
        elem.push_back(id);
        bool hang = (mask >> v) & 1u;
        unsigned bx = hang ? qx + ((v & 1) ? 2 * s : 0) : px + ((v & 1) ? s : 0);
        unsigned by = hang ? qy + ((v & 2) ? 2 * s : 0) : py + ((v & 2) ? s : 0);
        unsigned bz = hang ? qz + ((v & 4) ? 2 * s : 0) : pz + ((v & 4) ? s : 0);
        if (id < nvec) {
          node_xyz[3 * id] = bx;
          node_xyz[3 * id + 1] = by;
          node_xyz[3 * id + 2] = bz;
        }
      }
    }
  }
  da.vecRestoreBuffer<double>(ids, buf, false, false, true, 1);
  write_raw(dir + "/" + tag + "elem.u32", elem.data(), elem.size());
  write_raw(dir + "/" + tag + "node_xyz.u32", node_xyz.data(), node_xyz.size());
}

Vec make_vec(const std::vector<double>& a) {
  Vec v;
  VecCreate(MPI_COMM_WORLD, &v);
  VecSetSizes(v, int(a.size()), PETSC_DECIDE);
  double* p;
  VecGetArray(v, &p);
  std::memcpy(p, a.data(), 8 * a.size());
  VecRestoreArray(v, &p);
  return v;
}

std::vector<double> vec_data(Vec v) {
  double* p;
  int n;
  VecGetLocalSize(v, &n);
  VecGetArray(v, &p);
  std::vector<double> a(p, p + n);
  VecRestoreArray(v, &p);
  return a;
}

}  // namespace

static void on_fault(int sig) {
  void* bt[64];
  int n = backtrace(bt, 64);
  fprintf(stderr, "fatal signal %d\n", sig);
  backtrace_symbols_fd(bt, n, 2);
  _exit(128 + sig);
}

int main(int argc, char** argv) {
  signal(SIGSEGV, on_fault);
  std::cout.setstate(std::ios::badbit);  // the reference prints progress on every octant
  // every TreeNode constructor computes (unused, Morton build) Hilbert rotation
  // data from these tables; the reference's drivers fill them the same way
  // (examples/src/drivers/testPartition.C:35)
  initializeHilbetTable(2);
  initializeHilbetTable(3);
  const bool verbose = getenv("DG_REF_VERBOSE") != NULL;
  if (verbose) fprintf(stderr, "tables ready\n");
  if (argc < 2) {
    fprintf(stderr, "usage: see the header of ref_driver.cpp\n");
    return 2;
  }
  std::string mode = argv[1];
  if (mode == "octree" && argc >= 6) {
    std::vector<double> pts = read_raw<double>(argv[2]);
    unsigned D = atoi(argv[3]), m = atoi(argv[4]);
    std::string dir = argv[5];
    double gSize[3] = {1.0, 1.0, 1.0};
    std::vector<ot::TreeNode> lin, bal, tmp, coarse;
    ot::points2Octree(pts, gSize, lin, 3, D, m, MPI_COMM_WORLD);
    if (verbose) fprintf(stderr, "p2o %zu\n", lin.size());
    write_octs(dir + "/p2o.u32", lin);
    tmp = lin;
    ot::balanceOctree(tmp, bal, 3, D, true, MPI_COMM_WORLD, NULL, NULL);
    write_octs(dir + "/bal.u32", bal);
    ot::coarsenOctree(bal, coarse);
    write_octs(dir + "/coarse.u32", coarse);
    return 0;
  }
  if (mode == "balance" && argc >= 5) {
    unsigned D = atoi(argv[3]);
    std::string dir = argv[4];
    std::vector<ot::TreeNode> lin = read_octs(argv[2], D), bal, coarse;
    ot::balanceOctree(lin, bal, 3, D, true, MPI_COMM_WORLD, NULL, NULL);
    write_octs(dir + "/bal.u32", bal);
    ot::coarsenOctree(bal, coarse);
    write_octs(dir + "/coarse.u32", coarse);
    return 0;
  }
  if (mode == "timings" && argc >= 4) {
    // the set-up stages of examples/src/drivers/tstMatVec.C:165-275 on a
    // linear octree: balanceOctree, then the DA; seconds on stderr
    unsigned D = atoi(argv[3]);
    std::vector<ot::TreeNode> lin = read_octs(argv[2], D), bal;
    auto t0 = std::chrono::steady_clock::now();
    ot::balanceOctree(lin, bal, 3, D, true, MPI_COMM_WORLD, NULL, NULL);
    auto t1 = std::chrono::steady_clock::now();
    const size_t nbal = bal.size();
    ot::DA da(bal, MPI_COMM_WORLD, MPI_COMM_WORLD, false);
    auto t2 = std::chrono::steady_clock::now();
    fprintf(stderr, "%zu %u %.6f %.6f\n", nbal, da.getElementSize(),
            std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(t2 - t1).count());
    return 0;
  }
  if (mode == "jac3" && argc >= 6) {
    unsigned D = atoi(argv[3]);
    int nlevels = atoi(argv[4]);
    std::string dir = argv[5];
    std::vector<ot::TreeNode> octs = read_octs(argv[2], D);
    ot::DAMG* damg = NULL;
    ot::DAMG_Initialize(MPI_COMM_WORLD);
    ot::DAMGCreateAndSetDA(MPI_COMM_WORLD, nlevels, NULL, &damg, octs, 1, 1.5, false, true);
    ot::DAMGSetUp(damg);
    createLmatType2(LaplacianType2Stencil);
    createMmatType2(MassType2Stencil);
    createLmatType1(LaplacianType1Stencil);
    createMmatType1(MassType1Stencil);
    for (int l = 1; l < nlevels; ++l) {
      ot::DAMG fine = damg[nlevels - l], coarse = damg[nlevels - 1 - l];
      std::vector<double> coef = read_raw<double>(dir + "/coef" + std::to_string(l - 1) + ".f64");
      std::vector<double> matProp;
      fine->da->createVector(matProp, true, true, 2);
      for (size_t i = 0; i < matProp.size() && i < coef.size(); ++i) matProp[i] = coef[i];
      Jac3MFreeData data;
      std::memset((void*)&data, 0, sizeof(data));
      data.daf = fine->da;
      data.matPropFine = &matProp;
      data.isFinestLevel = false;
      data.isCoarsestLevel = (l == nlevels - 1);
      data.changedPartition = false;
      void* saved = coarse->user;
      coarse->user = &data;
      std::vector<double> x = read_raw<double>(dir + "/jin" + std::to_string(l) + ".f64");
      Mat J;
      MatCreateShell(MPI_COMM_WORLD, int(x.size()), int(x.size()), PETSC_DETERMINE, PETSC_DETERMINE, coarse, &J);
      Vec in = make_vec(x), out = make_vec(x);
      Jacobian3MatMult(J, in, out);
      std::vector<double> y = vec_data(out);
      write_raw(dir + "/jout" + std::to_string(l) + ".f64", y.data(), y.size());
      coarse->user = saved;
    }
    return 0;
  }
  if (mode == "dirichlet" && argc >= 6) {
    unsigned D = atoi(argv[3]);
    std::vector<ot::TreeNode> octs = read_octs(argv[2], D);
    ot::DA da(octs, MPI_COMM_WORLD, MPI_COMM_WORLD, false);
    createLmatType2(LaplacianType2Stencil);
    createMmatType2(MassType2Stencil);
    std::vector<double> x = read_raw<double>(argv[4]);
    std::string dir = argv[5];
    std::vector<unsigned char> flags;
    ot::assignBoundaryFlags(&da, flags);
    write_raw(dir + "/bdy.u8", flags.data(), flags.size());
    DirichletJacData data;
    std::memset((void*)&data, 0, sizeof(data));
    da.vecGetBuffer<unsigned char>(flags, data.bdyArr, false, false, true, 1);
    ot::DAMG damg = new ot::_p_DAMG;
    std::memset((void*)damg, 0, sizeof(ot::_p_DAMG));
    damg->da = &da;
    damg->nlevels = 1;
    damg->user = &data;
    Mat J;
    MatCreateShell(MPI_COMM_WORLD, int(x.size()), int(x.size()), PETSC_DETERMINE, PETSC_DETERMINE, damg, &J);
    Vec in = make_vec(x), out = make_vec(x), dg = make_vec(x);
    DirichletLaplacianMatMult(J, in, out);
    std::vector<double> y = vec_data(out);
    write_raw(dir + "/yL.f64", y.data(), y.size());
    DirichletJacobianMatMult(J, in, out);
    y = vec_data(out);
    write_raw(dir + "/yJ.f64", y.data(), y.size());
    DirichletLaplacianMatGetDiagonal(J, dg);
    y = vec_data(dg);
    write_raw(dir + "/dL.f64", y.data(), y.size());
    DirichletJacobianMatGetDiagonal(J, dg);
    y = vec_data(dg);
    write_raw(dir + "/dJ.f64", y.data(), y.size());
    return 0;
  }
  if (mode == "io" && argc >= 7) {
    unsigned D = atoi(argv[3]);
    std::vector<ot::TreeNode> octs = read_octs(argv[2], D);
    std::vector<double> pts = read_raw<double>(argv[4]), vals = read_raw<double>(argv[5]);
    std::string dir = argv[6];
    std::string fo = dir + "/octs.ot", fp = dir + "/pts.pts", fd = dir + "/data.pts";
    ot::writeNodesToFile(&fo[0], octs);
    ot::writePtsToFile(&fp[0], pts);
    ot::writeDataPtsToFile(&fd[0], pts, vals);
    std::vector<ot::TreeNode> o2;
    ot::readNodesFromFile(&fo[0], o2);
    write_octs(dir + "/octs_rt.u32", o2);
    std::vector<double> p2, p3, v3;
    if (!pts.empty()) ot::readPtsFromFile(&fp[0], p2);  // its writer leaves no header for no points
    write_raw(dir + "/pts_rt.f64", p2.data(), p2.size());
    ot::readDataPtsFromFile(&fd[0], p3, v3);
    write_raw(dir + "/data_pts_rt.f64", p3.data(), p3.size());
    write_raw(dir + "/data_vals_rt.f64", v3.data(), v3.size());
    return 0;
  }
  if (mode == "mesh" && argc >= 5) {
    unsigned D = atoi(argv[3]);
    std::vector<ot::TreeNode> octs = read_octs(argv[2], D);
    ot::DA da(octs, MPI_COMM_WORLD, MPI_COMM_WORLD, false);
    dump_mesh(da, argv[4], "");
    return 0;
  }
  if (mode == "matvec" && argc >= 7) {
    unsigned D = atoi(argv[3]);
    int reps = argc >= 8 ? atoi(argv[7]) : 0;
    std::vector<ot::TreeNode> octs = read_octs(argv[2], D);
    ot::DA da(octs, MPI_COMM_WORLD, MPI_COMM_WORLD, false);
    createLmatType2(LaplacianType2Stencil);
    createMmatType2(MassType2Stencil);
    std::vector<double> x = read_raw<double>(argv[4]);
    std::vector<double> coef;
    if (std::string(argv[5]) != "none") {
      coef = read_raw<double>(argv[5]);
    } else {
      coef.assign(2 * size_t(da.getElementSize()), 1.0);
    }
    std::vector<double> matProp;
    da.createVector(matProp, true, true, 2);
    for (size_t i = 0; i < matProp.size() && i < coef.size(); ++i) matProp[i] = coef[i];
    ot::DAMG damg = new ot::_p_DAMG;
    std::memset((void*)damg, 0, sizeof(ot::_p_DAMG));
    damg->da = &da;
    Jac2MFreeData data;
    data.matProp = &matProp;
    data.isFinestLevel = true;
    damg->user = &data;
    Mat J;
    MatCreateShell(MPI_COMM_WORLD, int(x.size()), int(x.size()), PETSC_DETERMINE, PETSC_DETERMINE, damg, &J);
    Vec in = make_vec(x), out = make_vec(x);
    Jacobian2MatMult(J, in, out);
    std::vector<double> y = vec_data(out);
    write_raw(argv[6], y.data(), y.size());
    if (reps > 0) {
      auto t0 = std::chrono::steady_clock::now();
      for (int r = 0; r < reps; ++r) Jacobian2MatMult(J, in, out);
      double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      fprintf(stderr, "%.9f\n", dt / reps);
    }
    return 0;
  }
  if (mode == "elastic" && argc >= 6) {
    unsigned D = atoi(argv[3]);
    std::vector<ot::TreeNode> octs = read_octs(argv[2], D);
    ot::DA da(octs, MPI_COMM_WORLD, MPI_COMM_WORLD, false);
    createLmatType2(LaplacianType2Stencil);
    createGDmatType2(GradDivType2Stencil);
    std::vector<double> x = read_raw<double>(argv[4]);
    // Dirichlet flags per octant-buffer entry: nodes on the domain boundary
    const unsigned Dm = da.getMaxDepth(), top = 1u << (Dm - 1);
    std::vector<unsigned char> bdy(da.getLocalBufferSize(), 0);
    for (da.init<ot::DA_FLAGS::ALL>(); da.curr() < da.end<ot::DA_FLAGS::ALL>(); da.next<ot::DA_FLAGS::ALL>()) {
      unsigned idx = da.curr();
      Point p = da.getCurrentOffset();
      unsigned s = 1u << (Dm - da.getLevel(idx));
      unsigned mask = da.getHangingNodeIndex(idx);
      unsigned nodes[8];
      da.getNodeIndices(nodes);
      for (int v = 0; v < 8; ++v) {
        if ((mask >> v) & 1u) continue;
        unsigned bx = p.xint() + ((v & 1) ? s : 0), by = p.yint() + ((v & 2) ? s : 0), bz = p.zint() + ((v & 4) ? s : 0);
        if (!bx || !by || !bz || bx == top || by == top || bz == top) bdy[nodes[v]] = 1;
      }
    }
    ot::DAMG damg = new ot::_p_DAMG;
    std::memset((void*)damg, 0, sizeof(ot::_p_DAMG));
    damg->da = &da;
    damg->nlevels = 1;
    ElasticityData data;
    data.bdyArr = bdy.data();
    data.mu = 1.0 / (2.0 * 1.3);
    data.lambda = 0.3 / (1.3 * 0.4);
    damg->user = &data;
    Mat J;
    MatCreateShell(MPI_COMM_WORLD, int(x.size()), int(x.size()), PETSC_DETERMINE, PETSC_DETERMINE, damg, &J);
    Vec in = make_vec(x), out = make_vec(x);
    ElasticityMatMult(J, in, out);
    std::vector<double> y = vec_data(out);
    write_raw(argv[5], y.data(), y.size());
    return 0;
  }
  if (mode == "transfer" && argc >= 6) {
    unsigned D = atoi(argv[3]);
    int nlevels = atoi(argv[4]);
    std::string dir = argv[5];
    std::vector<ot::TreeNode> octs = read_octs(argv[2], D);
    ot::DAMG* damg = NULL;
    ot::DAMG_Initialize(MPI_COMM_WORLD);
    ot::DAMGCreateAndSetDA(MPI_COMM_WORLD, nlevels, NULL, &damg, octs, 1, 1.5, false, true);
    ot::DAMGSetUp(damg);
    FILE* f = fopen((dir + "/levels.txt").c_str(), "w");
    fprintf(f, "%d\n", nlevels);
    fclose(f);
    // level numbering here: 0 = finest (damg[nlevels-1] in the reference)
    for (int l = 0; l < nlevels; ++l) {
      ot::DA* da = damg[nlevels - 1 - l]->da;
      dump_mesh(*da, dir, "level" + std::to_string(l) + "_");
    }
    for (int l = 0; l + 1 < nlevels; ++l) {
      ot::DAMG fine = damg[nlevels - 1 - l];
      std::string fin = dir + "/level" + std::to_string(l) + "_in.f64";
      std::string cin = dir + "/coarse" + std::to_string(l) + "_in.f64";
      std::vector<double> xf = read_raw<double>(fin), xc = read_raw<double>(cin);
      Vec vf = make_vec(xf), vc = make_vec(xc), of, oc;
      VecDuplicate(vc, &oc);
      VecDuplicate(vf, &of);
      MatMult(fine->R, vf, oc);           // restriction
      MatMultTranspose(fine->R, vc, of);  // prolongation
      std::vector<double> r = vec_data(oc), p = vec_data(of);
      write_raw(dir + "/restrict" + std::to_string(l) + ".f64", r.data(), r.size());
      write_raw(dir + "/prolong" + std::to_string(l) + ".f64", p.data(), p.size());
    }
    return 0;
  }
  if (mode == "elastic_transfer" && argc >= 6) {
    // The elasticity solver's set-up order (examples/src/drivers/newElasSolver.C:
    // DAMGCreateAndSetDA with dof 3, DAMGCreateSuppressedDOFs,
    // SetElasticityContexts), then the restriction / prolongation of 3-dof
    // vectors level<l>_in.f64 / coarse<l>_in.f64 -> restrict<l>.f64 /
    // prolong<l>.f64, and each level's boundary flags bdy<l>.u8
    unsigned D = atoi(argv[3]);
    int nlevels = atoi(argv[4]);
    std::string dir = argv[5];
    std::vector<ot::TreeNode> octs = read_octs(argv[2], D);
    ot::DAMG* damg = NULL;
    ot::DAMG_Initialize(MPI_COMM_WORLD);
    ot::DAMGCreateAndSetDA(MPI_COMM_WORLD, nlevels, NULL, &damg, octs, 3, 1.5, false, true);
    ot::DAMGCreateSuppressedDOFs(damg);
    SetElasticityContexts(damg);
    FILE* f = fopen((dir + "/levels.txt").c_str(), "w");
    fprintf(f, "%d\n", nlevels);
    fclose(f);
    for (int l = 0; l < nlevels; ++l) {
      ot::DA* da = damg[nlevels - 1 - l]->da;
      std::vector<unsigned char> bdy;
      assignBoundaryFlags(da, bdy);
      write_raw(dir + "/bdy" + std::to_string(l) + ".u8", bdy.data(), bdy.size());
    }
    for (int l = 0; l + 1 < nlevels; ++l) {
      ot::DAMG fine = damg[nlevels - 1 - l];
      std::vector<double> xf = read_raw<double>(dir + "/level" + std::to_string(l) + "_in.f64");
      std::vector<double> xc = read_raw<double>(dir + "/coarse" + std::to_string(l) + "_in.f64");
      Vec vf = make_vec(xf), vc = make_vec(xc), of, oc;
      VecDuplicate(vc, &oc);
      VecDuplicate(vf, &of);
      MatMult(fine->R, vf, oc);
      MatMultTranspose(fine->R, vc, of);
      std::vector<double> r = vec_data(oc), p = vec_data(of);
      write_raw(dir + "/restrict" + std::to_string(l) + ".f64", r.data(), r.size());
      write_raw(dir + "/prolong" + std::to_string(l) + ".f64", p.data(), p.size());
    }
    return 0;
  }
  fprintf(stderr, "bad arguments\n");
  return 2;
}
