// CPU ORACLE -- test infrastructure only.
//
// A plain C++ restatement of the reference (hsundar/dendro) algorithms on the
// matrix-free octree FEM path.  Only tests/, __graft_entry__.smoke() and the
// bench's cpu_baseline / reference arm may load this library, and only as the
// checker.  The product (dendro_b200/) never calls it.
//
// Every function cites the reference file:line whose behaviour it restates.
// Algorithms are deliberately written the simple way (dense stencil tables,
// sequential loops, split-until-stable balance) so that they are independent
// of the GPU formulations they check.
//
// Octant record: {x, y, z, level|flags}; flags use the reference bit layout
// (level mask 31, BOUNDARY 64, NODE 128: include/oct/TreeNode.h:77-78).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <numeric>
#include <vector>

namespace {

constexpr uint32_t LEVEL_MASK = 31u, BOUNDARY = 64u, NODE = 128u;

struct Oct {
  uint32_t x, y, z, lf;
  uint32_t lev() const { return lf & LEVEL_MASK; }
};

// Morton comparison: TreeNode.txx:160-188 (original Morton block) and
// src/hilbert/morton.cpp:18-60.  The most significant differing bit of
// x^y^z decides, preferring z over y over x; equal anchors order the coarser
// octant first.
inline bool msb_less(uint32_t a, uint32_t b) { return a < b && a < (a ^ b); }
inline bool morton_less(const Oct& a, const Oct& b) {
  if (a.x == b.x && a.y == b.y && a.z == b.z) return a.lev() < b.lev();
  uint32_t dx = a.x ^ b.x, dy = a.y ^ b.y, dz = a.z ^ b.z;
  // pick the axis holding the highest differing bit; ties go z > y > x
  int axis = 2;
  uint32_t m = dz;
  if (msb_less(m, dy)) { m = dy; axis = 1; }
  if (msb_less(m, dx)) { m = dx; axis = 0; }
  if (axis == 2) return a.z < b.z;
  if (axis == 1) return a.y < b.y;
  return a.x < b.x;
}
inline bool oct_eq(const Oct& a, const Oct& b) {  // TreeNode.txx:122-135
  return a.x == b.x && a.y == b.y && a.z == b.z && a.lev() == b.lev();
}
inline Oct make(uint32_t x, uint32_t y, uint32_t z, uint32_t l, uint32_t f = 0) {
  return Oct{x, y, z, l | f};
}
inline Oct parent_of(const Oct& o, uint32_t D) {  // TreeNode.txx:264-274
  uint32_t pl = o.lev() > 0 ? o.lev() - 1 : 0;
  uint32_t sh = D - pl;
  uint64_t m = ~((1ull << sh) - 1);
  return make(uint32_t(o.x & m), uint32_t(o.y & m), uint32_t(o.z & m), pl);
}
inline uint32_t child_number(const Oct& o, uint32_t D) {  // oda.txx:1087-1108
  uint32_t len = 1u << (D - o.lev());
  uint32_t i = (o.x / len) & 1u, j = (o.y / len) & 1u, k = (o.z / len) & 1u;
  return 4 * k + 2 * j + i;
}

// 64-bit interleaved Morton key of an anchor (z>y>x within each bit triple);
// integer order of keys equals morton_less for distinct anchors.
inline uint64_t spread3(uint32_t v) {
  uint64_t r = 0;
  for (int b = 0; b < 21; ++b) r |= uint64_t((v >> b) & 1u) << (3 * b);
  return r;
}
inline uint64_t akey(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// Index of the octant with the largest anchor key <= key (seq::maxLowerBound,
// include/seq/seqUtils.txx:55), or -1.
inline int64_t max_lower_bound(const std::vector<uint64_t>& keys, uint64_t k) {
  auto it = std::upper_bound(keys.begin(), keys.end(), k);
  if (it == keys.begin()) return -1;
  return int64_t(it - keys.begin()) - 1;
}

// ---------------------------------------------------------------- octree --
// points2OctreeSeq (src/oct/Construct.C:880-936): quantise, sort, then
// p2oLocal (Construct.C:940-1015).  p2oLocal's walk emits, in Morton order,
// the coarsest octants that hold at most maxNumPts points unless they are at
// maxDepth; stated here as the equivalent top-down recursion.
void p2o_rec(const std::vector<uint64_t>& pk, size_t lo, size_t hi, uint32_t x, uint32_t y,
             uint32_t z, uint32_t lev, uint32_t D, uint32_t maxNumPts, std::vector<Oct>& out) {
  if (hi - lo <= maxNumPts || lev == D) {
    out.push_back(make(x, y, z, lev));
    return;
  }
  uint32_t cl = 1u << (D - lev - 1);
  size_t a = lo;
  for (uint32_t c = 0; c < 8; ++c) {
    uint32_t cx = x + ((c & 1) ? cl : 0), cy = y + ((c & 2) ? cl : 0), cz = z + ((c & 4) ? cl : 0);
    uint64_t kend = akey(cx, cy, cz) + (1ull << (3 * (D - lev - 1)));
    size_t b = std::lower_bound(pk.begin() + a, pk.begin() + hi, kend) - pk.begin();
    p2o_rec(pk, a, b, cx, cy, cz, lev + 1, D, maxNumPts, out);
    a = b;
  }
}

std::vector<Oct> points2octree(const double* pts, size_t n, uint32_t D, uint32_t maxNumPts) {
  std::vector<uint64_t> pk(n);
  const double scale = double(1u << D);
  for (size_t i = 0; i < n; ++i) {
    // Construct.C:900-911 (gLens = 1)
    uint32_t px = uint32_t(pts[3 * i] * scale / 1.0);
    uint32_t py = uint32_t(pts[3 * i + 1] * scale / 1.0);
    uint32_t pz = uint32_t(pts[3 * i + 2] * scale / 1.0);
    pk[i] = akey(px, py, pz);
  }
  std::sort(pk.begin(), pk.end());
  std::vector<Oct> out;
  if (D == 0 || n <= maxNumPts) {  // Construct.C:884-888, 915-919
    out.push_back(make(0, 0, 0, 0));
    return out;
  }
  p2o_rec(pk, 0, n, 0, 0, 0, 0, D, maxNumPts, out);
  return out;
}

// 2:1 balance with corners (balanceOctree -> comboRipple, src/oct/Balance.C:31,
// 767, 1162).  The reference's ripple result is the coarsest 2:1-balanced
// refinement, which is unique; restated as split-until-stable: a leaf is split
// when it strictly contains a same-level neighbour of the parent of a finer
// leaf (the 26 directions, incCorner = true).
std::vector<Oct> balance(std::vector<Oct> in, uint32_t D) {
  const uint64_t side = 1ull << D;
  for (;;) {
    std::vector<uint64_t> keys(in.size());
    for (size_t i = 0; i < in.size(); ++i) keys[i] = akey(in[i].x, in[i].y, in[i].z);
    std::vector<char> split(in.size(), 0);
    bool any = false;
    for (size_t i = 0; i < in.size(); ++i) {
      uint32_t m = in[i].lev();
      if (m < 2) continue;
      Oct p = parent_of(in[i], D);
      int64_t s = int64_t(1) << (D - (m - 1));
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            if (!dx && !dy && !dz) continue;
            int64_t nx = int64_t(p.x) + dx * s, ny = int64_t(p.y) + dy * s,
                    nz = int64_t(p.z) + dz * s;
            if (nx < 0 || ny < 0 || nz < 0 || nx >= int64_t(side) || ny >= int64_t(side) ||
                nz >= int64_t(side))
              continue;
            int64_t j = max_lower_bound(keys, akey(uint32_t(nx), uint32_t(ny), uint32_t(nz)));
            if (j >= 0 && in[j].lev() < m - 1 && !split[j]) {
              split[j] = 1;
              any = true;
            }
          }
    }
    if (!any) return in;
    std::vector<Oct> nxt;
    nxt.reserve(in.size() + 8);
    for (size_t i = 0; i < in.size(); ++i) {
      if (!split[i]) {
        nxt.push_back(in[i]);
        continue;
      }
      uint32_t cl = 1u << (D - in[i].lev() - 1);
      for (uint32_t c = 0; c < 8; ++c)  // TreeNode.C addChildren order: x, then y, then z
        nxt.push_back(make(in[i].x + ((c & 1) ? cl : 0), in[i].y + ((c & 2) ? cl : 0),
                           in[i].z + ((c & 4) ? cl : 0), in[i].lev() + 1));
    }
    in.swap(nxt);
  }
}

// coarsenOctree, sequential form (src/oct/Coarsen.C:53-104): every complete
// family of 8 leaf siblings starting at a child-0 octant becomes its parent.
std::vector<Oct> coarsen(const std::vector<Oct>& in, uint32_t D) {
  std::vector<Oct> out;
  size_t n = in.size();
  if (n < 8) return in;
  size_t prev = 0;
  while (prev < n) {
    size_t cur = prev + 1;
    while (cur < n && child_number(in[cur], D) != 0) ++cur;
    if (cur >= prev + 8) {
      out.push_back(parent_of(in[prev], D));
      for (size_t k = prev + 8; k < cur; ++k) out.push_back(in[k]);
    } else {
      for (size_t k = prev; k < cur; ++k) out.push_back(in[k]);
    }
    prev = cur;
  }
  return out;
}

// ------------------------------------------------------------------ mesh --
// Mesh of one level: addBoundaryNodesType1 (src/oct/OctFunctions.C:636-716),
// flagNodesType3 (OctFunctions.C:1501-2025) and the element->node map of
// DA::buildNodeList (src/oda/private/odaBuildNlist.C:47-856).  Node ids are
// the positions of NODE-flagged octants among all octants in DA order, i.e.
// the PETSc Vec order of DA::vecGetBuffer (include/oda/oda.txx:948-970).
struct Mesh {
  uint32_t D = 0;  // embedded depth (maxDepth + 1)
  std::vector<Oct> oct;          // elements followed by boundary pseudo-octants
  size_t E = 0, N = 0;
  std::vector<uint32_t> nlist;   // [E][8] node ids
  std::vector<uint8_t> hmask;    // [E] hanging mask (bit v: vertex v hanging)
  std::vector<uint8_t> cnum;     // [E]
  std::vector<uint8_t> etype;    // [E] in [0,18)
  std::vector<uint8_t> elev;     // [E] embedded level
  std::vector<uint32_t> node_xyz;  // [N][3] node anchors (embedded coords)
  std::vector<uint8_t> node_bdy;   // [N] 1 if the node lies on the domain boundary
};

// Element-type table: the hanging masks of the 18 types for each child number
// (include/oda/cnumEtypes.h:19-229, getElemType include/oda/odaUtils.txx:13-94).
const uint8_t kEtypeMask[8][18] = {
    {0, 4, 2, 6, 16, 20, 18, 22, 14, 30, 84, 86, 94, 50, 54, 62, 118, 126},
    {0, 1, 8, 9, 32, 33, 40, 41, 13, 45, 49, 57, 61, 168, 169, 173, 185, 189},
    {0, 8, 1, 9, 64, 72, 65, 73, 11, 75, 200, 201, 203, 81, 89, 91, 217, 219},
    {0, 2, 4, 6, 128, 130, 132, 134, 7, 135, 162, 166, 167, 196, 198, 199, 230, 231},
    {0, 1, 32, 33, 64, 65, 96, 97, 35, 99, 69, 101, 103, 224, 225, 227, 229, 231},
    {0, 2, 128, 130, 16, 18, 144, 146, 138, 154, 19, 147, 155, 208, 210, 218, 211, 219},
    {0, 4, 16, 20, 128, 132, 144, 148, 21, 149, 140, 156, 157, 176, 180, 181, 188, 189},
    {0, 8, 64, 72, 32, 40, 96, 104, 76, 108, 42, 106, 110, 112, 120, 124, 122, 126}};

int etype_of(uint32_t c, uint32_t mask) {
  for (int t = 0; t < 18; ++t)
    if (kEtypeMask[c][t] == mask) return t;
  return -1;
}

int build_mesh(const std::vector<Oct>& tree, uint32_t maxDepth, Mesh& M) {
  const uint32_t D = maxDepth + 1;
  M.D = D;
  std::vector<Oct> elems, bdy;
  elems.reserve(tree.size());
  const uint32_t top = 1u << maxDepth;
  for (const Oct& o : tree) {
    uint32_t d = o.lev();
    uint32_t len = 1u << (maxDepth - d);
    uint32_t blen = top - len;  // TreeNode.C:247-271
    bool px = o.x == blen, py = o.y == blen, pz = o.z == blen;
    if (px) bdy.push_back(make(top, o.y, o.z, d + 1, BOUNDARY));
    if (py) bdy.push_back(make(o.x, top, o.z, d + 1, BOUNDARY));
    if (pz) bdy.push_back(make(o.x, o.y, top, d + 1, BOUNDARY));
    if (px && py) bdy.push_back(make(top, top, o.z, d + 1, BOUNDARY));
    if (px && pz) bdy.push_back(make(top, o.y, top, d + 1, BOUNDARY));
    if (py && pz) bdy.push_back(make(o.x, top, top, d + 1, BOUNDARY));
    if (px && py && pz) bdy.push_back(make(top, top, top, d + 1, BOUNDARY));
    elems.push_back(make(o.x, o.y, o.z, d + 1));
  }
  std::sort(bdy.begin(), bdy.end(), morton_less);
  M.E = elems.size();
  M.oct = elems;
  M.oct.insert(M.oct.end(), bdy.begin(), bdy.end());
  std::vector<Oct>& all = M.oct;
  const size_t n = all.size();

  // flagNodesType3: an octant's anchor is hanging when the parent of one of
  // its same-level negative neighbours (across the parent's faces/edges that
  // hold the anchor) is itself an octant of the tree.
  auto find_exact = [&](const Oct& key) -> bool {
    auto it = std::lower_bound(all.begin(), all.end(), key, morton_less);
    return it != all.end() && oct_eq(*it, key);
  };
  for (size_t i = 0; i < n; ++i) {
    Oct& o = all[i];
    uint32_t m = o.lev();
    bool hanging = false;
    if (m != 1) {
      uint32_t c = child_number(o, D);
      uint32_t s = 1u << (D - m);
      uint32_t zero_axes = (~c) & 7u;
      if (c != 0 && c != 7) {
        for (uint32_t S = 1; S < 8 && !hanging; ++S) {
          if ((S & zero_axes) != S) continue;
          if ((S & 1) && o.x == 0) continue;
          if ((S & 2) && o.y == 0) continue;
          if ((S & 4) && o.z == 0) continue;
          Oct nb = make(o.x - ((S & 1) ? s : 0), o.y - ((S & 2) ? s : 0), o.z - ((S & 4) ? s : 0), m);
          if (find_exact(parent_of(nb, D))) hanging = true;
        }
      }
    }
    if (!hanging) o.lf |= NODE;
  }

  // node numbering: NODE octants in DA order
  std::vector<uint64_t> nkeys;
  std::vector<uint32_t> nid(n, UINT32_MAX);
  for (size_t i = 0; i < n; ++i)
    if (all[i].lf & NODE) {
      nid[i] = uint32_t(M.node_xyz.size() / 3);
      M.node_xyz.push_back(all[i].x);
      M.node_xyz.push_back(all[i].y);
      M.node_xyz.push_back(all[i].z);
      nkeys.push_back(akey(all[i].x, all[i].y, all[i].z));
    }
  M.N = nkeys.size();
  M.node_bdy.resize(M.N);
  for (size_t k = 0; k < M.N; ++k) {
    uint32_t x = M.node_xyz[3 * k], y = M.node_xyz[3 * k + 1], z = M.node_xyz[3 * k + 2];
    M.node_bdy[k] = (x == 0 || y == 0 || z == 0 || x == top || y == top || z == top);
  }
  auto node_at = [&](uint32_t x, uint32_t y, uint32_t z) -> int64_t {
    uint64_t k = akey(x, y, z);
    auto it = std::lower_bound(nkeys.begin(), nkeys.end(), k);
    if (it != nkeys.end() && *it == k) return int64_t(it - nkeys.begin());
    return -1;
  };

  M.nlist.resize(8 * M.E);
  M.hmask.resize(M.E);
  M.cnum.resize(M.E);
  M.etype.resize(M.E);
  M.elev.resize(M.E);
  for (size_t e = 0; e < M.E; ++e) {
    const Oct& o = all[e];
    uint32_t m = o.lev(), s = 1u << (D - m);
    Oct p = parent_of(o, D);
    uint32_t mask = 0;
    for (uint32_t v = 0; v < 8; ++v) {
      uint32_t vx = o.x + ((v & 1) ? s : 0), vy = o.y + ((v & 2) ? s : 0), vz = o.z + ((v & 4) ? s : 0);
      int64_t k = node_at(vx, vy, vz);
      if (k < 0) {
        // hanging vertex: the parent's vertex v (odaBuildNlist.C:560-690)
        mask |= 1u << v;
        k = node_at(p.x + ((v & 1) ? 2 * s : 0), p.y + ((v & 2) ? 2 * s : 0),
                    p.z + ((v & 4) ? 2 * s : 0));
        if (k < 0) return -2;  // not 2:1 balanced
      }
      M.nlist[8 * e + v] = uint32_t(k);
    }
    uint32_t c = child_number(o, D);
    int t = mask ? etype_of(c, mask) : 0;
    if (t < 0) return -3;  // hanging configuration outside the 18 types
    M.hmask[e] = uint8_t(mask);
    M.cnum[e] = uint8_t(c);
    M.etype[e] = uint8_t(t);
    M.elev[e] = uint8_t(m);
  }
  return 0;
}

// -------------------------------------------------------------- stencils --
// Reference-cube Q1 matrices on [-1,1]^3 (vertex v has coordinates bits
// (x=bit0, y=bit1, z=bit2)), 3-point Gauss per axis (exact for these
// integrands).  The reference's tables (Stencils/{Lap,Mass,GD}Type2Stencils.inp,
// loaded by examples/src/backend/handleType2Stencils.C:449-470,912-960) equal
// T^T K T with T the hanging-vertex interpolation of (childNum, mask).
struct RefMats {
  double K[8][8], M[8][8], G[24][24];
  RefMats() {
    const double gp[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)};
    const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    std::memset(K, 0, sizeof K);
    std::memset(M, 0, sizeof M);
    std::memset(G, 0, sizeof G);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c) {
          double xi[3] = {gp[a], gp[b], gp[c]}, w = gw[a] * gw[b] * gw[c];
          double N[8], dN[8][3];
          for (int v = 0; v < 8; ++v) {
            double f[3], s[3];
            for (int d = 0; d < 3; ++d) {
              s[d] = ((v >> d) & 1) ? 1.0 : -1.0;
              f[d] = 0.5 * (1 + s[d] * xi[d]);
            }
            N[v] = f[0] * f[1] * f[2];
            dN[v][0] = 0.5 * s[0] * f[1] * f[2];
            dN[v][1] = 0.5 * s[1] * f[0] * f[2];
            dN[v][2] = 0.5 * s[2] * f[0] * f[1];
          }
          for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) {
              K[i][j] += w * (dN[i][0] * dN[j][0] + dN[i][1] * dN[j][1] + dN[i][2] * dN[j][2]);
              M[i][j] += w * N[i] * N[j];
              for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q) G[3 * i + p][3 * j + q] += w * dN[i][p] * dN[j][q];
            }
        }
  }
};
const RefMats& refmats() {
  static RefMats R;
  return R;
}

// Hanging interpolation: vertex value = T * node values.  A hanging vertex v
// of child c sits at the midpoint of the parent's edge/face between parent
// vertex v and the child's shared corner; it averages the 2 or 4 parent
// vertices that differ from v only on the axes where bits of v and c differ.
void hanging_T(uint32_t c, uint32_t mask, double T[8][8]) {
  std::memset(T, 0, sizeof(double) * 64);
  for (uint32_t i = 0; i < 8; ++i) {
    if (!((mask >> i) & 1u)) {
      T[i][i] = 1.0;
      continue;
    }
    uint32_t mid = (i ^ c) & 7u;
    int cnt = 1 << __builtin_popcount(mid);
    for (uint32_t j = 0; j < 8; ++j)
      if ((((j ^ i) & ~mid) & 7u) == 0) T[i][j] = 1.0 / cnt;
  }
}

struct Tables {
  double L[8][18][8][8], Ms[8][18][8][8], GD[8][18][24][24];
  double Rhs[8][18][8];  // T^T 1: the shape functions' integrals on the reference cube per node slot
  Tables() {
    const RefMats& R = refmats();
    for (uint32_t c = 0; c < 8; ++c)
      for (int t = 0; t < 18; ++t) {
        double T[8][8];
        hanging_T(c, kEtypeMask[c][t], T);
        for (int i = 0; i < 8; ++i) {
          double r = 0;
          for (int a = 0; a < 8; ++a) r += T[a][i];
          Rhs[c][t][i] = r;
        }
        for (int i = 0; i < 8; ++i)
          for (int j = 0; j < 8; ++j) {
            double l = 0, m = 0;
            for (int a = 0; a < 8; ++a)
              for (int b = 0; b < 8; ++b) {
                l += T[a][i] * R.K[a][b] * T[b][j];
                m += T[a][i] * R.M[a][b] * T[b][j];
              }
            L[c][t][i][j] = l;
            Ms[c][t][i][j] = m;
          }
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            double g = 0;
            for (int a = 0; a < 8; ++a)
              for (int b = 0; b < 8; ++b) g += T[a][i / 3] * R.G[3 * a + i % 3][3 * b + j % 3] * T[b][j / 3];
            GD[c][t][i][j] = g;
          }
      }
  }
};
Tables* g_tables = nullptr;
const Tables& tables() {
  if (!g_tables) g_tables = new Tables();
  return *g_tables;
}

// Type-1 tables (LapType1Stencils.inp / MassType1Stencils.inp, loaded by
// createLmatType1 / createMmatType1, examples/src/backend/handleType1Stencils.C:
// [coarse child number][element type][fine child][8][8]): the stiffness and mass
// of fine child f of a coarse element in the coarse element's vertex basis,
// T^T P_f^T (K/2) P_f T and T^T P_f^T (M/8) P_f T, with P_f the trilinear
// interpolation from the coarse vertices to child f's vertices and the
// factors 1/2, 1/8 the child's h/2 and h^3/8 against the coarse ones.
struct Tables1 {
  double L[8][18][8][8][8], Ms[8][18][8][8][8];
  Tables1() {
    const RefMats& R = refmats();
    for (uint32_t f = 0; f < 8; ++f) {
      double P[8][8];  // child vertex v <- coarse vertex w
      for (int v = 0; v < 8; ++v)
        for (int w = 0; w < 8; ++w) {
          double p = 1.0;
          for (int d = 0; d < 3; ++d) {
            const double s = 0.5 * (((f >> d) & 1) + ((v >> d) & 1));  // coordinate in [0, 1]
            p *= ((w >> d) & 1) ? s : 1.0 - s;
          }
          P[v][w] = p;
        }
      double Kf[8][8], Mf[8][8];  // P^T K P / 2, P^T M P / 8
      for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
          double k = 0, m = 0;
          for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b) {
              k += P[a][i] * R.K[a][b] * P[b][j];
              m += P[a][i] * R.M[a][b] * P[b][j];
            }
          Kf[i][j] = k / 2.0;
          Mf[i][j] = m / 8.0;
        }
      for (uint32_t c = 0; c < 8; ++c)
        for (int t = 0; t < 18; ++t) {
          double T[8][8];
          hanging_T(c, kEtypeMask[c][t], T);
          for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) {
              double l = 0, m = 0;
              for (int a = 0; a < 8; ++a)
                for (int b = 0; b < 8; ++b) {
                  l += T[a][i] * Kf[a][b] * T[b][j];
                  m += T[a][i] * Mf[a][b] * T[b][j];
                }
              L[c][t][f][i][j] = l;
              Ms[c][t][f][i][j] = m;
            }
        }
    }
  }
};
Tables1* g_tables1 = nullptr;
const Tables1& tables1() {
  if (!g_tables1) g_tables1 = new Tables1();
  return *g_tables1;
}

// -------------------------------------------------------------- operators --
// JAC_TYPE2_ELEM_MULT_BLOCK / JAC_TYPE2_MULT_BLOCK (examples/src/backend/
// omgNeumann.C:468-530): y = sum_e (a_e h/2 L[c][t] + b_e h^3/8 M[c][t]) x_e,
// h = 2^-(lev-1).  coef == nullptr means a = b = 1 (odaJac.C:271-288).
// matvec_elems adds the sum over the elements listed in `elems` (all of them
// when elems is null) into y; matvec clears y first.
void matvec_elems(const Mesh& M, const double* coef, const double* x, double* y, const int64_t* elems, int64_t ne) {
  const Tables& T = tables();
  const int64_t n = elems ? ne : int64_t(M.E);
  for (int64_t i = 0; i < n; ++i) {
    const size_t e = elems ? size_t(elems[i]) : size_t(i);
    double h = std::ldexp(1.0, 1 - int(M.elev[e]));
    double a = coef ? coef[2 * e] : 1.0, b = coef ? coef[2 * e + 1] : 1.0;
    double f1 = a * h / 2.0, f2 = b * h * h * h / 8.0;
    const uint32_t* idx = &M.nlist[8 * e];
    uint32_t c = M.cnum[e], t = M.etype[e];
    for (int k = 0; k < 8; ++k)
      for (int j = 0; j < 8; ++j)
        y[idx[k]] += (f1 * T.L[c][t][k][j] + f2 * T.Ms[c][t][k][j]) * x[idx[j]];
  }
}

void matvec(const Mesh& M, const double* coef, const double* x, double* y) {
  std::fill(y, y + M.N, 0.0);
  matvec_elems(M, coef, x, y, nullptr, 0);
}

// ComputeRHS_omgNeumann (examples/src/backend/omgNeumann.C:749-785): the
// force sampled at each element's centre times RHSType2Stencil (the integral
// of each vertex's shape function on the reference cube, hanging vertices'
// shares moved to their nodes) times h^3 / 8, summed at the nodes.
void load_vector(const Mesh& M, const double* force, double* b) {
  const Tables& T = tables();
  std::fill(b, b + M.N, 0.0);
  for (size_t e = 0; e < M.E; ++e) {
    const double h = std::ldexp(1.0, 1 - int(M.elev[e]));
    const double fac = force[e] * h * h * h / 8.0;
    const uint32_t c = M.cnum[e], t = M.etype[e];
    for (int k = 0; k < 8; ++k) b[M.nlist[8 * e + k]] += T.Rhs[c][t][k] * fac;
  }
}

// JAC_TYPE2_ELEM_DIAG_BLOCK (omgNeumann.C:396-438).
void diagonal(const Mesh& M, const double* coef, double* d) {
  const Tables& T = tables();
  std::fill(d, d + M.N, 0.0);
  for (size_t e = 0; e < M.E; ++e) {
    double h = std::ldexp(1.0, 1 - int(M.elev[e]));
    double a = coef ? coef[2 * e] : 1.0, b = coef ? coef[2 * e + 1] : 1.0;
    double f1 = a * h / 2.0, f2 = b * h * h * h / 8.0;
    uint32_t c = M.cnum[e], t = M.etype[e];
    for (int k = 0; k < 8; ++k) d[M.nlist[8 * e + k]] += f1 * T.L[c][t][k][k] + f2 * T.Ms[c][t][k][k];
  }
}

// ELASTICITY_ELEM_MULT_BLOCK (examples/src/backend/elasticityJac.C:130-166):
// mu h/2 (L (x) I3) + (mu+lambda) h/2 GD; Dirichlet rows copy the input and
// Dirichlet columns are skipped.
void elasticity_matvec(const Mesh& M, double mu, double lam, const uint8_t* bdy, const double* x,
                       double* y) {
  const Tables& T = tables();
  std::fill(y, y + 3 * M.N, 0.0);
  for (size_t e = 0; e < M.E; ++e) {
    double h = std::ldexp(1.0, 1 - int(M.elev[e]));
    double fac = h / 2.0;
    const uint32_t* idx = &M.nlist[8 * e];
    uint32_t c = M.cnum[e], t = M.etype[e];
    for (int k = 0; k < 8; ++k) {
      if (bdy[idx[k]]) {
        for (int d = 0; d < 3; ++d) y[3 * idx[k] + d] = x[3 * idx[k] + d];
        continue;
      }
      for (int j = 0; j < 8; ++j) {
        if (bdy[idx[j]]) continue;
        for (int d = 0; d < 3; ++d)
          y[3 * idx[k] + d] += mu * fac * T.L[c][t][k][j] * x[3 * idx[j] + d];
        for (int p = 0; p < 3; ++p)
          for (int q = 0; q < 3; ++q)
            y[3 * idx[k] + p] += (mu + lam) * fac * T.GD[c][t][3 * k + p][3 * j + q] * x[3 * idx[j] + q];
      }
    }
  }
}

// ELASTICITY_DIAG_BLOCK (examples/src/backend/elasticityJac.C:60-100): the
// diagonal of the element tables; 1 on Dirichlet rows.
void elasticity_diagonal(const Mesh& M, double mu, double lam, const uint8_t* bdy, double* d) {
  const Tables& T = tables();
  std::fill(d, d + 3 * M.N, 0.0);
  for (size_t e = 0; e < M.E; ++e) {
    double fac = std::ldexp(1.0, 1 - int(M.elev[e])) / 2.0;
    const uint32_t* idx = &M.nlist[8 * e];
    uint32_t c = M.cnum[e], t = M.etype[e];
    for (int k = 0; k < 8; ++k) {
      if (bdy[idx[k]]) continue;
      for (int p = 0; p < 3; ++p)
        d[3 * idx[k] + p] += mu * fac * T.L[c][t][k][k] + (mu + lam) * fac * T.GD[c][t][3 * k + p][3 * k + p];
    }
  }
  for (size_t i = 0; i < M.N; ++i)
    if (bdy[i]) d[3 * i] = d[3 * i + 1] = d[3 * i + 2] = 1.0;
}

// ---------------------------------------------------------------- transfer --
// Prolongation P (fine nodes x coarse nodes): the coarse conforming FE
// function evaluated at each fine node, i.e. what prolongMatVecType1
// (src/omg/ProlongMatVec.C:154-284) computes with RmatType1/RmatType2 tables
// (RmatType2Stencil[c][t] == T^T, checked in the tests) and the
// FineTouchedStatus de-duplication (RestrictMatVec.C:410-484).
struct CSR {
  std::vector<int64_t> ptr;
  std::vector<uint32_t> col;
  std::vector<double> val;
};

int build_prolongation(const Mesh& F, const Mesh& C, CSR& P) {
  if (F.D != C.D) return -1;
  const uint32_t D = F.D, top = 1u << (D - 1);
  std::vector<uint64_t> ckeys(C.E);
  for (size_t e = 0; e < C.E; ++e) ckeys[e] = akey(C.oct[e].x, C.oct[e].y, C.oct[e].z);
  P.ptr.assign(F.N + 1, 0);
  P.col.clear();
  P.val.clear();
  for (size_t f = 0; f < F.N; ++f) {
    uint32_t px = F.node_xyz[3 * f], py = F.node_xyz[3 * f + 1], pz = F.node_xyz[3 * f + 2];
    // locate the coarse element holding the point; points on the positive
    // boundary belong to the element on their negative side
    uint32_t qx = px == top ? px - 1 : px, qy = py == top ? py - 1 : py, qz = pz == top ? pz - 1 : pz;
    int64_t e = max_lower_bound(ckeys, akey(qx, qy, qz));
    if (e < 0) return -2;
    const Oct& o = C.oct[e];
    uint32_t s = 1u << (D - o.lev());
    if (qx < o.x || qy < o.y || qz < o.z || qx >= o.x + s || qy >= o.y + s || qz >= o.z + s) return -3;
    double lx = double(px - o.x) / s, ly = double(py - o.y) / s, lz = double(pz - o.z) / s;
    double phi[8];
    for (int v = 0; v < 8; ++v)
      phi[v] = ((v & 1) ? lx : 1 - lx) * ((v & 2) ? ly : 1 - ly) * ((v & 4) ? lz : 1 - lz);
    double T[8][8];
    hanging_T(C.cnum[e], C.hmask[e], T);
    for (int j = 0; j < 8; ++j) {
      double w = 0;
      for (int v = 0; v < 8; ++v) w += phi[v] * T[v][j];
      if (w != 0.0) {
        P.col.push_back(C.nlist[8 * e + j]);
        P.val.push_back(w);
      }
    }
    P.ptr[f + 1] = int64_t(P.col.size());
  }
  return 0;
}

void prolong_add(const CSR& P, size_t nf, const double* xc, double* xf) {
  for (size_t f = 0; f < nf; ++f)
    for (int64_t k = P.ptr[f]; k < P.ptr[f + 1]; ++k) xf[f] += P.val[k] * xc[P.col[k]];
}
void restrict_(const CSR& P, size_t nf, size_t nc, const double* rf, double* rc) {
  std::fill(rc, rc + nc, 0.0);
  for (size_t f = 0; f < nf; ++f)
    for (int64_t k = P.ptr[f]; k < P.ptr[f + 1]; ++k) rc[P.col[k]] += P.val[k] * rf[f];
}
// The same transfers on dof interleaved components, each component moved by
// the scalar entries: the reference's transfer loops apply one R entry to
// every dof (RestrictMatVec.C:109-115); its elasticity driver creates the
// transfers before the suppressed-DOF arrays exist (DAMGSetUp inside
// DAMGCreateAndSetDA, omg.C:2167, copies their null pointers, omg.C:2259-2260),
// so no Dirichlet dof is suppressed.
void prolong_add_dof(const CSR& P, size_t nf, int dof, const double* xc, double* xf) {
  for (size_t f = 0; f < nf; ++f)
    for (int64_t k = P.ptr[f]; k < P.ptr[f + 1]; ++k)
      for (int d = 0; d < dof; ++d) xf[dof * f + d] += P.val[k] * xc[size_t(dof) * P.col[k] + d];
}
void restrict_dof(const CSR& P, size_t nf, size_t nc, int dof, const double* rf, double* rc) {
  std::fill(rc, rc + dof * nc, 0.0);
  for (size_t f = 0; f < nf; ++f)
    for (int64_t k = P.ptr[f]; k < P.ptr[f + 1]; ++k)
      for (int d = 0; d < dof; ++d) rc[size_t(dof) * P.col[k] + d] += P.val[k] * rf[dof * f + d];
}

// Coefficients of a coarse level (ASSIGN_MAT_PROP_FINE_TO_COARSE_ELEM_BLOCK,
// omgNeumann.C:73-113): copy when the coarse element is a fine element,
// otherwise the mean of its 8 children.
int coarse_coef(const Mesh& F, const double* fc, const Mesh& C, std::vector<double>& cc) {
  cc.assign(2 * C.E, 0.0);
  size_t f = 0;
  for (size_t e = 0; e < C.E; ++e) {
    const Oct& o = C.oct[e];
    while (f < F.E && !(F.oct[f].x == o.x && F.oct[f].y == o.y && F.oct[f].z == o.z)) ++f;
    if (f >= F.E) return -1;
    if (F.oct[f].lev() == o.lev()) {
      cc[2 * e] = fc[2 * f];
      cc[2 * e + 1] = fc[2 * f + 1];
      ++f;
    } else {
      double a = 0, b = 0;
      for (int k = 0; k < 8; ++k, ++f) {
        a += fc[2 * f];
        b += fc[2 * f + 1];
      }
      cc[2 * e] = a / 8.0;
      cc[2 * e + 1] = b / 8.0;
    }
  }
  return 0;
}

// DirichletLaplacianMatMult / DirichletJacobianMatMult and their diagonals
// (examples/src/backend/omgJac.C:859-1160): unit coefficients, h/2 L plus
// h^3/8 M when mass is set; a Dirichlet row is the identity, a Dirichlet
// column is skipped.
void dirichlet_matvec(const Mesh& M, int mass, const uint8_t* bdy, const double* x, double* y) {
  const Tables& T = tables();
  std::fill(y, y + M.N, 0.0);
  for (size_t e = 0; e < M.E; ++e) {
    const double h = std::ldexp(1.0, 1 - int(M.elev[e]));
    const double f1 = h / 2.0, f2 = mass ? h * h * h / 8.0 : 0.0;
    const uint32_t* idx = &M.nlist[8 * e];
    const uint32_t c = M.cnum[e], t = M.etype[e];
    for (int k = 0; k < 8; ++k) {
      if (bdy[idx[k]]) {
        y[idx[k]] = x[idx[k]];
        continue;
      }
      for (int j = 0; j < 8; ++j)
        if (!bdy[idx[j]]) y[idx[k]] += (f1 * T.L[c][t][k][j] + f2 * T.Ms[c][t][k][j]) * x[idx[j]];
    }
  }
}
void dirichlet_diagonal(const Mesh& M, int mass, const uint8_t* bdy, double* d) {
  const Tables& T = tables();
  std::fill(d, d + M.N, 0.0);
  for (size_t e = 0; e < M.E; ++e) {
    const double h = std::ldexp(1.0, 1 - int(M.elev[e]));
    const double f1 = h / 2.0, f2 = mass ? h * h * h / 8.0 : 0.0;
    const uint32_t* idx = &M.nlist[8 * e];
    const uint32_t c = M.cnum[e], t = M.etype[e];
    for (int k = 0; k < 8; ++k)
      d[idx[k]] = bdy[idx[k]] ? 1.0 : d[idx[k]] + f1 * T.L[c][t][k][k] + f2 * T.Ms[c][t][k][k];
  }
}

// JAC_TYPE3_MULT_BLOCK (examples/src/backend/omgJac.C:2139-2233): the
// operator of a coarse level from the next finer level's coefficients fc.
// A coarse element that is also a fine element uses its coefficients with the
// type-2 tables; one split into 8 fine children uses their mean with the
// type-2 tables when the children's a and b each vary by at most tol times
// their maximum (-tolToCoarsenMatProp, default 1e-12), else the sum over the
// children of their own a, b with the type-1 tables.
int jacobian3(const Mesh& F, const double* fc, const Mesh& C, const double* x, double* y, double tol = 1e-12) {
  const Tables& T2 = tables();
  const Tables1& T1 = tables1();
  std::fill(y, y + C.N, 0.0);
  size_t f = 0;
  for (size_t e = 0; e < C.E; ++e) {
    const Oct& o = C.oct[e];
    while (f < F.E && !(F.oct[f].x == o.x && F.oct[f].y == o.y && F.oct[f].z == o.z)) ++f;
    if (f >= F.E) return -1;
    const double h = std::ldexp(1.0, 1 - int(C.elev[e]));
    const uint32_t* idx = &C.nlist[8 * e];
    const uint32_t c = C.cnum[e], t = C.etype[e];
    double A[8][8];
    if (F.oct[f].lev() == o.lev()) {
      const double f1 = fc[2 * f] * h / 2.0, f2 = fc[2 * f + 1] * h * h * h / 8.0;
      for (int k = 0; k < 8; ++k)
        for (int j = 0; j < 8; ++j) A[k][j] = f1 * T2.L[c][t][k][j] + f2 * T2.Ms[c][t][k][j];
      ++f;
    } else {
      double p1[8], p2[8];
      for (int k = 0; k < 8; ++k, ++f) {
        p1[k] = fc[2 * f];
        p2[k] = fc[2 * f + 1];
      }
      double mx1 = p1[0], mn1 = p1[0], mx2 = p2[0], mn2 = p2[0], s1 = 0, s2 = 0;
      for (int k = 0; k < 8; ++k) {
        mx1 = std::max(mx1, p1[k]);
        mn1 = std::min(mn1, p1[k]);
        mx2 = std::max(mx2, p2[k]);
        mn2 = std::min(mn2, p2[k]);
        s1 += p1[k];
        s2 += p2[k];
      }
      if (mx1 - mn1 <= tol * mx1 && mx2 - mn2 <= tol * mx2) {
        const double f1 = s1 * h / 16.0, f2 = s2 * h * h * h / 64.0;
        for (int k = 0; k < 8; ++k)
          for (int j = 0; j < 8; ++j) A[k][j] = f1 * T2.L[c][t][k][j] + f2 * T2.Ms[c][t][k][j];
      } else {
        for (int k = 0; k < 8; ++k)
          for (int j = 0; j < 8; ++j) A[k][j] = 0.0;
        for (int q = 0; q < 8; ++q) {
          const double f1 = p1[q] * h / 2.0, f2 = p2[q] * h * h * h / 8.0;
          for (int k = 0; k < 8; ++k)
            for (int j = 0; j < 8; ++j) A[k][j] += f1 * T1.L[c][t][q][k][j] + f2 * T1.Ms[c][t][q][k][j];
        }
      }
    }
    for (int k = 0; k < 8; ++k)
      for (int j = 0; j < 8; ++j) y[idx[k]] += A[k][j] * x[idx[j]];
  }
  return 0;
}

// ------------------------------------------------------------------ solver --
// DAMGSolve with the options of bin/options:50-53,182-207: CG outer,
// multiplicative V-cycle, Richardson(omega)+Jacobi smoothing with zero initial
// guess on each level, residual by the level matvec, coarse level by a dense
// direct (Cholesky) solve of the assembled operator (BUILD_FULL_JAC_TYPE2_BLOCK,
// omgNeumann.C:560-613).  PETSc is a third-party dependency whose source is not
// vendored; this is a restatement of KSPCG + PCMG, not a copy.
struct Level {
  Mesh mesh;
  std::vector<double> coef, diag;
  CSR P;  // to this level from the next coarser one
  std::vector<double> r, b, x, t;
};

// Profile (envelope) Cholesky of a sparse SPD matrix in reverse Cuthill-McKee
// order: row i of L holds columns first[i] .. i, and the factor never fills
// outside that envelope.  Used for coarsest levels too large for the dense
// factor; PETSc's coarse LU (bin/options: -mg_coarse_pc_type lu) is a sparse
// direct solve as well, so the two agree up to rounding.
struct Envelope {
  size_t n = 0;
  std::vector<uint32_t> perm, iperm;  // perm[new] = old, iperm[old] = new
  std::vector<size_t> first, start;   // per row: first column, offset of L[i][first[i]] in val
  std::vector<double> val;
};

struct Hierarchy {
  std::vector<Level> lv;  // lv[0] finest
  int coarse_op = 0;      // 1: levels below the finest apply Jacobian3 (J); diag stays type 2 (B)
  std::vector<double> chol;  // dense Cholesky of the coarsest operator
  Envelope env;              // or its envelope Cholesky (large coarsest levels)
  size_t nc = 0;
  int dof = 1;               // 3: linear elasticity on every level, its boundary nodes Dirichlet
  double mu = 1.0, lam = 1.0;
  int nu_pre = 2, nu_post = 2;
  double omega = 2.0 / 3.0;
};

// The operator J of level l: type 2 with the level's coefficients, or with
// coarse_op 1 below the finest level Jacobian3 from the finer level's.
void level_apply(const Hierarchy& H, size_t l, const double* x, double* y) {
  const Level& L = H.lv[l];
  if (H.dof == 3) {
    elasticity_matvec(L.mesh, H.mu, H.lam, L.mesh.node_bdy.data(), x, y);
    return;
  }
  if (H.coarse_op == 1 && l > 0 && !H.lv[l - 1].coef.empty()) {
    jacobian3(H.lv[l - 1].mesh, H.lv[l - 1].coef.data(), L.mesh, x, y);
    return;
  }
  matvec(L.mesh, L.coef.empty() ? nullptr : L.coef.data(), x, y);
}

// Node adjacency of a mesh: two nodes are coupled when an element lists both
// (a hanging vertex's interpolation nodes are among its element's 8 listed
// nodes, so the element couples exactly its listed nodes).
std::vector<std::vector<uint32_t>> node_graph(const Mesh& M, int dof = 1) {
  std::vector<std::vector<uint32_t>> adj(M.N * dof);
  for (size_t e = 0; e < M.E; ++e)
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b)
        for (int p = 0; p < dof; ++p)
          for (int q = 0; q < dof; ++q)
            adj[size_t(dof) * M.nlist[8 * e + a] + p].push_back(uint32_t(dof * M.nlist[8 * e + b] + q));
  for (auto& v : adj) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  return adj;
}

// Reverse Cuthill-McKee order, component by component, each started from a
// pseudo-peripheral node (the last node reached by a BFS from a minimum-degree
// node).
std::vector<uint32_t> rcm_order(const std::vector<std::vector<uint32_t>>& adj) {
  const size_t n = adj.size();
  std::vector<uint32_t> order;
  order.reserve(n);
  std::vector<char> seen(n, 0);
  std::vector<uint32_t> queue;
  auto bfs = [&](uint32_t s, std::vector<char>& mark, std::vector<uint32_t>& out) {
    out.clear();
    out.push_back(s);
    mark[s] = 1;
    for (size_t h = 0; h < out.size(); ++h) {
      const uint32_t u = out[h];
      std::vector<uint32_t> nb;
      for (uint32_t w : adj[u])
        if (!mark[w]) {
          mark[w] = 1;
          nb.push_back(w);
        }
      std::sort(nb.begin(), nb.end(), [&](uint32_t a, uint32_t b) {
        return adj[a].size() != adj[b].size() ? adj[a].size() < adj[b].size() : a < b;
      });
      out.insert(out.end(), nb.begin(), nb.end());
    }
  };
  for (size_t s0 = 0; s0 < n; ++s0) {
    if (seen[s0]) continue;
    // the component of s0 and its minimum-degree node
    std::vector<char> mark(seen);
    bfs(uint32_t(s0), mark, queue);
    uint32_t start = queue[0];
    for (uint32_t u : queue)
      if (adj[u].size() < adj[start].size()) start = u;
    mark = seen;
    bfs(start, mark, queue);
    start = queue.back();
    mark = seen;
    bfs(start, mark, queue);
    for (uint32_t u : queue) seen[u] = 1;
    order.insert(order.end(), queue.begin(), queue.end());
  }
  std::reverse(order.begin(), order.end());
  return order;
}

// Assemble the coarsest operator by probing (columns of one colour of a
// distance-2 colouring share one product with the level operator) into the
// envelope of its RCM order, then factor in place.
int envelope_factor(Hierarchy& H) {
  const size_t l = H.lv.size() - 1;
  const Mesh& M = H.lv[l].mesh;
  const size_t n = M.N * H.dof;
  Envelope& V = H.env;
  std::vector<std::vector<uint32_t>> adj = node_graph(M, H.dof);
  V.n = n;
  V.perm = rcm_order(adj);
  V.iperm.assign(n, 0);
  for (size_t i = 0; i < n; ++i) V.iperm[V.perm[i]] = uint32_t(i);
  V.first.assign(n, 0);
  V.start.assign(n + 1, 0);
  for (size_t i = 0; i < n; ++i) {
    size_t f = i;
    for (uint32_t w : adj[V.perm[i]]) f = std::min<size_t>(f, V.iperm[w]);
    V.first[i] = f;
    V.start[i + 1] = V.start[i] + (i - f + 1);
  }
  V.val.assign(V.start[n], 0.0);
  // distance-2 colouring, greedy in node order
  std::vector<int> colour(n, -1);
  int ncol = 0;
  std::vector<int> used;
  for (size_t j = 0; j < n; ++j) {
    used.clear();
    for (uint32_t i : adj[j])
      for (uint32_t k : adj[i])
        if (colour[k] >= 0) used.push_back(colour[k]);
    std::sort(used.begin(), used.end());
    int c = 0;
    for (int u : used) {
      if (u == c) ++c;
      else if (u > c) break;
    }
    colour[j] = c;
    ncol = std::max(ncol, c + 1);
  }
  std::vector<double> e(n), y(n);
  for (int c = 0; c < ncol; ++c) {
    for (size_t j = 0; j < n; ++j) e[j] = colour[j] == c ? 1.0 : 0.0;
    level_apply(H, l, e.data(), y.data());
    for (size_t j = 0; j < n; ++j) {
      if (colour[j] != c) continue;
      const size_t pj = V.iperm[j];
      for (uint32_t i : adj[j]) {  // column j: A[i][j] = y[i]
        const size_t pi = V.iperm[i];
        if (pj <= pi) V.val[V.start[pi] + (pj - V.first[pi])] = y[i];
      }
    }
  }
  // row-oriented Cholesky inside the envelope
  for (size_t i = 0; i < n; ++i) {
    double* Li = &V.val[V.start[i]] - V.first[i];  // Li[k], k in [first[i], i]
    for (size_t j = V.first[i]; j < i; ++j) {
      const double* Lj = &V.val[V.start[j]] - V.first[j];
      double t = Li[j];
      for (size_t k = std::max(V.first[i], V.first[j]); k < j; ++k) t -= Li[k] * Lj[k];
      Li[j] = t / Lj[j];
    }
    double d = Li[i];
    for (size_t k = V.first[i]; k < i; ++k) d -= Li[k] * Li[k];
    if (!(d > 0)) return -1;
    Li[i] = std::sqrt(d);
  }
  return 0;
}

void envelope_solve(const Envelope& V, const double* b, double* x) {
  const size_t n = V.n;
  std::vector<double> w(n);
  for (size_t i = 0; i < n; ++i) w[i] = b[V.perm[i]];
  for (size_t i = 0; i < n; ++i) {  // L w' = w
    const double* Li = &V.val[V.start[i]] - V.first[i];
    double t = w[i];
    for (size_t k = V.first[i]; k < i; ++k) t -= Li[k] * w[k];
    w[i] = t / Li[i];
  }
  for (size_t i = n; i-- > 0;) {  // L^T x = w', column by column
    const double* Li = &V.val[V.start[i]] - V.first[i];
    w[i] /= Li[i];
    for (size_t k = V.first[i]; k < i; ++k) w[k] -= Li[k] * w[i];
  }
  for (size_t i = 0; i < n; ++i) x[V.perm[i]] = w[i];
}

// Coarsest levels above this many nodes use the envelope factor.
constexpr size_t kDenseCoarseMax = 4096;

int assemble_and_factor(Hierarchy& H) {
  Level& L = H.lv.back();
  size_t n = L.mesh.N * H.dof;
  H.nc = n;
  H.env = Envelope();
  H.chol.clear();
  if (n > kDenseCoarseMax) return envelope_factor(H);
  H.chol.assign(n * n, 0.0);
  std::vector<double> e(n, 0.0), col(n);
  for (size_t j = 0; j < n; ++j) {
    e[j] = 1.0;
    level_apply(H, H.lv.size() - 1, e.data(), col.data());
    e[j] = 0.0;
    for (size_t i = 0; i < n; ++i) H.chol[i * n + j] = col[i];
  }
  double* A = H.chol.data();
  for (size_t j = 0; j < n; ++j) {
    double s = A[j * n + j];
    for (size_t k = 0; k < j; ++k) s -= A[j * n + k] * A[j * n + k];
    if (!(s > 0)) return -1;
    double d = std::sqrt(s);
    A[j * n + j] = d;
    for (size_t i = j + 1; i < n; ++i) {
      double t = A[i * n + j];
      for (size_t k = 0; k < j; ++k) t -= A[i * n + k] * A[j * n + k];
      A[i * n + j] = t / d;
    }
  }
  return 0;
}

void chol_solve(const Hierarchy& H, const double* b, double* x) {
  if (H.env.n) {
    envelope_solve(H.env, b, x);
    return;
  }
  size_t n = H.nc;
  const double* A = H.chol.data();
  for (size_t i = 0; i < n; ++i) {
    double t = b[i];
    for (size_t k = 0; k < i; ++k) t -= A[i * n + k] * x[k];
    x[i] = t / A[i * n + i];
  }
  for (size_t ii = n; ii-- > 0;) {
    double t = x[ii];
    for (size_t k = ii + 1; k < n; ++k) t -= A[k * n + ii] * x[k];
    x[ii] = t / A[ii * n + ii];
  }
}

void vcycle(Hierarchy& H, size_t l, const double* b, double* x) {
  Level& L = H.lv[l];
  size_t n = L.mesh.N * H.dof;
  if (l + 1 == H.lv.size()) {
    chol_solve(H, b, x);
    return;
  }
  std::fill(x, x + n, 0.0);
  for (int s = 0; s < H.nu_pre; ++s) {
    level_apply(H, l, x, L.t.data());
    for (size_t i = 0; i < n; ++i) x[i] += H.omega * (b[i] - L.t[i]) / L.diag[i];
  }
  level_apply(H, l, x, L.t.data());
  for (size_t i = 0; i < n; ++i) L.r[i] = b[i] - L.t[i];
  Level& C = H.lv[l + 1];
  restrict_dof(L.P, L.mesh.N, C.mesh.N, H.dof, L.r.data(), C.b.data());
  vcycle(H, l + 1, C.b.data(), C.x.data());
  prolong_add_dof(L.P, L.mesh.N, H.dof, C.x.data(), x);
  for (int s = 0; s < H.nu_post; ++s) {
    level_apply(H, l, x, L.t.data());
    for (size_t i = 0; i < n; ++i) x[i] += H.omega * (b[i] - L.t[i]) / L.diag[i];
  }
}

double dot(const double* a, const double* b, size_t n) {
  double s = 0;
  for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

}  // namespace

// =================================================================== C ABI ==
extern "C" {

struct orc_octant {
  uint32_t x, y, z, level_flags;
};

void orc_free(void* p) { std::free(p); }

static orc_octant* to_c(const std::vector<Oct>& v) {
  orc_octant* o = (orc_octant*)std::malloc(sizeof(orc_octant) * (v.size() ? v.size() : 1));
  for (size_t i = 0; i < v.size(); ++i) o[i] = {v[i].x, v[i].y, v[i].z, v[i].lf};
  return o;
}
static std::vector<Oct> from_c(const orc_octant* p, int64_t n) {
  std::vector<Oct> v(size_t(n > 0 ? n : 0));
  for (int64_t i = 0; i < n; ++i) v[i] = Oct{p[i].x, p[i].y, p[i].z, p[i].level_flags};
  return v;
}

int orc_points2octree(const double* pts, int64_t n, uint32_t maxDepth, uint32_t maxNumPts,
                      orc_octant** out, int64_t* nout) {
  if (maxDepth > 20) return -1;
  std::vector<Oct> v = points2octree(pts, size_t(n), maxDepth, maxNumPts);
  *out = to_c(v);
  *nout = int64_t(v.size());
  return 0;
}

int orc_balance(const orc_octant* in, int64_t n, uint32_t maxDepth, orc_octant** out, int64_t* nout) {
  std::vector<Oct> v = balance(from_c(in, n), maxDepth);
  *out = to_c(v);
  *nout = int64_t(v.size());
  return 0;
}

int orc_coarsen(const orc_octant* in, int64_t n, uint32_t maxDepth, orc_octant** out, int64_t* nout) {
  std::vector<Oct> v = coarsen(from_c(in, n), maxDepth);
  *out = to_c(v);
  *nout = int64_t(v.size());
  return 0;
}

int orc_is_sorted_linear(const orc_octant* in, int64_t n) {
  std::vector<Oct> v = from_c(in, n);
  for (size_t i = 1; i < v.size(); ++i)
    if (!morton_less(v[i - 1], v[i])) return 0;
  return 1;
}

void* orc_mesh_create(const orc_octant* tree, int64_t n, uint32_t maxDepth, int* status) {
  Mesh* M = new Mesh();
  int s = build_mesh(from_c(tree, n), maxDepth, *M);
  *status = s;
  if (s) {
    delete M;
    return nullptr;
  }
  return M;
}
void orc_mesh_destroy(void* m) { delete (Mesh*)m; }
void orc_mesh_sizes(void* m, int64_t* E, int64_t* N, int64_t* nOct) {
  Mesh* M = (Mesh*)m;
  *E = int64_t(M->E);
  *N = int64_t(M->N);
  *nOct = int64_t(M->oct.size());
}
void orc_mesh_export(void* m, uint32_t* nlist, uint8_t* hmask, uint8_t* cnum, uint8_t* etype,
                     uint8_t* elev, uint32_t* node_xyz, uint8_t* node_bdy, orc_octant* octs) {
  Mesh* M = (Mesh*)m;
  if (nlist) std::memcpy(nlist, M->nlist.data(), 4 * M->nlist.size());
  if (hmask) std::memcpy(hmask, M->hmask.data(), M->E);
  if (cnum) std::memcpy(cnum, M->cnum.data(), M->E);
  if (etype) std::memcpy(etype, M->etype.data(), M->E);
  if (elev) std::memcpy(elev, M->elev.data(), M->E);
  if (node_xyz) std::memcpy(node_xyz, M->node_xyz.data(), 4 * M->node_xyz.size());
  if (node_bdy) std::memcpy(node_bdy, M->node_bdy.data(), M->N);
  if (octs)
    for (size_t i = 0; i < M->oct.size(); ++i)
      octs[i] = {M->oct[i].x, M->oct[i].y, M->oct[i].z, M->oct[i].lf};
}

void orc_matvec(void* m, const double* coef, const double* x, double* y) {
  matvec(*(Mesh*)m, coef, x, y);
}
void orc_matvec_elems(void* m, const double* coef, const double* x, double* y, const int64_t* elems, int64_t n) {
  matvec_elems(*(Mesh*)m, coef, x, y, elems, n);
}
void orc_diagonal(void* m, const double* coef, double* d) { diagonal(*(Mesh*)m, coef, d); }
void orc_load_vector(void* m, const double* force, double* b) { load_vector(*(Mesh*)m, force, b); }
// RHSType2Stencil as derived here, [8][18][8].
void orc_rhs_table(double* R) { std::memcpy(R, tables().Rhs, sizeof(tables().Rhs)); }
void orc_elasticity_matvec(void* m, double mu, double lam, const uint8_t* bdy, const double* x, double* y) {
  elasticity_matvec(*(Mesh*)m, mu, lam, bdy, x, y);
}

// Stencil tables, [8][18][8][8] (L, M) and [8][18][24][24] (GD).
void orc_stencils(double* L, double* Mm, double* GD) {
  const Tables& T = tables();
  if (L) std::memcpy(L, T.L, sizeof T.L);
  if (Mm) std::memcpy(Mm, T.Ms, sizeof T.Ms);
  if (GD) std::memcpy(GD, T.GD, sizeof T.GD);
}
void orc_hanging_T(uint32_t c, uint32_t mask, double* T) { hanging_T(c, mask, (double(*)[8])T); }

int orc_prolongation(void* fine, void* coarse, int64_t** ptr, uint32_t** col, double** val, int64_t* nnz) {
  CSR P;
  int s = build_prolongation(*(Mesh*)fine, *(Mesh*)coarse, P);
  if (s) return s;
  *nnz = int64_t(P.col.size());
  *ptr = (int64_t*)std::malloc(8 * P.ptr.size());
  std::memcpy(*ptr, P.ptr.data(), 8 * P.ptr.size());
  *col = (uint32_t*)std::malloc(4 * (P.col.size() + 1));
  std::memcpy(*col, P.col.data(), 4 * P.col.size());
  *val = (double*)std::malloc(8 * (P.val.size() + 1));
  std::memcpy(*val, P.val.data(), 8 * P.val.size());
  return 0;
}

int orc_coarse_coef(void* fine, const double* fc, void* coarse, double* cc) {
  std::vector<double> v;
  int s = coarse_coef(*(Mesh*)fine, fc, *(Mesh*)coarse, v);
  if (s) return s;
  std::memcpy(cc, v.data(), 8 * v.size());
  return 0;
}

// Build the multigrid hierarchy (DAMGCreateAndSetDA, src/omg/omg.C:1306-1420):
// coarsen + balance per level until nlevels or a level below 500 octants.
// coef_mode 0: a = b = 1; 1: per-element coefficients given for the finest.
void* orc_damg_create_dof(const orc_octant* finest, int64_t n, uint32_t maxDepth, int nlevels,
                          const double* coef, int dof, double mu, double lam, int* status, int* levels_out);
void* orc_damg_create(const orc_octant* finest, int64_t n, uint32_t maxDepth, int nlevels,
                      const double* coef, int* status, int* levels_out) {
  return orc_damg_create_dof(finest, n, maxDepth, nlevels, coef, 1, 1.0, 1.0, status, levels_out);
}
// dof 3: ElasticityMatMult on every level with that level's boundary nodes
// Dirichlet (SetElasticityContexts, examples/src/backend/elasticityJac.C:396-480).
void* orc_damg_create_dof(const orc_octant* finest, int64_t n, uint32_t maxDepth, int nlevels,
                          const double* coef, int dof, double mu, double lam, int* status, int* levels_out) {
  Hierarchy* H = new Hierarchy();
  H->dof = dof;
  H->mu = mu;
  H->lam = lam;
  std::vector<std::vector<Oct>> trees;
  trees.push_back(from_c(finest, n));
  int idx = -1;
  bool repeat = nlevels > 1;
  while (idx < nlevels - 2 && repeat) {
    std::vector<Oct> c = balance(coarsen(trees.back(), maxDepth), maxDepth);
    ++idx;
    trees.push_back(c);
    if (c.size() < 500) repeat = false;
  }
  H->lv.resize(trees.size());
  for (size_t l = 0; l < trees.size(); ++l) {
    int s = build_mesh(trees[l], maxDepth, H->lv[l].mesh);
    if (s) {
      *status = s;
      delete H;
      return nullptr;
    }
  }
  if (coef) {
    H->lv[0].coef.assign(coef, coef + 2 * H->lv[0].mesh.E);
    for (size_t l = 1; l < H->lv.size(); ++l)
      coarse_coef(H->lv[l - 1].mesh, H->lv[l - 1].coef.data(), H->lv[l].mesh, H->lv[l].coef);
  }
  for (size_t l = 0; l < H->lv.size(); ++l) {
    Level& L = H->lv[l];
    size_t N = L.mesh.N * dof;
    L.diag.resize(N);
    if (dof == 3)
      elasticity_diagonal(L.mesh, mu, lam, L.mesh.node_bdy.data(), L.diag.data());
    else
      diagonal(L.mesh, L.coef.empty() ? nullptr : L.coef.data(), L.diag.data());
    L.r.assign(N, 0);
    L.b.assign(N, 0);
    L.x.assign(N, 0);
    L.t.assign(N, 0);
    if (l + 1 < H->lv.size()) {
      int s = build_prolongation(L.mesh, H->lv[l + 1].mesh, L.P);
      if (s) {
        *status = s;
        delete H;
        return nullptr;
      }
    }
  }
  if (assemble_and_factor(*H)) {
    *status = -10;
    delete H;
    return nullptr;
  }
  *status = 0;
  *levels_out = int(H->lv.size());
  return H;
}
void orc_damg_destroy(void* h) { delete (Hierarchy*)h; }
// coarse_op 1: Jacobian3 below the finest level (the coarsest is re-factored)
int orc_damg_set_coarse_op(void* h, int op) {
  Hierarchy* H = (Hierarchy*)h;
  H->coarse_op = op;
  return assemble_and_factor(*H);
}
void orc_damg_level_apply(void* h, int l, const double* x, double* y) { level_apply(*(Hierarchy*)h, l, x, y); }
void orc_type1_stencils(double* L, double* M) {
  const Tables1& T = tables1();
  std::memcpy(L, T.L, sizeof T.L);
  std::memcpy(M, T.Ms, sizeof T.Ms);
}
void orc_dirichlet_matvec(void* m, int mass, const uint8_t* bdy, const double* x, double* y) {
  dirichlet_matvec(*(Mesh*)m, mass, bdy, x, y);
}
void orc_dirichlet_diagonal(void* m, int mass, const uint8_t* bdy, double* d) {
  dirichlet_diagonal(*(Mesh*)m, mass, bdy, d);
}
int orc_jacobian3(void* fine, const double* fc, void* coarse, const double* x, double* y) {
  return jacobian3(*(Mesh*)fine, fc, *(Mesh*)coarse, x, y);
}
void orc_damg_level_sizes(void* h, int64_t* E, int64_t* N) {
  Hierarchy* H = (Hierarchy*)h;
  for (size_t l = 0; l < H->lv.size(); ++l) {
    E[l] = int64_t(H->lv[l].mesh.E);
    N[l] = int64_t(H->lv[l].mesh.N);
  }
}
void* orc_damg_level_mesh(void* h, int l) { return &((Hierarchy*)h)->lv[l].mesh; }
void orc_damg_vcycle(void* h, const double* b, double* x) {
  Hierarchy* H = (Hierarchy*)h;
  vcycle(*H, 0, b, x);
}

// Preconditioned CG to ||b - A x||_2 <= rtol ||b||_2, zero initial guess.
// Returns the iteration count; history[i] = relative true residual after i.
int orc_damg_pcg(void* h, const double* b, double* x, double rtol, int maxit, double* history) {
  Hierarchy* H = (Hierarchy*)h;
  Level& L = H->lv[0];
  size_t n = L.mesh.N * H->dof;
  std::vector<double> r(b, b + n), z(n), p(n), q(n);
  std::fill(x, x + n, 0.0);
  double bn = std::sqrt(dot(b, b, n));
  if (bn == 0) return 0;
  if (history) history[0] = 1.0;
  vcycle(*H, 0, r.data(), z.data());
  p = z;
  double rz = dot(r.data(), z.data(), n);
  for (int it = 1; it <= maxit; ++it) {
    level_apply(*H, 0, p.data(), q.data());
    double alpha = rz / dot(p.data(), q.data(), n);
    for (size_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    double rel = std::sqrt(dot(r.data(), r.data(), n)) / bn;
    if (history) history[it] = rel;
    if (rel <= rtol) return it;
    vcycle(*H, 0, r.data(), z.data());
    double rz2 = dot(r.data(), z.data(), n);
    double beta = rz2 / rz;
    rz = rz2;
    for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  return -maxit;
}

}  // extern "C"
