// File formats of the reference's drivers, written and read on the host:
//   * point files (.pts): uint32 count, then 3 count FP64 coordinates
//     (readPtsFromFile / writePtsToFile, src/oct/OctFunctions.C:313-341,
//     370-385); with values attached: the count, the coordinates, then
//     count FP64 values (readDataPtsFromFile / writeDataPtsToFile,
//     OctFunctions.C:343-368, 387-401);
//   * octree files (.ot): text "dim maxDepth", the count, then one line
//     "x y z level" per octant (readNodesFromFile / writeNodesToFile,
//     OctFunctions.C:403-439);
//   * the single-rank mesh dump of examples/src/drivers/dumpMesh.C: files
//     <prefix>_NL_0_1.out (node count; per node, in order of first visit over
//     the elements, its anchor x y z as uint32 and its global id), _EL_0_1.out
//     (maxDepth and element count; per element x y z, level - 1 and global id)
//     and _M_0_1.out (element count; per element its id and its 8 node ids),
//     all integers 4 bytes (DendroIntL of the 32-bit build, include/dendro.h).
// None of these touches the GPU except through dg_octree / dg_da exports.
#include <cstdio>
#include <string>
#include <vector>

#include "dg_internal.h"

using namespace dg;

namespace {

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) : f(fopen(path, mode)) {}
  ~File() {
    if (f) fclose(f);
  }
};

dg_status io_error(const char* what, const char* path) {
  set_error(__FILE__, __LINE__, std::string(what) + ": " + path);
  return DG_EINVAL;
}

}  // namespace

extern "C" {

dg_status dg_write_pts(const char* path, const double* pts, int64_t n) {
  DG_CHECK(path && n >= 0 && (n == 0 || pts) && n <= 0xffffffffll, DG_EINVAL, "write_pts: bad arguments");
  File out(path, "wb");
  if (!out.f) return io_error("write_pts: cannot open", path);
  if (n > 0) {  // like the reference, no header at all for no points
    const uint32_t c = uint32_t(n);
    if (fwrite(&c, 4, 1, out.f) != 1 || fwrite(pts, 8, size_t(3 * n), out.f) != size_t(3 * n))
      return io_error("write_pts: write failed", path);
  }
  return DG_OK;
}

dg_status dg_read_pts(const char* path, double* pts, int64_t capacity, int64_t* n) {
  DG_CHECK(path && n, DG_EINVAL, "read_pts: bad arguments");
  File in(path, "rb");
  if (!in.f) return io_error("read_pts: cannot open", path);
  uint32_t c = 0;
  if (fread(&c, 4, 1, in.f) != 1) c = 0;  // an empty file holds no points
  *n = c;
  if (!pts) return DG_OK;  // size query
  DG_CHECK(capacity >= int64_t(c), DG_EINVAL, "read_pts: buffer smaller than the point count");
  if (c && fread(pts, 8, size_t(3) * c, in.f) != size_t(3) * c) return io_error("read_pts: file truncated", path);
  return DG_OK;
}

dg_status dg_write_data_pts(const char* path, const double* pts, const double* vals, int64_t n) {
  DG_CHECK(path && n >= 0 && (n == 0 || (pts && vals)) && n <= 0xffffffffll, DG_EINVAL,
           "write_data_pts: bad arguments");
  File out(path, "wb");
  if (!out.f) return io_error("write_data_pts: cannot open", path);
  const uint32_t c = uint32_t(n);
  if (fwrite(&c, 4, 1, out.f) != 1 || (n && fwrite(pts, 8, size_t(3 * n), out.f) != size_t(3 * n)) ||
      (n && fwrite(vals, 8, size_t(n), out.f) != size_t(n)))
    return io_error("write_data_pts: write failed", path);
  return DG_OK;
}

dg_status dg_read_data_pts(const char* path, double* pts, double* vals, int64_t capacity, int64_t* n) {
  DG_CHECK(path && n, DG_EINVAL, "read_data_pts: bad arguments");
  File in(path, "rb");
  if (!in.f) return io_error("read_data_pts: cannot open", path);
  uint32_t c = 0;
  if (fread(&c, 4, 1, in.f) != 1) return io_error("read_data_pts: no header", path);
  *n = c;
  if (!pts && !vals) return DG_OK;
  DG_CHECK(pts && vals && capacity >= int64_t(c), DG_EINVAL, "read_data_pts: buffers smaller than the point count");
  if (c && (fread(pts, 8, size_t(3) * c, in.f) != size_t(3) * c || fread(vals, 8, c, in.f) != c))
    return io_error("read_data_pts: file truncated", path);
  return DG_OK;
}

dg_status dg_octree_write(const dg_octree* t, const char* path) {
  DG_CHECK(t && path, DG_EINVAL, "octree_write: bad arguments");
  std::vector<dg_octant> o(size_t(t->n));
  if (t->n) DG_TRY(dg_octree_export(t, o.data()));
  File out(path, "w");
  if (!out.f) return io_error("octree_write: cannot open", path);
  if (!o.empty()) {  // like the reference, an empty file for no octants
    fprintf(out.f, "%u %u\n", 3u, t->max_depth);
    fprintf(out.f, "%u\n", static_cast<unsigned>(o.size()));
    for (const dg_octant& q : o) fprintf(out.f, "%u %u %u %u\n", q.x, q.y, q.z, q.level_flags & 31u);
  }
  if (ferror(out.f)) return io_error("octree_write: write failed", path);
  return DG_OK;
}

dg_status dg_octree_read(const char* path, dg_octree** out) {
  DG_CHECK(path && out, DG_EINVAL, "octree_read: bad arguments");
  File in(path, "r");
  if (!in.f) return io_error("octree_read: cannot open", path);
  unsigned dim = 0, depth = 0, n = 0;
  if (fscanf(in.f, "%u %u %u", &dim, &depth, &n) != 3) return io_error("octree_read: no header", path);
  DG_CHECK(dim == 3, DG_EINVAL, "octree_read: only three-dimensional octrees");
  DG_CHECK(n > 0, DG_EINVAL, "octree_read: no octants");
  std::vector<dg_octant> o(n);
  for (unsigned i = 0; i < n; ++i) {
    unsigned x, y, z, l;
    if (fscanf(in.f, "%u %u %u %u", &x, &y, &z, &l) != 4) return io_error("octree_read: file truncated", path);
    o[i] = dg_octant{x, y, z, l};
  }
  return dg_octree_from_octants(o.data(), n, 0, depth, out);
}

dg_status dg_da_dump_mesh(const dg_da* da, const char* prefix) {
  DG_CHECK(da && prefix, DG_EINVAL, "da_dump_mesh: bad arguments");
  int64_t E = 0, N = 0, P = 0;
  DG_TRY(dg_da_sizes(da, &E, &N, &P));
  DG_CHECK(E <= 0x7fffffffll && N <= 0x7fffffffll, DG_EINVAL, "da_dump_mesh: ids do not fit 32-bit DendroIntL");
  std::vector<uint32_t> nl(size_t(E) * 8), nxyz(size_t(N) * 3), exyz(size_t(E) * 3);
  std::vector<uint8_t> lev(static_cast<size_t>(E));
  DG_TRY(dg_da_export(da, nl.data(), nullptr, nullptr, nullptr, lev.data(), nxyz.data(), exyz.data(), nullptr));
  const std::string p(prefix);
  {  // nodes in order of first visit over the elements and their vertices
    File out((p + "_NL_0_1.out").c_str(), "wb");
    if (!out.f) return io_error("da_dump_mesh: cannot open", (p + "_NL_0_1.out").c_str());
    const uint32_t nn = uint32_t(N);
    fwrite(&nn, 4, 1, out.f);
    std::vector<char> seen(size_t(N), 0);
    std::vector<uint32_t> rec;
    rec.reserve(size_t(N) * 4);
    for (int64_t e = 0; e < E; ++e)
      for (int j = 0; j < 8; ++j) {
        const uint32_t id = nl[size_t(e) * 8 + j];
        DG_CHECK(id < uint64_t(N), DG_EINVAL, "da_dump_mesh: node id out of range");
        if (seen[id]) continue;
        seen[id] = 1;
        rec.insert(rec.end(), {nxyz[3 * size_t(id)], nxyz[3 * size_t(id) + 1], nxyz[3 * size_t(id) + 2], id});
      }
    DG_CHECK(rec.size() == size_t(N) * 4, DG_EINVAL, "da_dump_mesh: a node belongs to no element");
    if (fwrite(rec.data(), 4, rec.size(), out.f) != rec.size())
      return io_error("da_dump_mesh: write failed", (p + "_NL_0_1.out").c_str());
  }
  {  // elements: anchor, level - 1 (the octree's own level), id
    File out((p + "_EL_0_1.out").c_str(), "wb");
    if (!out.f) return io_error("da_dump_mesh: cannot open", (p + "_EL_0_1.out").c_str());
    const uint32_t hdr[2] = {dg_da_max_depth(da) - 1, uint32_t(E)};
    fwrite(hdr, 4, 2, out.f);
    std::vector<uint32_t> rec(size_t(E) * 5);
    for (int64_t e = 0; e < E; ++e) {
      uint32_t* r = &rec[size_t(e) * 5];
      r[0] = exyz[3 * size_t(e)];
      r[1] = exyz[3 * size_t(e) + 1];
      r[2] = exyz[3 * size_t(e) + 2];
      r[3] = uint32_t(lev[size_t(e)]) - 1u;
      r[4] = uint32_t(e);
    }
    if (fwrite(rec.data(), 4, rec.size(), out.f) != rec.size())
      return io_error("da_dump_mesh: write failed", (p + "_EL_0_1.out").c_str());
  }
  {  // element -> node map
    File out((p + "_M_0_1.out").c_str(), "wb");
    if (!out.f) return io_error("da_dump_mesh: cannot open", (p + "_M_0_1.out").c_str());
    const uint32_t ne = uint32_t(E);
    fwrite(&ne, 4, 1, out.f);
    std::vector<uint32_t> rec(size_t(E) * 9);
    for (int64_t e = 0; e < E; ++e) {
      rec[size_t(e) * 9] = uint32_t(e);
      for (int j = 0; j < 8; ++j) rec[size_t(e) * 9 + 1 + j] = nl[size_t(e) * 8 + j];
    }
    if (fwrite(rec.data(), 4, rec.size(), out.f) != rec.size())
      return io_error("da_dump_mesh: write failed", (p + "_M_0_1.out").c_str());
  }
  return DG_OK;
}

}  // extern "C"
