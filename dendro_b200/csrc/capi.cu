// extern "C" entry points (include/dendro_b200.h).
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "dg_internal.h"

namespace dg {

static thread_local std::string g_last_error;

void set_error(const char* file, int line, const std::string& msg) {
  const char* base = strrchr(file, '/');
  g_last_error = std::string(base ? base + 1 : file) + ":" + std::to_string(line) + ": " + msg;
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                                                   cudaSuccess || n <= 0)
      n = 148;
  }
  return n;
}

namespace {
__global__ void octants_to_keys(const dg_octant* __restrict__ o, int64_t n, uint64_t* __restrict__ k,
                                uint32_t* __restrict__ bad, uint32_t D) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t l = o[i].level_flags & kLevelMask;
    if (l > D) atomicOr(bad, 1u);
    k[i] = okey(morton(o[i].x, o[i].y, o[i].z), l);
    if (i > 0) {
      uint32_t pl = o[i - 1].level_flags & kLevelMask;
      if (okey(morton(o[i - 1].x, o[i - 1].y, o[i - 1].z), pl) >= k[i]) atomicOr(bad, 2u);
    }
  }
}
__global__ void keys_to_octants(const uint64_t* __restrict__ k, int64_t n, dg_octant* __restrict__ o, uint32_t flags) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t x, y, z;
    demorton(okey_m(k[i]), x, y, z);
    o[i] = dg_octant{x, y, z, okey_l(k[i]) | flags};
  }
}
__global__ void decode_xyz(const uint64_t* __restrict__ k, int64_t n, int is_octkey, uint32_t* __restrict__ xyz) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t x, y, z;
    demorton(is_octkey ? okey_m(k[i]) : k[i], x, y, z);
    xyz[3 * i] = x;
    xyz[3 * i + 1] = y;
    xyz[3 * i + 2] = z;
  }
}
__global__ void centers_kernel(const uint64_t* __restrict__ ek, int64_t E, uint32_t Dp, double* __restrict__ c) {
  const double inv = 1.0 / double(1u << (Dp - 1));
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < E; i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t x, y, z;
    demorton(okey_m(ek[i]), x, y, z);
    double hs = 0.5 * double(1u << (Dp - okey_l(ek[i])));
    c[3 * i] = (x + hs) * inv;
    c[3 * i + 1] = (y + hs) * inv;
    c[3 * i + 2] = (z + hs) * inv;
  }
}
__global__ void node_bdy_kernel(const uint64_t* __restrict__ nk, int64_t N, uint32_t top, uint8_t* __restrict__ b) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < N; i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t x, y, z;
    demorton(nk[i], x, y, z);
    b[i] = (x == 0 || y == 0 || z == 0 || x == top || y == top || z == top) ? 1 : 0;
  }
}
__global__ void f64_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    b[i] = float(a[i]);
}
}  // namespace

dg_status node_boundary_flags(const dg_da* da, uint8_t* d_out, cudaStream_t s) {
  node_bdy_kernel<<<grid_for(da->N, 256), 256, 0, s>>>(da->nkey.p, da->N, 1u << (da->D - 1), d_out);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status convert_f64_to_f32(const double* a, float* b, int64_t n, cudaStream_t s) {
  f64_to_f32<<<grid_for(n, 256), 256, 0, s>>>(a, b, n);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace dg

using namespace dg;

namespace {
cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

template <class T>
dg_status upload(DBuf<T>& buf, const T* host, int64_t n) {
  DG_TRY(buf.alloc(n));
  if (n) DG_CUDA(cudaMemcpy(buf.p, host, sizeof(T) * n, cudaMemcpyHostToDevice));
  return DG_OK;
}
}  // namespace

extern "C" {

const char* dg_status_string(dg_status s) {
  switch (s) {
    case DG_OK: return "ok";
    case DG_EINVAL: return "invalid argument";
    case DG_ENOMEM: return "out of device memory";
    case DG_ECUDA: return "CUDA error";
    case DG_ENOTCONVERGED: return "not converged";
    case DG_ETIMEOUT: return "device wait timed out";
    case DG_EUNBALANCED: return "octree not linear/complete/balanced";
    case DG_EDEPTH: return "unsupported depth";
    case DG_ENOTIMPL: return "not implemented";
  }
  return "unknown status";
}

void dg_last_error(char* buf, size_t n) {
  if (!buf || !n) return;
  strncpy(buf, g_last_error.c_str(), n - 1);
  buf[n - 1] = 0;
}

int dg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

// ------------------------------------------------------------------ octree
dg_status dg_points2octree(const double* pts, int64_t n, int pts_on_device, uint32_t max_depth, uint32_t max_num_pts,
                           dg_octree** out) {
  DG_CHECK(out && (pts || n == 0) && n >= 0, DG_EINVAL, "points2octree: bad arguments");
  DG_CHECK(max_depth <= kMaxDepth, DG_EDEPTH, "points2octree: maxDepth must be <= 19");
  auto* t = new dg_octree();
  DBuf<double> dp;
  const double* src = pts;
  if (!pts_on_device && n) {
    dg_status st = upload(dp, pts, 3 * n);
    if (st) { delete t; return st; }
    src = dp.p;
  }
  dg_status st = points_to_octree(src, n, max_depth, max_num_pts, t, nullptr);
  if (st) { delete t; return st; }
  *out = t;
  return DG_OK;
}

dg_status dg_octree_from_octants(const dg_octant* octs, int64_t n, int on_device, uint32_t max_depth, dg_octree** out) {
  DG_CHECK(out && octs && n > 0, DG_EINVAL, "octree_from_octants: bad arguments");
  DG_CHECK(max_depth <= kMaxDepth, DG_EDEPTH, "octree_from_octants: maxDepth must be <= 19");
  DBuf<dg_octant> d;
  const dg_octant* src = octs;
  if (!on_device) {
    DG_TRY(upload(d, octs, n));
    src = d.p;
  }
  auto* t = new dg_octree();
  t->max_depth = max_depth;
  t->n = n;
  DBuf<uint32_t> bad;
  dg_status st = t->keys.alloc(n);
  if (!st) st = bad.alloc(1);
  if (st) { delete t; return st; }
  cudaMemset(bad.p, 0, 4);
  octants_to_keys<<<grid_for(n, 256), 256>>>(src, n, t->keys.p, bad.p, max_depth);
  uint32_t h = 0;
  if (cudaMemcpy(&h, bad.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess) { delete t; DG_CUDA(cudaGetLastError()); }
  if (h) {
    delete t;
    set_error(__FILE__, __LINE__, (h & 1) ? "octant level above maxDepth" : "octants not strictly Morton sorted");
    return DG_EUNBALANCED;
  }
  *out = t;
  return DG_OK;
}

dg_status dg_balance_octree(const dg_octree* in, dg_octree** out) {
  DG_CHECK(in && out, DG_EINVAL, "balance: bad arguments");
  auto* t = new dg_octree();
  dg_status st = balance_octree(in, t, nullptr);
  if (st) { delete t; return st; }
  *out = t;
  return DG_OK;
}

dg_status dg_coarsen_octree(const dg_octree* in, dg_octree** out) {
  DG_CHECK(in && out, DG_EINVAL, "coarsen: bad arguments");
  auto* t = new dg_octree();
  dg_status st = coarsen_octree(in, t, nullptr);
  if (st) { delete t; return st; }
  *out = t;
  return DG_OK;
}

int64_t dg_octree_size(const dg_octree* t) { return t ? t->n : 0; }
uint32_t dg_octree_max_depth(const dg_octree* t) { return t ? t->max_depth : 0; }

dg_status dg_octree_export(const dg_octree* t, dg_octant* host_out) {
  DG_CHECK(t && host_out, DG_EINVAL, "octree_export: bad arguments");
  DBuf<dg_octant> d;
  DG_TRY(d.alloc(t->n));
  keys_to_octants<<<grid_for(t->n, 256), 256>>>(t->keys.p, t->n, d.p, 0u);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaMemcpy(host_out, d.p, sizeof(dg_octant) * t->n, cudaMemcpyDeviceToHost));
  return DG_OK;
}

void dg_octree_destroy(dg_octree* t) { delete t; }

// -------------------------------------------------------------------- mesh
dg_status dg_da_create(const dg_octree* balanced, dg_da** out) {
  DG_CHECK(balanced && out, DG_EINVAL, "da_create: bad arguments");
  auto* da = new dg_da();
  dg_status st = build_mesh(balanced, da, nullptr);
  if (st) { delete da; return st; }
  *out = da;
  return DG_OK;
}

dg_status dg_da_create_from_maps(int64_t E, int64_t N, uint32_t max_depth, const uint32_t* nlist, const uint8_t* level,
                                 const uint8_t* cnum, const uint8_t* hmask, const uint32_t* node_xyz,
                                 const uint32_t* elem_xyz, dg_da** out) {
  DG_CHECK(out && nlist && level && cnum && hmask && node_xyz && elem_xyz && E > 0 && N > 0, DG_EINVAL,
           "da_create_from_maps: bad arguments");
  DG_CHECK(max_depth + 1 <= kMaxEmbeddedDepth, DG_EDEPTH, "da_create_from_maps: maxDepth must be <= 18");
  auto* da = new dg_da();
  da->D = max_depth + 1;
  da->E = E;
  da->N = N;
  std::vector<uint32_t> nl(8 * E), meta(E);
  std::vector<uint64_t> ek(E), nk(N);
  for (int64_t e = 0; e < E; ++e) {
    for (int v = 0; v < 8; ++v) {
      if (nlist[8 * e + v] >= uint64_t(N)) {
        delete da;
        set_error(__FILE__, __LINE__, "node id out of range");
        return DG_EINVAL;
      }
      nl[int64_t(v) * E + e] = nlist[8 * e + v];
    }
    meta[e] = meta_pack(level[e], cnum[e], hmask[e], 0);
    ek[e] = okey(morton(elem_xyz[3 * e], elem_xyz[3 * e + 1], elem_xyz[3 * e + 2]), level[e]);
  }
  for (int64_t i = 0; i < N; ++i) nk[i] = morton(node_xyz[3 * i], node_xyz[3 * i + 1], node_xyz[3 * i + 2]);
  dg_status st = upload(da->nl, nl.data(), 8 * E);
  if (!st) st = upload(da->meta, meta.data(), E);
  if (!st) st = upload(da->ekey, ek.data(), E);
  if (!st) st = upload(da->nkey, nk.data(), N);
  if (!st) st = build_tiles(da, nullptr);
  // octets: the corners a hanging vertex needs are nodes its own element
  // lists, so a mesh of any subset of elements has them
  if (!st) st = build_octets(da, nullptr);
  if (st) { delete da; return st; }
  *out = da;
  return DG_OK;
}

dg_status dg_da_sizes(const dg_da* da, int64_t* elements, int64_t* nodes, int64_t* pseudo) {
  DG_CHECK(da, DG_EINVAL, "da_sizes: null mesh");
  if (elements) *elements = da->E;
  if (nodes) *nodes = da->N;
  if (pseudo) *pseudo = da->P;
  return DG_OK;
}

uint32_t dg_da_max_depth(const dg_da* da) { return da ? da->D : 0; }

int64_t dg_da_octets(const dg_da* da) { return da ? da->octs.n : 0; }

dg_status dg_da_load_vector(const dg_da* da, const double* force, double* b, int on_device) {
  DG_CHECK(da && force && b, DG_EINVAL, "da_load_vector: bad arguments");
  if (on_device) {
    DG_TRY(load_vector(da, force, b, 0));
    DG_CUDA(cudaDeviceSynchronize());
    return DG_OK;
  }
  DBuf<double> df, db;
  DG_TRY(df.alloc(da->E));
  DG_TRY(db.alloc(da->N));
  if (da->E) DG_CUDA(cudaMemcpy(df.p, force, 8 * size_t(da->E), cudaMemcpyHostToDevice));
  DG_TRY(load_vector(da, df.p, db.p, 0));
  if (da->N) DG_CUDA(cudaMemcpy(b, db.p, 8 * size_t(da->N), cudaMemcpyDeviceToHost));
  return DG_OK;
}

dg_status dg_da_compress_maps(dg_da* da, int quotient_bits) {
  DG_CHECK(da, DG_EINVAL, "compress_maps: null mesh");
  DG_TRY(build_cmap(da, quotient_bits, 0));
  DG_CUDA(cudaDeviceSynchronize());
  return DG_OK;
}

int64_t dg_da_compressed_map_bytes(const dg_da* da, int64_t* wide_tiles) {
  if (wide_tiles) *wide_tiles = da ? da->cmap.wide_tiles : 0;
  return (da && da->cmap.qbits) ? da->cmap.bytes() : 0;
}

dg_status dg_da_decompress_maps(const dg_da* da, uint32_t* nlist) {
  DG_CHECK(da && nlist, DG_EINVAL, "decompress_maps: bad arguments");
  const int64_t E = da->E;
  if (!E) return DG_OK;
  DBuf<uint32_t> d;
  DG_TRY(d.alloc(8 * E));
  DG_TRY(cmap_decode(da, d.p, 0));
  std::vector<uint32_t> nl(8 * E);
  DG_CUDA(cudaMemcpy(nl.data(), d.p, 4 * 8 * E, cudaMemcpyDeviceToHost));
  for (int64_t e = 0; e < E; ++e)
    for (int v = 0; v < 8; ++v) nlist[8 * e + v] = nl[int64_t(v) * E + e];
  return DG_OK;
}

dg_status dg_da_export(const dg_da* da, uint32_t* nlist, uint8_t* hmask, uint8_t* cnum, uint8_t* etype, uint8_t* level,
                       uint32_t* node_xyz, uint32_t* elem_xyz, uint8_t* node_bdy) {
  DG_CHECK(da, DG_EINVAL, "da_export: null mesh");
  const int64_t E = da->E, N = da->N;
  if (nlist) {
    std::vector<uint32_t> nl(8 * E);
    DG_CUDA(cudaMemcpy(nl.data(), da->nl.p, 4 * 8 * E, cudaMemcpyDeviceToHost));
    for (int64_t e = 0; e < E; ++e)
      for (int v = 0; v < 8; ++v) nlist[8 * e + v] = nl[int64_t(v) * E + e];
  }
  if (hmask || cnum || etype || level) {
    std::vector<uint32_t> meta(E);
    DG_CUDA(cudaMemcpy(meta.data(), da->meta.p, 4 * E, cudaMemcpyDeviceToHost));
    for (int64_t e = 0; e < E; ++e) {
      if (hmask) hmask[e] = uint8_t(meta_mask(meta[e]));
      if (cnum) cnum[e] = uint8_t(meta_cnum(meta[e]));
      if (etype) etype[e] = uint8_t(meta_type(meta[e]));
      if (level) level[e] = uint8_t(meta_lev(meta[e]));
    }
  }
  if (node_xyz || elem_xyz) {
    DBuf<uint32_t> d;
    DG_TRY(d.alloc(3 * (N > E ? N : E)));
    if (node_xyz) {
      decode_xyz<<<grid_for(N, 256), 256>>>(da->nkey.p, N, 0, d.p);
      DG_CUDA(cudaMemcpy(node_xyz, d.p, 12 * N, cudaMemcpyDeviceToHost));
    }
    if (elem_xyz) {
      decode_xyz<<<grid_for(E, 256), 256>>>(da->ekey.p, E, 1, d.p);
      DG_CUDA(cudaMemcpy(elem_xyz, d.p, 12 * E, cudaMemcpyDeviceToHost));
    }
  }
  if (node_bdy) {
    DBuf<uint8_t> b;
    DG_TRY(b.alloc(N));
    DG_TRY(node_boundary_flags(da, b.p, nullptr));
    DG_CUDA(cudaMemcpy(node_bdy, b.p, N, cudaMemcpyDeviceToHost));
  }
  return DG_OK;
}

dg_status dg_da_element_centers(const dg_da* da, double* host_out) {
  DG_CHECK(da && host_out, DG_EINVAL, "element_centers: bad arguments");
  DBuf<double> c;
  DG_TRY(c.alloc(3 * da->E));
  centers_kernel<<<grid_for(da->E, 256), 256>>>(da->ekey.p, da->E, da->D, c.p);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaMemcpy(host_out, c.p, 24 * da->E, cudaMemcpyDeviceToHost));
  return DG_OK;
}

void dg_da_destroy(dg_da* da) { delete da; }

// --------------------------------------------------------------- operators
dg_status dg_mat_create_lapmass(dg_da* da, const double* coef, dg_mat** out) {
  DG_CHECK(da && out, DG_EINVAL, "mat_create_lapmass: bad arguments");
  auto* A = new dg_mat();
  A->da = da;
  A->kind = 0;
  A->dof = 1;
  if (coef) {
    A->has_coef = true;
    std::vector<double> soa(2 * da->E);
    for (int64_t e = 0; e < da->E; ++e) {
      soa[e] = coef[2 * e];
      soa[da->E + e] = coef[2 * e + 1];
    }
    dg_status st = A->coef.alloc(2 * da->E + kCoefPad);
    if (!st && cudaMemcpy(A->coef.p, soa.data(), 16 * da->E, cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error(__FILE__, __LINE__, "cudaMemcpy of the coefficients");
      st = DG_ECUDA;
    }
    if (!st) st = A->coef32.alloc(2 * da->E + kCoefPad);
    if (!st) st = convert_f64_to_f32(A->coef.p, A->coef32.p, 2 * da->E, nullptr);
    if (st) { delete A; return st; }
  }
  *out = A;
  return DG_OK;
}

dg_status dg_mat_create_elasticity(dg_da* da, double mu, double lambda, const uint8_t* dirichlet, dg_mat** out) {
  DG_CHECK(da && out, DG_EINVAL, "mat_create_elasticity: bad arguments");
  auto* A = new dg_mat();
  A->da = da;
  A->kind = 1;
  A->dof = 3;
  A->mu = mu;
  A->lam = lambda;
  dg_status st = A->dirichlet.alloc(da->N);
  if (!st) {
    if (dirichlet) {
      if (cudaMemcpy(A->dirichlet.p, dirichlet, da->N, cudaMemcpyHostToDevice) != cudaSuccess) st = DG_ECUDA;
    } else {
      st = node_boundary_flags(da, A->dirichlet.p, nullptr);
    }
  }
  if (st) { delete A; return st; }
  *out = A;
  return DG_OK;
}

dg_status dg_mat_create_dirichlet(dg_da* da, int with_mass, const uint8_t* dirichlet, dg_mat** out) {
  DG_CHECK(da && out, DG_EINVAL, "mat_create_dirichlet: bad arguments");
  auto* A = new dg_mat();
  A->da = da;
  A->kind = with_mass ? 3 : 2;
  A->dof = 1;
  dg_status st = A->dirichlet.alloc(da->N);
  if (!st) {
    if (dirichlet) {
      if (cudaMemcpy(A->dirichlet.p, dirichlet, da->N, cudaMemcpyHostToDevice) != cudaSuccess) st = DG_ECUDA;
    } else {
      st = node_boundary_flags(da, A->dirichlet.p, nullptr);
    }
  }
  if (st) { delete A; return st; }
  *out = A;
  return DG_OK;
}

dg_status dg_mat_mult(dg_mat* A, const double* x, double* y, void* stream) {
  DG_CHECK(A && x && y, DG_EINVAL, "mat_mult: bad arguments");
  if (A->kind == 1) return elasticity_apply_f64(A, x, y, as_stream(stream));
  if (A->kind >= 2) return dirichlet_apply_f64(A, x, y, as_stream(stream));
  return lapmass_apply_f64(A, x, y, as_stream(stream));
}

dg_status dg_mat_mult_add(dg_mat* A, const double* x, double* y, void* stream) {
  DG_CHECK(A && x && y, DG_EINVAL, "mat_mult_add: bad arguments");
  DG_CHECK(A->kind == 0, DG_ENOTIMPL, "mat_mult_add: scalar operator only");
  return lapmass_apply_add_f64(A, x, y, as_stream(stream));
}

dg_status dg_mat_mult_add_f32(dg_mat* A, const float* x, float* y, void* stream) {
  DG_CHECK(A && x && y, DG_EINVAL, "mat_mult_add_f32: bad arguments");
  DG_CHECK(A->kind == 0, DG_ENOTIMPL, "mat_mult_add_f32: scalar operator only");
  return lapmass_apply_add_f32(A, x, y, as_stream(stream));
}

dg_status dg_mat_mult_f32(dg_mat* A, const float* x, float* y, void* stream) {
  DG_CHECK(A && x && y, DG_EINVAL, "mat_mult_f32: bad arguments");
  DG_CHECK(A->kind == 0, DG_ENOTIMPL, "mat_mult_f32: scalar operator only");
  return lapmass_apply_f32(A, x, y, as_stream(stream));
}

dg_status dg_mat_get_diagonal(dg_mat* A, double* d, void* stream) {
  DG_CHECK(A && d, DG_EINVAL, "mat_get_diagonal: bad arguments");
  if (A->kind == 1) return elasticity_diag(A, d, as_stream(stream));
  if (A->kind >= 2) return dirichlet_diag(A, d, as_stream(stream));
  return lapmass_diag(A, d, as_stream(stream));
}

dg_status dg_mat_mult_host(dg_mat* A, const double* x, double* y) {
  DG_CHECK(A && x && y, DG_EINVAL, "mat_mult_host: bad arguments");
  const int64_t n = int64_t(A->dof) * A->da->N;
  if (A->host_x.n != n) DG_TRY(A->host_x.alloc(n));
  if (A->host_y.n != n) DG_TRY(A->host_y.alloc(n));
  // large scalar meshes: copies pipelined against the operator (after the
  // first call, which tunes the launch shape); the others copy, apply, copy
  const dg_status ps = lapmass_apply_host_pipelined_f64(A, x, y);
  if (ps != DG_ENOTIMPL) return ps;
  DG_CUDA(cudaMemcpyAsync(A->host_x.p, x, 8 * n, cudaMemcpyHostToDevice, nullptr));
  DG_TRY(dg_mat_mult(A, A->host_x.p, A->host_y.p, nullptr));
  DG_CUDA(cudaMemcpyAsync(y, A->host_y.p, 8 * n, cudaMemcpyDeviceToHost, nullptr));
  return device_wait_status(nullptr);  // synchronises
}

dg_status dg_device_check(void* stream) { return device_wait_status(as_stream(stream)); }

dg_status dg_set_device_wait_limit(int64_t cycles) {
  set_wait_limit(static_cast<long long>(cycles));
  return DG_OK;
}

int64_t dg_mat_size(const dg_mat* A) { return A ? int64_t(A->dof) * A->da->N : 0; }

const char* dg_mat_kernel_name(const dg_mat* A, int prec) {
  if (!A) return "none";
  if (A->kind == 1) return "elasticity";
  if (A->kind >= 2) return "dirichlet";
  return matvec_variant_name(prec == DG_PREC_F64 ? A->da->tuned_f64 : A->da->tuned_f32);
}

int dg_mat_kernel_count(void) { return matvec_variant_count(); }

dg_status dg_mat_mult_multi(dg_mat* A, const float* X, float* Y, int nrhs, int split, void* stream) {
  DG_CHECK(A && X && Y, DG_EINVAL, "mat_mult_multi: null argument");
  return mrhs_apply(A, X, Y, nrhs, split, static_cast<cudaStream_t>(stream));
}

dg_status dg_mat_set_kernel(dg_mat* A, int prec, int variant) {
  DG_CHECK(A && A->kind == 0, DG_EINVAL, "set_kernel: scalar operator expected");
  DG_CHECK(variant >= 0 && variant < matvec_variant_count(), DG_EINVAL, "set_kernel: variant out of range");
  DG_CHECK(prec == DG_PREC_F64 || prec == DG_PREC_F32, DG_EINVAL, "set_kernel: precision");
  (prec == DG_PREC_F64 ? A->da->tuned_f64 : A->da->tuned_f32) = variant;
  return DG_OK;
}

void dg_mat_destroy(dg_mat* A) { delete A; }

}  // extern "C"
