// One mesh over several ranks: the partition, one rank's halo, and the
// kernels of its ghost exchange -- ot::DA with npes > 1 (include/oda/oda.h:500-512;
// ReadFromGhostsBegin/End and WriteToGhostsBegin/End, include/oda/oda.txx:479-650).
//
// Elements are split into contiguous Morton ranges of equal weight by the rule
// of par::partitionW (include/par/parUtils.txx:1011-1177).  A node belongs to
// the rank whose range holds its anchor: node ids follow the Morton order of
// the anchors, so every rank owns one contiguous id range, as the reference's
// ranks own the nodes anchored at their octants.  A rank keeps every element
// with a vertex it owns: its independent elements (all eight vertices owned)
// and its dependent ones (the DEPENDENT loop of Jacobian2MatMult,
// examples/src/backend/omgNeumann.C:517-523, which with the pre-ghost
// elements of src/oda/private/odaBuildNlist.C:815-821 covers the partition
// boundary).  One exchange of ghost node values, owner to reader, before the
// dependent elements then makes y = A x complete on the owned nodes.
//
// Local node numbering of a rank: its owned nodes first (global id minus the
// first owned id), then its ghost nodes in ascending global id, which groups
// them by owner in rank order, so an all-to-all of the owners' packed values
// lands directly after the owned nodes.  The independent elements form one
// local mesh over the owned nodes; the dependent elements another over all
// local nodes, applied with y += A x into the local vector.
//
// The partition and the maps are host set-up and touch no GPU; the exchange
// is a pack kernel, one all-to-all of the packed values and, for
// accumulation to the owners, a gather-sum kernel in a fixed order.
#include <algorithm>
#include <memory>
#include <numeric>
#include <vector>

#include "dg_internal.h"

using dg::DBuf;

struct dg_halo {
  int nranks = 1, rank = 0;
  uint32_t max_depth = 0;
  std::vector<int64_t> elem_first, node_first;  // [nranks + 1]
  int64_t n_own = 0;
  std::vector<uint32_t> ghosts;                 // global ids, ascending
  std::vector<int64_t> send_count, recv_count;  // per peer
  std::vector<uint32_t> send_idx;               // local ids of owned nodes, by peer, then ascending
  // 0: independent elements over the owned nodes; 1: dependent elements over all local nodes
  struct Part {
    std::vector<int64_t> elems;  // global element ids, ascending
    std::vector<uint32_t> nl;    // [E][8] local node ids
    std::vector<uint8_t> level, cnum, hmask;
    std::vector<uint32_t> exyz, nxyz;
  } part[2];
  // accumulation to owners: the positions of send_idx grouped by node
  std::vector<uint32_t> acc_node, acc_ptr, acc_pos;
  // device copies, uploaded on the first exchange call
  int device = -1;
  DBuf<uint32_t> d_send_idx, d_acc_node, d_acc_ptr, d_acc_pos;
};

// Rows of a sparse matrix M (a transfer between two partitioned levels) that
// one rank owns, with the columns it reads: owned columns first (global id
// minus the first owned id), then ghost columns ascending by global id.
struct dg_parcsr {
  int nranks = 1, rank = 0;
  int64_t row0 = 0, nrow = 0, col0 = 0, ncol_own = 0;
  std::vector<uint32_t> ptr, col;
  std::vector<double> val;
  std::vector<uint32_t> ghosts;                 // global column ids, ascending
  std::vector<int64_t> send_count, recv_count;  // per peer
  std::vector<uint32_t> send_idx;               // owned columns the peers read, by peer, then ascending
  int device = -1;
  DBuf<uint32_t> d_ptr, d_col, d_send_idx;
  DBuf<double> d_val;
  DBuf<float> d_val32;  // FP32 copy of the entries, for the FP32 products
};

namespace {

constexpr int kHaloThreads = 256;

// par::partitionW (include/par/parUtils.txx:1130-1177) applied to a list held
// whole: with s the inclusive scan of the weights, W their sum, avg = W / P
// and extra = W % P, an item goes to rank 0 when s == 0, to (s - 1) / (avg + 1)
// while s <= extra (avg + 1), else to (s - 1 - extra) / avg; with avg == 0
// every item goes to rank 0.  The scan is monotone, so every rank receives one
// contiguous range: first[r] .. first[r + 1].
void partition_weighted(int64_t n, const uint32_t* w, int P, int64_t* first) {
  std::vector<int64_t> cnt(P, 0);
  int64_t W = 0;
  for (int64_t i = 0; i < n; ++i) W += w ? int64_t(w[i]) : 1;
  const int64_t avg = W / P, extra = W % P;
  if (avg == 0) {
    cnt[0] = n;
  } else {
    int64_t s = 0;
    for (int64_t i = 0; i < n; ++i) {
      s += w ? int64_t(w[i]) : 1;
      int64_t r = 0;
      if (s != 0) r = s <= extra * (avg + 1) ? (s - 1) / (avg + 1) : (s - 1 - extra) / avg;
      ++cnt[r];
    }
  }
  first[0] = 0;
  for (int r = 0; r < P; ++r) first[r + 1] = first[r] + cnt[r];
}

template <class T>
__global__ void __launch_bounds__(kHaloThreads)
halo_gather(const uint32_t* __restrict__ idx, int64_t n, int dof, const T* __restrict__ x, T* __restrict__ out) {
  const int64_t total = n * dof;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t k = t / dof;
    out[t] = x[int64_t(idx[k]) * dof + (t - k * dof)];
  }
}

// y[node[u]] += each received value of node u in turn, in peer order (the
// order of WriteToGhostsEnd's loop over the scatter map, oda.txx:628-633)
__global__ void __launch_bounds__(kHaloThreads)
halo_accumulate(const uint32_t* __restrict__ node, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ pos,
                int64_t nu, int dof, const double* __restrict__ recv, double* __restrict__ y) {
  const int64_t total = nu * dof;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t u = t / dof;
    const int c = int(t - u * dof);
    double* out = y + int64_t(node[u]) * dof + c;
    double s = *out;
    for (uint32_t j = ptr[u]; j < ptr[u + 1]; ++j) s += recv[int64_t(pos[j]) * dof + c];
    *out = s;
  }
}

// y[i] (+)= sum_k val[k] x[col[k]] over the rank's rows; a column below
// nown reads the owned values, the rest the ghost values (FP64 or FP32)
template <class T>
__global__ void __launch_bounds__(kHaloThreads)
parcsr_spmv(const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col, const T* __restrict__ val,
            int64_t nrow, int64_t nown, const T* __restrict__ x_own, const T* __restrict__ x_ghost,
            T* __restrict__ y, int add) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nrow; i += int64_t(gridDim.x) * blockDim.x) {
    T s = add ? y[i] : T(0);
    for (uint32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
      const int64_t c = col[k];
      s += val[k] * (c < nown ? x_own[c] : x_ghost[c - nown]);
    }
    y[i] = s;
  }
}

// x[i] += omega dinv[i] (b[i] - ax[i]): one damped Jacobi sweep's update
template <class T>
__global__ void __launch_bounds__(kHaloThreads)
jacobi_update(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ ax, const T* __restrict__ dinv,
              T omega, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] += omega * dinv[i] * (b[i] - ax[i]);
}

template <class T>
dg_status upload_vec(DBuf<T>& d, const std::vector<T>& h) {
  DG_TRY(d.alloc(int64_t(h.size())));
  if (!h.empty()) DG_CUDA(cudaMemcpy(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return DG_OK;
}

dg_status ensure_device(dg_halo* h) {
  int dev = -1;
  DG_CUDA(cudaGetDevice(&dev));
  if (h->device == dev) return DG_OK;
  DG_CHECK(h->device < 0, DG_EINVAL, "halo: used on a second device");
  DG_TRY(upload_vec(h->d_send_idx, h->send_idx));
  DG_TRY(upload_vec(h->d_acc_node, h->acc_node));
  DG_TRY(upload_vec(h->d_acc_ptr, h->acc_ptr));
  DG_TRY(upload_vec(h->d_acc_pos, h->acc_pos));
  h->device = dev;
  return DG_OK;
}

template <class T>
void gather_rows(std::vector<T>& out, const T* src, const std::vector<int64_t>& rows, int width) {
  out.resize(rows.size() * width);
  for (size_t i = 0; i < rows.size(); ++i)
    for (int c = 0; c < width; ++c) out[i * width + c] = src[rows[i] * width + c];
}

}  // namespace

extern "C" {

dg_status dg_partition_weighted(int64_t n, const uint32_t* weights, int nranks, int64_t* first) {
  DG_CHECK(n >= 0 && nranks >= 1 && first, DG_EINVAL, "partition_weighted: bad arguments");
  partition_weighted(n, weights, nranks, first);
  return DG_OK;
}

dg_status dg_halo_create(int64_t E, int64_t N, uint32_t max_depth, const uint32_t* nlist, const uint8_t* level,
                         const uint8_t* cnum, const uint8_t* hmask, const uint32_t* node_xyz, const uint32_t* elem_xyz,
                         const uint32_t* weights, int nranks, int rank, dg_halo** out) {
  DG_CHECK(out && nlist && level && cnum && hmask && node_xyz && elem_xyz && E > 0 && N > 0, DG_EINVAL,
           "halo_create: bad arguments");
  DG_CHECK(nranks >= 1 && rank >= 0 && rank < nranks, DG_EINVAL, "halo_create: rank out of range");
  DG_CHECK(N <= int64_t(UINT32_MAX), DG_EINVAL, "halo_create: too many nodes");
  DG_CHECK(max_depth + 1 <= dg::kMaxEmbeddedDepth, DG_EDEPTH, "halo_create: maxDepth must be <= 18");
  auto h = std::make_unique<dg_halo>();
  const int P = nranks;
  h->nranks = P;
  h->rank = rank;
  h->max_depth = max_depth;
  h->elem_first.resize(P + 1);
  partition_weighted(E, weights, P, h->elem_first.data());

  // node ranges: the nodes whose anchors lie between the anchors of the first
  // elements of consecutive non-empty ranks
  std::vector<uint64_t> nk(N);
  for (int64_t i = 0; i < N; ++i) nk[i] = dg::morton(node_xyz[3 * i], node_xyz[3 * i + 1], node_xyz[3 * i + 2]);
  for (int64_t i = 1; i < N; ++i)
    DG_CHECK(nk[i - 1] < nk[i], DG_EINVAL, "halo_create: node ids must follow the Morton order of their anchors");
  auto& nf = h->node_first;
  nf.assign(P + 1, 0);
  nf[P] = N;
  int first_nonempty = P;
  for (int r = P - 1; r >= 0; --r) {
    if (h->elem_first[r] == h->elem_first[r + 1]) {
      nf[r] = nf[r + 1];
      continue;
    }
    const int64_t e = h->elem_first[r];
    const uint64_t key = dg::morton(elem_xyz[3 * e], elem_xyz[3 * e + 1], elem_xyz[3 * e + 2]);
    nf[r] = std::min<int64_t>(std::lower_bound(nk.begin(), nk.end(), key) - nk.begin(), nf[r + 1]);
    first_nonempty = r;
  }
  for (int r = 0; r <= first_nonempty && r <= P; ++r) nf[r] = 0;
  std::vector<int32_t> owner(N);
  for (int r = 0; r < P; ++r)
    for (int64_t v = nf[r]; v < nf[r + 1]; ++v) owner[v] = r;

  const int64_t n0 = nf[rank];
  h->n_own = nf[rank + 1] - n0;
  std::vector<int64_t>& ind = h->part[0].elems;
  std::vector<int64_t>& dep = h->part[1].elems;
  std::vector<uint32_t> ghost_refs;
  std::vector<uint64_t> sends;  // peer << 32 | local id of an owned node
  for (int64_t e = 0; e < E; ++e) {
    const uint32_t* ids = nlist + 8 * e;
    int ranks[8], nr = 0;
    bool mine = false;
    for (int k = 0; k < 8; ++k) {
      DG_CHECK(ids[k] < uint64_t(N), DG_EINVAL, "halo_create: node id out of range");
      const int q = owner[ids[k]];
      mine |= q == rank;
      bool seen = false;
      for (int j = 0; j < nr; ++j) seen |= ranks[j] == q;
      if (!seen) ranks[nr++] = q;
    }
    if (!mine) continue;
    if (nr == 1) {
      ind.push_back(e);
      continue;
    }
    dep.push_back(e);
    for (int k = 0; k < 8; ++k) {
      if (owner[ids[k]] != rank) {
        ghost_refs.push_back(ids[k]);
        continue;
      }
      for (int j = 0; j < nr; ++j)
        if (ranks[j] != rank) sends.push_back(uint64_t(ranks[j]) << 32 | uint64_t(ids[k] - n0));
    }
  }
  std::sort(ghost_refs.begin(), ghost_refs.end());
  ghost_refs.erase(std::unique(ghost_refs.begin(), ghost_refs.end()), ghost_refs.end());
  h->ghosts = std::move(ghost_refs);
  std::sort(sends.begin(), sends.end());
  sends.erase(std::unique(sends.begin(), sends.end()), sends.end());
  h->send_count.assign(P, 0);
  h->recv_count.assign(P, 0);
  h->send_idx.resize(sends.size());
  for (size_t k = 0; k < sends.size(); ++k) {
    ++h->send_count[sends[k] >> 32];
    h->send_idx[k] = uint32_t(sends[k]);
  }
  for (uint32_t g : h->ghosts) ++h->recv_count[owner[g]];

  // accumulation order: positions of send_idx by node, peers ascending within a node
  {
    std::vector<uint32_t> order(h->send_idx.size());
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return h->send_idx[a] < h->send_idx[b]; });
    h->acc_pos = order;
    h->acc_ptr.push_back(0);
    for (size_t j = 0; j < order.size(); ++j) {
      if (j == 0 || h->send_idx[order[j]] != h->send_idx[order[j - 1]]) {
        if (j) h->acc_ptr.push_back(uint32_t(j));
        h->acc_node.push_back(h->send_idx[order[j]]);
      }
    }
    if (!order.empty()) h->acc_ptr.push_back(uint32_t(order.size()));
  }

  auto local_id = [&](uint32_t v) -> uint32_t {
    if (owner[v] == rank) return uint32_t(v - n0);
    return uint32_t(h->n_own + (std::lower_bound(h->ghosts.begin(), h->ghosts.end(), v) - h->ghosts.begin()));
  };
  for (int p = 0; p < 2; ++p) {
    auto& pt = h->part[p];
    gather_rows(pt.level, level, pt.elems, 1);
    gather_rows(pt.cnum, cnum, pt.elems, 1);
    gather_rows(pt.hmask, hmask, pt.elems, 1);
    gather_rows(pt.exyz, elem_xyz, pt.elems, 3);
    gather_rows(pt.nl, nlist, pt.elems, 8);
    for (auto& v : pt.nl) v = local_id(v);
  }
  h->part[0].nxyz.assign(node_xyz + 3 * n0, node_xyz + 3 * (n0 + h->n_own));
  {
    auto& nx = h->part[1].nxyz;
    nx = h->part[0].nxyz;
    nx.reserve(3 * (h->n_own + h->ghosts.size()));
    for (uint32_t g : h->ghosts) nx.insert(nx.end(), node_xyz + 3 * int64_t(g), node_xyz + 3 * int64_t(g) + 3);
  }
  *out = h.release();
  return DG_OK;
}

dg_status dg_halo_create_from_da(const dg_da* da, const uint32_t* weights, int nranks, int rank, dg_halo** out) {
  DG_CHECK(da && out, DG_EINVAL, "halo_create_from_da: bad arguments");
  const int64_t E = da->E, N = da->N;
  std::vector<uint32_t> nl(8 * E), nxyz(3 * N), exyz(3 * E);
  std::vector<uint8_t> hm(E), cn(E), lv(E);
  DG_TRY(dg_da_export(da, nl.data(), hm.data(), cn.data(), nullptr, lv.data(), nxyz.data(), exyz.data(), nullptr));
  return dg_halo_create(E, N, da->D - 1, nl.data(), lv.data(), cn.data(), hm.data(), nxyz.data(), exyz.data(), weights,
                        nranks, rank, out);
}

dg_status dg_halo_sizes(const dg_halo* h, int64_t* n_owned, int64_t* n_ghost, int64_t* first_owned,
                        int64_t* n_independent, int64_t* n_dependent) {
  DG_CHECK(h, DG_EINVAL, "halo_sizes: null halo");
  if (n_owned) *n_owned = h->n_own;
  if (n_ghost) *n_ghost = int64_t(h->ghosts.size());
  if (first_owned) *first_owned = h->node_first[h->rank];
  if (n_independent) *n_independent = int64_t(h->part[0].elems.size());
  if (n_dependent) *n_dependent = int64_t(h->part[1].elems.size());
  return DG_OK;
}

dg_status dg_halo_ranges(const dg_halo* h, int64_t* elem_first, int64_t* node_first) {
  DG_CHECK(h, DG_EINVAL, "halo_ranges: null halo");
  if (elem_first) std::copy(h->elem_first.begin(), h->elem_first.end(), elem_first);
  if (node_first) std::copy(h->node_first.begin(), h->node_first.end(), node_first);
  return DG_OK;
}

dg_status dg_halo_comm(const dg_halo* h, int64_t* send_counts, int64_t* recv_counts, uint32_t* send_idx,
                       uint32_t* ghosts) {
  DG_CHECK(h, DG_EINVAL, "halo_comm: null halo");
  if (send_counts) std::copy(h->send_count.begin(), h->send_count.end(), send_counts);
  if (recv_counts) std::copy(h->recv_count.begin(), h->recv_count.end(), recv_counts);
  if (send_idx) std::copy(h->send_idx.begin(), h->send_idx.end(), send_idx);
  if (ghosts) std::copy(h->ghosts.begin(), h->ghosts.end(), ghosts);
  return DG_OK;
}

dg_status dg_halo_part(const dg_halo* h, int which, int64_t* elems, uint32_t* nlist) {
  DG_CHECK(h && (which == 0 || which == 1), DG_EINVAL, "halo_part: bad arguments");
  const auto& pt = h->part[which];
  if (elems) std::copy(pt.elems.begin(), pt.elems.end(), elems);
  if (nlist) std::copy(pt.nl.begin(), pt.nl.end(), nlist);
  return DG_OK;
}

dg_status dg_halo_local_da(const dg_halo* h, int which, dg_da** out) {
  DG_CHECK(h && out && (which == 0 || which == 1), DG_EINVAL, "halo_local_da: bad arguments");
  const auto& pt = h->part[which];
  DG_CHECK(!pt.elems.empty(), DG_EINVAL, "halo_local_da: the part has no elements");
  const int64_t n = int64_t(pt.nxyz.size() / 3);
  return dg_da_create_from_maps(int64_t(pt.elems.size()), n, h->max_depth, pt.nl.data(), pt.level.data(),
                                pt.cnum.data(), pt.hmask.data(), pt.nxyz.data(), pt.exyz.data(), out);
}

dg_status dg_halo_pack(dg_halo* h, const double* x_local, double* send, int dof, void* stream) {
  DG_CHECK(h && dof >= 1 && (h->send_idx.empty() || (x_local && send)), DG_EINVAL, "halo_pack: bad arguments");
  DG_TRY(ensure_device(h));
  const int64_t n = int64_t(h->send_idx.size());
  if (n == 0) return DG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  halo_gather<<<dg::grid_for(n * dof, kHaloThreads), kHaloThreads, 0, s>>>(h->d_send_idx.p, n, dof, x_local, send);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dg_halo_pack_f32(dg_halo* h, const float* x_local, float* send, int dof, void* stream) {
  DG_CHECK(h && dof >= 1 && (h->send_idx.empty() || (x_local && send)), DG_EINVAL, "halo_pack_f32: bad arguments");
  DG_TRY(ensure_device(h));
  const int64_t n = int64_t(h->send_idx.size());
  if (n == 0) return DG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  halo_gather<<<dg::grid_for(n * dof, kHaloThreads), kHaloThreads, 0, s>>>(h->d_send_idx.p, n, dof, x_local, send);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dg_halo_accumulate(dg_halo* h, const double* recv, double* y_local, int dof, void* stream) {
  DG_CHECK(h && dof >= 1 && (h->acc_node.empty() || (recv && y_local)), DG_EINVAL, "halo_accumulate: bad arguments");
  DG_TRY(ensure_device(h));
  const int64_t nu = int64_t(h->acc_node.size());
  if (nu == 0) return DG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  halo_accumulate<<<dg::grid_for(nu * dof, kHaloThreads), kHaloThreads, 0, s>>>(
      h->d_acc_node.p, h->d_acc_ptr.p, h->d_acc_pos.p, nu, dof, recv, y_local);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

void dg_halo_destroy(dg_halo* h) { delete h; }

dg_status dg_parcsr_create(int64_t nrows, int64_t ncols, const uint32_t* ptr, const uint32_t* col, const double* val,
                           const int64_t* row_first, const int64_t* col_first, int nranks, int rank, dg_parcsr** out) {
  DG_CHECK(out && ptr && row_first && col_first && nrows >= 0 && ncols >= 0, DG_EINVAL, "parcsr_create: bad arguments");
  DG_CHECK(nranks >= 1 && rank >= 0 && rank < nranks, DG_EINVAL, "parcsr_create: rank out of range");
  DG_CHECK(ncols <= int64_t(UINT32_MAX), DG_EINVAL, "parcsr_create: too many columns");
  const int P = nranks;
  DG_CHECK(row_first[0] == 0 && row_first[P] == nrows && col_first[0] == 0 && col_first[P] == ncols, DG_EINVAL,
           "parcsr_create: ranges must cover the rows and the columns");
  for (int r = 0; r < P; ++r)
    DG_CHECK(row_first[r] <= row_first[r + 1] && col_first[r] <= col_first[r + 1], DG_EINVAL,
             "parcsr_create: ranges must be ascending");
  const int64_t nnz = ptr[nrows];
  DG_CHECK(nnz == 0 || (col && val), DG_EINVAL, "parcsr_create: missing entries");
  for (int64_t i = 0; i < nrows; ++i) DG_CHECK(ptr[i] <= ptr[i + 1], DG_EINVAL, "parcsr_create: bad row pointers");
  for (int64_t k = 0; k < nnz; ++k) DG_CHECK(col[k] < uint64_t(ncols), DG_EINVAL, "parcsr_create: column out of range");
  std::vector<int32_t> cown(ncols);
  for (int r = 0; r < P; ++r)
    for (int64_t c = col_first[r]; c < col_first[r + 1]; ++c) cown[c] = r;

  auto pc = std::make_unique<dg_parcsr>();
  pc->nranks = P;
  pc->rank = rank;
  pc->row0 = row_first[rank];
  pc->nrow = row_first[rank + 1] - pc->row0;
  pc->col0 = col_first[rank];
  pc->ncol_own = col_first[rank + 1] - pc->col0;
  std::vector<uint32_t> ghost_refs;
  std::vector<uint64_t> sends;  // peer << 32 | local id of an owned column
  for (int q = 0; q < P; ++q)
    for (int64_t i = row_first[q]; i < row_first[q + 1]; ++i)
      for (uint32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
        const int o = cown[col[k]];
        if (q == rank && o != rank) ghost_refs.push_back(col[k]);
        if (q != rank && o == rank) sends.push_back(uint64_t(q) << 32 | uint64_t(col[k] - pc->col0));
      }
  std::sort(ghost_refs.begin(), ghost_refs.end());
  ghost_refs.erase(std::unique(ghost_refs.begin(), ghost_refs.end()), ghost_refs.end());
  pc->ghosts = std::move(ghost_refs);
  std::sort(sends.begin(), sends.end());
  sends.erase(std::unique(sends.begin(), sends.end()), sends.end());
  pc->send_count.assign(P, 0);
  pc->recv_count.assign(P, 0);
  pc->send_idx.resize(sends.size());
  for (size_t k = 0; k < sends.size(); ++k) {
    ++pc->send_count[sends[k] >> 32];
    pc->send_idx[k] = uint32_t(sends[k]);
  }
  for (uint32_t g : pc->ghosts) ++pc->recv_count[cown[g]];
  const uint32_t base = ptr[pc->row0];
  pc->ptr.resize(pc->nrow + 1);
  for (int64_t i = 0; i <= pc->nrow; ++i) pc->ptr[i] = ptr[pc->row0 + i] - base;
  const int64_t lnnz = pc->ptr[pc->nrow];
  pc->col.resize(lnnz);
  pc->val.assign(val + base, val + base + lnnz);
  for (int64_t k = 0; k < lnnz; ++k) {
    const uint32_t c = col[base + k];
    pc->col[k] = cown[c] == rank ? uint32_t(c - pc->col0)
                                 : uint32_t(pc->ncol_own + (std::lower_bound(pc->ghosts.begin(), pc->ghosts.end(), c) -
                                                            pc->ghosts.begin()));
  }
  *out = pc.release();
  return DG_OK;
}

dg_status dg_parcsr_sizes(const dg_parcsr* pc, int64_t* n_rows, int64_t* n_cols_owned, int64_t* n_ghost,
                          int64_t* nnz) {
  DG_CHECK(pc, DG_EINVAL, "parcsr_sizes: null matrix");
  if (n_rows) *n_rows = pc->nrow;
  if (n_cols_owned) *n_cols_owned = pc->ncol_own;
  if (n_ghost) *n_ghost = int64_t(pc->ghosts.size());
  if (nnz) *nnz = int64_t(pc->col.size());
  return DG_OK;
}

dg_status dg_parcsr_comm(const dg_parcsr* pc, int64_t* send_counts, int64_t* recv_counts, uint32_t* send_idx,
                         uint32_t* ghosts) {
  DG_CHECK(pc, DG_EINVAL, "parcsr_comm: null matrix");
  if (send_counts) std::copy(pc->send_count.begin(), pc->send_count.end(), send_counts);
  if (recv_counts) std::copy(pc->recv_count.begin(), pc->recv_count.end(), recv_counts);
  if (send_idx) std::copy(pc->send_idx.begin(), pc->send_idx.end(), send_idx);
  if (ghosts) std::copy(pc->ghosts.begin(), pc->ghosts.end(), ghosts);
  return DG_OK;
}

static dg_status parcsr_device(dg_parcsr* pc) {
  int dev = -1;
  DG_CUDA(cudaGetDevice(&dev));
  if (pc->device == dev) return DG_OK;
  DG_CHECK(pc->device < 0, DG_EINVAL, "parcsr: used on a second device");
  DG_TRY(upload_vec(pc->d_ptr, pc->ptr));
  DG_TRY(upload_vec(pc->d_col, pc->col));
  DG_TRY(upload_vec(pc->d_val, pc->val));
  DG_TRY(upload_vec(pc->d_val32, std::vector<float>(pc->val.begin(), pc->val.end())));
  DG_TRY(upload_vec(pc->d_send_idx, pc->send_idx));
  pc->device = dev;
  return DG_OK;
}

dg_status dg_parcsr_pack(dg_parcsr* pc, const double* x_own, double* send, void* stream) {
  DG_CHECK(pc && (pc->send_idx.empty() || (x_own && send)), DG_EINVAL, "parcsr_pack: bad arguments");
  DG_TRY(parcsr_device(pc));
  const int64_t n = int64_t(pc->send_idx.size());
  if (n == 0) return DG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  halo_gather<<<dg::grid_for(n, kHaloThreads), kHaloThreads, 0, s>>>(pc->d_send_idx.p, n, 1, x_own, send);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dg_parcsr_apply(dg_parcsr* pc, const double* x_own, const double* x_ghost, double* y, int add,
                          void* stream) {
  DG_CHECK(pc && (pc->nrow == 0 || y) && (pc->ncol_own == 0 || x_own) && (pc->ghosts.empty() || x_ghost), DG_EINVAL,
           "parcsr_apply: bad arguments");
  DG_TRY(parcsr_device(pc));
  if (pc->nrow == 0) return DG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  parcsr_spmv<<<dg::grid_for(pc->nrow, kHaloThreads), kHaloThreads, 0, s>>>(
      pc->d_ptr.p, pc->d_col.p, pc->d_val.p, pc->nrow, pc->ncol_own, x_own, x_ghost, y, add);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dg_parcsr_pack_f32(dg_parcsr* pc, const float* x_own, float* send, void* stream) {
  DG_CHECK(pc && (pc->send_idx.empty() || (x_own && send)), DG_EINVAL, "parcsr_pack_f32: bad arguments");
  DG_TRY(parcsr_device(pc));
  const int64_t n = int64_t(pc->send_idx.size());
  if (n == 0) return DG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  halo_gather<<<dg::grid_for(n, kHaloThreads), kHaloThreads, 0, s>>>(pc->d_send_idx.p, n, 1, x_own, send);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dg_parcsr_apply_f32(dg_parcsr* pc, const float* x_own, const float* x_ghost, float* y, int add,
                              void* stream) {
  DG_CHECK(pc && (pc->nrow == 0 || y) && (pc->ncol_own == 0 || x_own) && (pc->ghosts.empty() || x_ghost), DG_EINVAL,
           "parcsr_apply_f32: bad arguments");
  DG_TRY(parcsr_device(pc));
  if (pc->nrow == 0) return DG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  parcsr_spmv<<<dg::grid_for(pc->nrow, kHaloThreads), kHaloThreads, 0, s>>>(
      pc->d_ptr.p, pc->d_col.p, pc->d_val32.p, pc->nrow, pc->ncol_own, x_own, x_ghost, y, add);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

void dg_parcsr_destroy(dg_parcsr* pc) { delete pc; }

dg_status dg_vec_jacobi_update(double* x, const double* b, const double* ax, const double* dinv, double omega,
                               int64_t n, void* stream) {
  DG_CHECK(n >= 0 && (n == 0 || (x && b && ax && dinv)), DG_EINVAL, "vec_jacobi_update: bad arguments");
  if (n == 0) return DG_OK;
  jacobi_update<<<dg::grid_for(n, kHaloThreads), kHaloThreads, 0, static_cast<cudaStream_t>(stream)>>>(x, b, ax, dinv,
                                                                                                     omega, n);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dg_vec_jacobi_update_f32(float* x, const float* b, const float* ax, const float* dinv, float omega,
                                   int64_t n, void* stream) {
  DG_CHECK(n >= 0 && (n == 0 || (x && b && ax && dinv)), DG_EINVAL, "vec_jacobi_update_f32: bad arguments");
  if (n == 0) return DG_OK;
  jacobi_update<<<dg::grid_for(n, kHaloThreads), kHaloThreads, 0, static_cast<cudaStream_t>(stream)>>>(x, b, ax, dinv,
                                                                                                     omega, n);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // extern "C"
