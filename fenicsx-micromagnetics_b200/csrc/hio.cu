// H-matrix contents to and from the reference's cache representation
// (HMatrixCPUData, lindholm_hmatrix_gpu/storage.py:29-325):
//   perm (Nb), diag_jump (Nb, original order), near field as CSR in permutation space with
//   exact zeros dropped, far blocks as (row/col start/stop, rank) with U (m x k) and V (k x n)
//   row-major FP64 factors and their ACA relative residual.
// The npz file itself is written and read by the Python layer (numpy); this file moves the
// arrays between the host and the device pools of an HMatrix.
//
// Transpose (HMatrix::transposed): B^T has the same cluster tree and the transposed block
// partition.  A far block U V (U: m x k, V: k x n) becomes V^T U^T, whose "U^T" is V (k x n,
// already stored) and whose "V" is U^T (k x m, already stored): the far pool is copied as is
// and only the offsets swap.  Near tiles are transposed element by element.
//
// Import: the cluster tree is rebuilt from the boundary points (bit-exact), and the cached
// permutation must equal it.  Far blocks keep their ranges; the near CSR is split into dense
// leaf x leaf tiles (every tile row and column range is a leaf cluster), which is all the
// apply-side packing needs.
#include <algorithm>
#include <cstring>
#include <unordered_map>

#include "hmat.cuh"

namespace spx {

void hmat_near_csr(const HMatrix& H, std::vector<int32_t>& indptr, std::vector<int32_t>& indices,
                   std::vector<double>& data) {
  const int64_t Nb = H.Nb;
  std::vector<double> pool(H.near_pool64.n);
  if (!pool.empty())
    SPX_CUDA(cudaMemcpy(pool.data(), H.near_pool64.p, pool.size() * sizeof(double), cudaMemcpyDeviceToHost));
  // rows of the near blocks, each block contributing its nonzero columns in order
  std::vector<std::vector<int32_t>> rows_of(Nb);
  for (size_t bi = 0; bi < H.blocks.size(); ++bi)
    if (H.blocks[bi].type == 0)
      for (int32_t r = H.blocks[bi].rs; r < H.blocks[bi].re; ++r) rows_of[r].push_back(static_cast<int32_t>(bi));
  indptr.assign(Nb + 1, 0);
  indices.clear();
  data.clear();
  std::vector<std::pair<int32_t, double>> row;
  for (int64_t r = 0; r < Nb; ++r) {
    row.clear();
    for (int32_t bi : rows_of[r]) {
      const HBlock& b = H.blocks[bi];
      const int32_t n = b.ce - b.cs;
      const double* src = pool.data() + b.off_u + static_cast<int64_t>(r - b.rs) * n;
      for (int32_t c = 0; c < n; ++c)
        if (src[c] != 0.0) row.push_back({b.cs + c, src[c]});
    }
    std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (const auto& e : row) {
      indices.push_back(e.first);
      data.push_back(e.second);
    }
    SPX_CHECK(indices.size() < (size_t(1) << 31), "near field has more than 2^31 nonzeros");
    indptr[r + 1] = static_cast<int32_t>(indices.size());
  }
}

void hmat_far_sizes(const HMatrix& H, int64_t& nfar, int64_t& u_entries, int64_t& v_entries) {
  nfar = u_entries = v_entries = 0;
  for (const HBlock& b : H.blocks)
    if (b.type == 1) {
      ++nfar;
      u_entries += static_cast<int64_t>(b.re - b.rs) * b.rank;
      v_entries += static_cast<int64_t>(b.rank) * (b.ce - b.cs);
    }
}

void hmat_export_far(const HMatrix& H, int64_t* meta5, double* relres, double* U, double* V) {
  int64_t f = 0, uo = 0, vo = 0;
  std::vector<double> ut;
  for (const HBlock& b : H.blocks) {
    if (b.type != 1) continue;
    const int64_t m = b.re - b.rs, n = b.ce - b.cs, k = b.rank;
    if (meta5) {
      meta5[5 * f + 0] = b.rs;
      meta5[5 * f + 1] = b.re;
      meta5[5 * f + 2] = b.cs;
      meta5[5 * f + 3] = b.ce;
      meta5[5 * f + 4] = k;
    }
    if (relres) relres[f] = b.relres;
    if (U && k * m > 0) {  // pool holds U^T (k x m); the cache holds U (m x k)
      ut.resize(k * m);
      SPX_CUDA(cudaMemcpy(ut.data(), H.far_pool64.p + b.off_u, k * m * sizeof(double), cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < m; ++i)
        for (int64_t q = 0; q < k; ++q) U[uo + i * k + q] = ut[q * m + i];
    }
    if (V && k * n > 0)
      SPX_CUDA(cudaMemcpy(V + vo, H.far_pool64.p + b.off_v, k * n * sizeof(double), cudaMemcpyDeviceToHost));
    uo += k * m;
    vo += k * n;
    ++f;
  }
}

void hmat_import(HMatrix& H, const BoundaryDev& bd, const HBuildConfig& c, Prec p, int64_t nfar, const int64_t* meta5,
                 const double* relres, const double* U, const double* V, const int32_t* indptr,
                 const int32_t* indices, const double* data, const int32_t* perm_in, const double* diag_jump,
                 cudaStream_t s) {
  SPX_CUDA(cudaGetDevice(&H.device));
  H.cfg = c;
  H.Nb = bd.host.Nb;
  const int64_t Nb = H.Nb;
  build_cluster_tree(bd.host.Xb.data(), Nb, c.leaf_size, H.tree);
  if (perm_in)
    SPX_CHECK(std::equal(H.tree.perm.begin(), H.tree.perm.end(), perm_in),
              "cached permutation differs from this geometry's cluster tree (other mesh or leaf size)");
  H.perm.upload(H.tree.perm, s);
  {
    std::vector<double> dj(Nb);
    for (int64_t i = 0; i < Nb; ++i) {
      const int32_t o = H.tree.perm[i];
      dj[i] = diag_jump ? diag_jump[o] : bd.host.omega_sum[o] / (4.0 * 3.141592653589793) - 1.0;
    }
    H.diag_perm.upload(dj, s);
  }
  H.stats = HStats{};
  H.blocks.clear();
  // far blocks: U (m x k) -> U^T (k x m) in the FP64 pool, V as is
  int64_t fpos = 0;
  for (int64_t f = 0; f < nfar; ++f) {
    const int64_t rs = meta5[5 * f], re = meta5[5 * f + 1], cs = meta5[5 * f + 2], ce = meta5[5 * f + 3],
                  k = meta5[5 * f + 4];
    SPX_CHECK(0 <= rs && rs < re && re <= Nb && 0 <= cs && cs < ce && ce <= Nb && k >= 0 && k <= std::min(re - rs, ce - cs),
              "far block out of range");
    fpos += k * ((re - rs) + (ce - cs));
  }
  H.far_pool64.alloc(std::max<int64_t>(fpos, 1));
  {
    int64_t uo = 0, vo = 0, pos = 0;
    std::vector<double> ut;
    for (int64_t f = 0; f < nfar; ++f) {
      const int32_t rs = static_cast<int32_t>(meta5[5 * f]), re = static_cast<int32_t>(meta5[5 * f + 1]);
      const int32_t cs = static_cast<int32_t>(meta5[5 * f + 2]), ce = static_cast<int32_t>(meta5[5 * f + 3]);
      const int32_t k = static_cast<int32_t>(meta5[5 * f + 4]);
      const int64_t m = re - rs, n = ce - cs;
      ut.resize(static_cast<size_t>(k) * m);
      for (int64_t i = 0; i < m; ++i)
        for (int64_t q = 0; q < k; ++q) ut[q * m + i] = U[uo + i * k + q];
      if (k > 0) {
        SPX_CUDA(cudaMemcpy(H.far_pool64.p + pos, ut.data(), ut.size() * sizeof(double), cudaMemcpyHostToDevice));
        SPX_CUDA(cudaMemcpy(H.far_pool64.p + pos + k * m, V + vo, k * n * sizeof(double), cudaMemcpyHostToDevice));
      }
      H.blocks.push_back(HBlock{rs, re, cs, ce, 1, k, pos, pos + k * m, relres ? relres[f] : 0.0});
      H.stats.low_rank_blocks++;
      H.stats.max_observed_rank = std::max<int64_t>(H.stats.max_observed_rank, k);
      H.stats.sum_observed_rank += k;
      H.stats.far_entries += k * (m + n);
      uo += k * m;
      vo += k * n;
      pos += k * (m + n);
    }
  }
  // near field: leaf x leaf dense tiles of the CSR
  std::vector<int32_t> leaf_of(Nb, -1), leaf_start, leaf_stop;
  for (const TreeNode& nd : H.tree.nodes)
    if (nd.leaf()) {
      for (int32_t i = nd.start; i < nd.stop; ++i) leaf_of[i] = static_cast<int32_t>(leaf_start.size());
      leaf_start.push_back(nd.start);
      leaf_stop.push_back(nd.stop);
    }
  const int64_t nleaf = static_cast<int64_t>(leaf_start.size());
  std::unordered_map<int64_t, int64_t> tile_of;
  std::vector<int64_t> keys;
  for (int64_t r = 0; r < Nb; ++r)
    for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) {
      const int32_t j = indices[e];
      SPX_CHECK(j >= 0 && j < Nb, "near column out of range");
      const int64_t key = static_cast<int64_t>(leaf_of[r]) * nleaf + leaf_of[j];
      if (tile_of.emplace(key, 0).second) keys.push_back(key);
    }
  std::sort(keys.begin(), keys.end());
  int64_t npos = 0;
  for (int64_t key : keys) {
    const int64_t lr = key / nleaf, lc = key % nleaf;
    tile_of[key] = npos;
    npos += static_cast<int64_t>(leaf_stop[lr] - leaf_start[lr]) * (leaf_stop[lc] - leaf_start[lc]);
  }
  std::vector<double> near(std::max<int64_t>(npos, 1), 0.0);
  for (int64_t r = 0; r < Nb; ++r)
    for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) {
      const int32_t j = indices[e];
      const int64_t lr = leaf_of[r], lc = leaf_of[j];
      const int64_t n = leaf_stop[lc] - leaf_start[lc];
      near[tile_of[lr * nleaf + lc] + (r - leaf_start[lr]) * n + (j - leaf_start[lc])] += data[e];
    }
  for (int64_t key : keys) {
    const int64_t lr = key / nleaf, lc = key % nleaf;
    H.blocks.push_back(HBlock{leaf_start[lr], leaf_stop[lr], leaf_start[lc], leaf_stop[lc], 0, 0, tile_of[key], 0, 0.0});
    H.stats.dense_blocks++;
    H.stats.near_entries += static_cast<int64_t>(leaf_stop[lr] - leaf_start[lr]) * (leaf_stop[lc] - leaf_start[lc]);
  }
  H.near_pool64.upload(near, s);
  H.stats.n_far = H.stats.low_rank_blocks;
  H.stats.n_near = H.stats.dense_blocks;
  SPX_CUDA(cudaStreamSynchronize(s));
  H.pack(p, s);
}

HMatrix& HMatrix::transposed(cudaStream_t s) {
  if (tr) return *tr;
  SPX_CHECK(packed, "H-matrix is not packed");
  auto T = std::make_unique<HMatrix>();
  T->device = device;
  T->Nb = Nb;
  T->cfg = cfg;
  T->stats = stats;
  T->tree = tree;
  T->perm.upload(tree.perm, s);
  T->diag_perm.alloc(diag_perm.n);
  if (diag_perm.n)
    SPX_CUDA(cudaMemcpyAsync(T->diag_perm.p, diag_perm.p, diag_perm.bytes(), cudaMemcpyDeviceToDevice, s));
  T->far_pool64.alloc(far_pool64.n);
  if (far_pool64.n)
    SPX_CUDA(cudaMemcpyAsync(T->far_pool64.p, far_pool64.p, far_pool64.bytes(), cudaMemcpyDeviceToDevice, s));
  std::vector<double> near(near_pool64.n), neart(near_pool64.n, 0.0);
  if (!near.empty()) {
    SPX_CUDA(cudaMemcpyAsync(near.data(), near_pool64.p, near.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    SPX_CUDA(cudaStreamSynchronize(s));
  }
  T->blocks.reserve(blocks.size());
  for (const HBlock& b : blocks) {
    HBlock t = b;
    t.rs = b.cs; t.re = b.ce; t.cs = b.rs; t.ce = b.re;
    if (b.type == 1) {
      t.off_u = b.off_v;
      t.off_v = b.off_u;
    } else {
      const int64_t m = b.re - b.rs, n = b.ce - b.cs;
      for (int64_t i = 0; i < m; ++i)
        for (int64_t j = 0; j < n; ++j) neart[b.off_u + j * m + i] = near[b.off_u + i * n + j];
    }
    T->blocks.push_back(t);
  }
  T->near_pool64.upload(neart, s);
  SPX_CUDA(cudaStreamSynchronize(s));
  T->pack(prec, s);
  tr = std::move(T);
  return *tr;
}

}  // namespace spx
