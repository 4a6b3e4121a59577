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
  H.recompressed = false;
  H.sigma.clear();
  if (c.recompress) H.recompress(s);
  H.pack(p, s);
}

namespace {
template <class T>
std::vector<T> download(const DevBuf<T>& b) {
  std::vector<T> h(b.n);
  if (b.n) SPX_CUDA(cudaMemcpy(h.data(), b.p, b.n * sizeof(T), cudaMemcpyDeviceToHost));
  return h;
}
size_t factor_bytes(Prec p) { return p == Prec::F64 ? 8 : (p == Prec::F32 ? 4 : 2); }
size_t tile_bytes(Prec p) { return p == Prec::F64 ? 8 : 4; }
}  // namespace

// Block-diagonal concatenation of packed H-matrices (ensembles): the boundary index space,
// the permuted space, the factor and tile pools, the far-field z vectors and partial sums,
// the groups, the k_far_z warps and the row segments of part k follow those of parts < k,
// so one apply (k_hgather, k_far_z, k_rows) serves all parts.  Only the apply-side data is
// merged (no tree, no FP64 pools: the result cannot be repacked or transposed).
void hmat_merge(const std::vector<const HMatrix*>& parts, HMatrix& M, cudaStream_t s) {
  SPX_CHECK(!parts.empty(), "nothing to merge");
  const Prec p = parts[0]->prec;
  const size_t fb = factor_bytes(p), nbt = tile_bytes(p);
  std::vector<int32_t> perm, warp_first(1, 0), seg_start;
  std::vector<double> diag;
  std::vector<FarUnit> units;
  std::vector<FarGroup> groups;
  std::vector<int64_t> item_ptr(1, 0), near_begin;
  std::vector<RowItem> items;
  int64_t c0 = 0, z0 = 0, zp0 = 0, g0 = 0, u0 = 0, i0 = 0, fbytes = 0, nbytes = 0, nwarps = 0;
  std::vector<int64_t> foff, noff;
  for (const HMatrix* H : parts) {
    SPX_CHECK(H->packed && H->prec == p, "merged H-matrices must be packed in the same precision");
    SPX_CHECK(p != Prec::SPLIT, "the f32/f16 split packing is not available for merged (ensemble) H-matrices");
    foff.push_back(fbytes);
    noff.push_back(nbytes);
    fbytes += ((static_cast<int64_t>(H->far_f.n) + 255) / 256) * 256;
    nbytes += ((static_cast<int64_t>(H->near_f.n) + 255) / 256) * 256;
  }
  M.far_f.alloc(std::max<int64_t>(fbytes, 1));
  M.near_f.alloc(std::max<int64_t>(nbytes, 1));
  for (size_t k = 0; k < parts.size(); ++k) {
    const HMatrix& H = *parts[k];
    const int64_t F = foff[k] / static_cast<int64_t>(fb), Nn = noff[k] / static_cast<int64_t>(nbt);
    if (H.far_f.n)
      SPX_CUDA(cudaMemcpyAsync(M.far_f.p + foff[k], H.far_f.p, H.far_f.n, cudaMemcpyDeviceToDevice, s));
    if (H.near_f.n)
      SPX_CUDA(cudaMemcpyAsync(M.near_f.p + noff[k], H.near_f.p, H.near_f.n, cudaMemcpyDeviceToDevice, s));
    for (int32_t v : download(H.perm)) perm.push_back(static_cast<int32_t>(v + c0));
    for (double v : download(H.diag_perm)) diag.push_back(v);
    for (FarUnit U : download(H.units)) {
      U.voff += F;
      U.xc += static_cast<int32_t>(c0);
      U.zout += static_cast<int32_t>((U.flags & 3) == 2 ? zp0 : z0);
      if (U.grp >= 0) U.grp += static_cast<int32_t>(g0);
      units.push_back(U);
    }
    for (FarGroup G : download(H.groups)) {
      G.pbase += static_cast<int32_t>(zp0);
      G.zdst += static_cast<int32_t>(z0);
      groups.push_back(G);
    }
    const std::vector<int32_t> wf = download(H.warp_first);
    for (int64_t w = 0; w < H.nwarps_z; ++w) warp_first.push_back(static_cast<int32_t>(wf[w + 1] + u0));
    const std::vector<int32_t> ss = download(H.seg_start);
    const std::vector<int64_t> ip = download(H.item_ptr), nb = download(H.near_begin);
    const std::vector<RowItem> it = download(H.items);
    for (int64_t g = 0; g < H.nseg; ++g) {
      seg_start.push_back(static_cast<int32_t>(ss[g] + c0));
      near_begin.push_back(nb[g] + i0);
      for (int64_t q = ip[g]; q < ip[g + 1]; ++q) {
        RowItem r = it[q];
        if (q < nb[g]) {  // far: U tile, scaled by z
          r.off += F;
          r.src += static_cast<int32_t>(z0);
        } else {  // near: tile, scaled by x~
          r.off += Nn;
          r.src += static_cast<int32_t>(c0);
        }
        items.push_back(r);
      }
      item_ptr.push_back(static_cast<int64_t>(items.size()));
    }
    c0 += H.Nb;
    z0 += H.zlen;
    zp0 += H.zpart_len;
    g0 += static_cast<int64_t>(H.groups.n);
    u0 += H.nunits;
    i0 += static_cast<int64_t>(it.size());
    nwarps += H.nwarps_z;
    M.n_far += H.n_far;
    M.n_near += H.n_near;
    M.bytes_far += H.bytes_far;
    M.bytes_near += H.bytes_near;
  }
  SPX_CHECK(z0 < (int64_t(1) << 31) && zp0 < (int64_t(1) << 31) && c0 < (int64_t(1) << 31),
            "merged H-matrix too large for 32-bit indices");
  seg_start.push_back(static_cast<int32_t>(c0));
  M.device = parts[0]->device;
  M.Nb = c0;
  M.prec = p;
  M.perm.upload(perm, s);
  M.diag_perm.upload(diag, s);
  M.units.upload(units, s);
  M.warp_first.upload(warp_first, s);
  M.groups.upload(groups, s);
  M.gcnt.alloc(std::max<size_t>(groups.size(), 1));
  M.gcnt.zero(s);
  M.seg_start.upload(seg_start, s);
  M.item_ptr.upload(item_ptr, s);
  M.near_begin.upload(near_begin, s);
  M.items.upload(items, s);
  M.nseg = static_cast<int64_t>(seg_start.size()) - 1;
  M.zlen = z0;
  M.zpart_len = zp0;
  M.nunits = u0;
  M.nwarps_z = nwarps;
  M.packed = true;
  SPX_CUDA(cudaStreamSynchronize(s));
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
  // the split packing scales the columns of U by their singular values, which the transpose
  // moves to V: the transpose of a split-packed matrix is packed in FP32
  T->pack(prec == Prec::SPLIT ? Prec::F32 : prec, s);
  tr = std::move(T);
  return *tr;
}

}  // namespace spx
