// Ensembles of independent samples (batched, one launch per pipeline phase for all samples).
//
// An ensemble is the disjoint union of the samples' meshes: sample s owns the nodes
// [off_s, off_(s+1)) and the tetrahedra that reference them.  Every FEM operator, both Poisson
// solves and all LLG kernels run on the union unchanged: the union's operators are block
// diagonal, so the samples never couple (the AMG's coarsest level keeps one null vector per
// connected component, amg_setup.cpp).  Only the boundary operator must be built per sample,
// because the double layer of the union would couple every boundary to every other:
//   B = blockdiag(B_s),  B_s = Lindholm operator of sample s's own boundary triangles.
// Samples with Nb_s <= dense_max_nb keep a dense block; a single launch applies all dense
// blocks (a warp per boundary row over the concatenated rows, ragged row lengths).  Larger
// samples get an H-matrix built on the sample's own boundary; these are concatenated into
// one block-diagonal H-matrix (hmat_merge) applied by one k_hgather / k_far_z / k_rows
// sequence for all of them, the boundary gather / scatter fused through an index map.
#include <algorithm>

#include "fem.cuh"

namespace spx {

namespace {

template <class TM>
__global__ void k_to_tm(int64_t n, const double* __restrict__ src, TM* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = static_cast<TM>(src[i]);
}

template <class TV>
__global__ void k_gather_b(int64_t n, const int32_t* __restrict__ idx, const TV* __restrict__ src,
                           TV* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

template <class TV>
__global__ void k_scatter_rows(int64_t n, const int32_t* __restrict__ idx, const TV* __restrict__ src,
                               TV* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[idx[i]] = src[i];
}

// warp per dense boundary row r (concatenated over the dense samples):
// g = B_s[i, :] . xb[b0_s : b0_s + nb_s],  gB[b0_s + i] = g,  phi[bverts[b0_s + i]] = u1 + g
template <class TV, class TM>
__global__ void __launch_bounds__(256) k_block_gemv(int64_t nrows, int ndense, const int64_t* __restrict__ row0,
                                                    const int64_t* __restrict__ b0, const int64_t* __restrict__ nbv,
                                                    const int64_t* __restrict__ off, const TM* __restrict__ pool,
                                                    const TV* __restrict__ xb, const int32_t* __restrict__ bverts,
                                                    const TV* __restrict__ u1, TV* __restrict__ phi,
                                                    TV* __restrict__ gB) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t r = w; r < nrows; r += nw) {
    int lo = 0, hi = ndense;  // row0[lo] <= r < row0[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (row0[mid] <= r) lo = mid;
      else hi = mid;
    }
    const int64_t i = r - row0[lo], n = nbv[lo], base = b0[lo];
    const TM* row = pool + off[lo] + i * n;
    const TV* x = xb + base;
    double acc0 = 0.0, acc1 = 0.0;
    int64_t j = lane;
    for (; j + 32 < n; j += 64) {
      acc0 += static_cast<double>(row[j]) * static_cast<double>(x[j]);
      acc1 += static_cast<double>(row[j + 32]) * static_cast<double>(x[j + 32]);
    }
    if (j < n) acc0 += static_cast<double>(row[j]) * static_cast<double>(x[j]);
    const double g = warp_sum(acc0 + acc1);
    if (lane == 0) {
      const TV y = static_cast<TV>(g);
      gB[base + i] = y;
      const int32_t v = bverts[base + i];
      phi[v] = u1[v] + y;
    }
  }
}

}  // namespace

int64_t BlockBoundary::device_bytes() const {
  int64_t t = static_cast<int64_t>(pool.bytes() + d_row0.bytes() + d_b0.bytes() + d_nb.bytes() + d_off.bytes());
  for (const auto& h : H)
    if (h) t += h->device_bytes();
  if (Hm) t += Hm->device_bytes() + static_cast<int64_t>(hidx.bytes() + hmap.bytes() + gbh.bytes());
  return t;
}

template <class TM>
void block_boundary_build(BlockBoundary& bb, const BoundaryDev& bd, const double* X, int64_t N, const int32_t* tets,
                          int64_t E, const DemagOptions& o, cudaStream_t s) {
  const std::vector<int64_t>& off = o.sample_offsets;
  const int64_t ns = static_cast<int64_t>(off.size()) - 1;
  SPX_CHECK(ns >= 1 && off.front() == 0 && off.back() == N, "sample offsets must run from 0 to N");
  for (int64_t k = 0; k < ns; ++k) SPX_CHECK(off[k] < off[k + 1], "every sample needs at least one node");
  const std::vector<int32_t>& bv = bd.host.bverts;
  bb.nsamples = ns;
  bb.b0.assign(ns, 0);
  bb.nb.assign(ns, 0);
  bb.dense.assign(ns, 0);
  bb.H.clear();
  bb.H.resize(ns);
  for (int64_t k = 0; k < ns; ++k) {
    const auto lo = std::lower_bound(bv.begin(), bv.end(), static_cast<int32_t>(off[k]));
    const auto hi = std::lower_bound(bv.begin(), bv.end(), static_cast<int32_t>(off[k + 1]));
    bb.b0[k] = lo - bv.begin();
    bb.nb[k] = hi - lo;
    SPX_CHECK(bb.nb[k] > 0, "a sample has no boundary");
    bb.dense[k] = bb.nb[k] <= o.dense_max_nb ? 1 : 0;
  }
  // tetrahedra per sample (a tetrahedron belongs to the sample of its vertices)
  std::vector<std::vector<int32_t>> stets(ns);
  for (int64_t e = 0; e < E; ++e) {
    const int32_t v0 = tets[4 * e];
    const int64_t k = std::upper_bound(off.begin(), off.end(), static_cast<int64_t>(v0)) - off.begin() - 1;
    for (int q = 0; q < 4; ++q)
      SPX_CHECK(tets[4 * e + q] >= off[k] && tets[4 * e + q] < off[k + 1], "a tetrahedron spans two samples");
    if (!bb.dense[k])
      for (int q = 0; q < 4; ++q) stets[k].push_back(static_cast<int32_t>(tets[4 * e + q] - off[k]));
  }
  // dense blocks: B_s = fill(rows_s, rows_s) + diag(Omega/4pi - 1), stored in TM
  std::vector<int64_t> row0(1, 0), db0, dnb, doff;
  int64_t pos = 0;
  for (int64_t k = 0; k < ns; ++k)
    if (bb.dense[k]) {
      db0.push_back(bb.b0[k]);
      dnb.push_back(bb.nb[k]);
      doff.push_back(pos);
      pos += bb.nb[k] * bb.nb[k];
      row0.push_back(row0.back() + bb.nb[k]);
    }
  bb.ndense = static_cast<int64_t>(db0.size());
  bb.dense_rows = row0.back();
  bb.dense_entries = pos;
  bb.pool.alloc(std::max<int64_t>(pos, 1) * sizeof(TM));
  if (bb.ndense) {
    int64_t maxnb = 0;
    for (int64_t v : dnb) maxnb = std::max(maxnb, v);
    DevBuf<double> tmp(static_cast<size_t>(maxnb * maxnb));
    DevBuf<int32_t> rows(static_cast<size_t>(maxnb));
    std::vector<int32_t> hr(maxnb);
    for (int64_t q = 0; q < bb.ndense; ++q) {
      const int64_t n = dnb[q];
      for (int64_t i = 0; i < n; ++i) hr[i] = static_cast<int32_t>(db0[q] + i);
      SPX_CUDA(cudaMemcpyAsync(rows.p, hr.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
      bd.fill_block(rows.p, n, rows.p, n, tmp.p, s);
      launch_add_diag(n, bd.omega_sum.p + db0[q], tmp.p, s);
      k_to_tm<TM><<<grid_for(n * n, 256), 256, 0, s>>>(n * n, tmp.p, reinterpret_cast<TM*>(bb.pool.p) + doff[q]);
      SPX_LAUNCH_CHECK();
    }
    bb.d_row0.upload(row0, s);
    bb.d_b0.upload(db0, s);
    bb.d_nb.upload(dnb, s);
    bb.d_off.upload(doff, s);
  }
  // H-matrix samples: built on the sample's own boundary
  for (int64_t k = 0; k < ns; ++k) {
    if (bb.dense[k]) continue;
    const int64_t Nk = off[k + 1] - off[k];
    BoundaryDev bk;
    bk.create(X + 3 * off[k], Nk, stets[k].data(), static_cast<int64_t>(stets[k].size() / 4));
    SPX_CHECK(bk.host.Nb == bb.nb[k], "sample boundary differs from its part of the ensemble boundary");
    for (int64_t i = 0; i < bk.host.Nb; ++i)
      SPX_CHECK(bk.host.bverts[i] + off[k] == bv[bb.b0[k] + i], "sample boundary order differs from the ensemble's");
    bb.H[k] = std::make_unique<HMatrix>();
    bb.H[k]->build(bk, o.hcfg, s);
    bb.H[k]->pack(o.hprec, s);
  }
  // one block-diagonal H-matrix for all H-matrix samples
  std::vector<const HMatrix*> parts;
  std::vector<int32_t> hidx, hmap;
  for (int64_t k = 0; k < ns; ++k)
    if (bb.H[k]) {
      parts.push_back(bb.H[k].get());
      for (int64_t i = 0; i < bb.nb[k]; ++i) {
        hidx.push_back(bv[bb.b0[k] + i]);
        hmap.push_back(static_cast<int32_t>(bb.b0[k] + i));
      }
    }
  if (!parts.empty()) {
    bb.Hm = std::make_unique<HMatrix>();
    hmat_merge(parts, *bb.Hm, s);
    bb.hidx.upload(hidx, s);
    bb.hmap.upload(hmap, s);
    bb.gbh.alloc(hidx.size() * sizeof(double));
    for (auto& h : bb.H) h.reset();
  }
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class TV, class TM>
int block_boundary_apply(BlockBoundary& bb, int64_t Nb, const int32_t* bverts, const TV* u1, TV* xb, TV* phi, TV* gB,
                         cudaStream_t s) {
  int launches = 0;
  if (bb.ndense) {
    k_gather_b<TV><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, bverts, u1, xb);
    SPX_LAUNCH_CHECK();
    const unsigned g = static_cast<unsigned>(std::min<int64_t>((bb.dense_rows + 7) / 8, 148 * 16));
    k_block_gemv<TV, TM><<<g, 256, 0, s>>>(bb.dense_rows, static_cast<int>(bb.ndense), bb.d_row0.p, bb.d_b0.p,
                                           bb.d_nb.p, bb.d_off.p, reinterpret_cast<const TM*>(bb.pool.p), xb, bverts,
                                           u1, phi, gB);
    SPX_LAUNCH_CHECK();
    launches += 2;
  }
  if (bb.Hm) {
    TV* yh = reinterpret_cast<TV*>(bb.gbh.p);
    bb.Hm->apply_gather<TV>(u1, bb.hidx.p, phi, u1, yh, s);
    const int64_t nh = bb.Hm->Nb;
    k_scatter_rows<TV><<<grid_for(nh, 256), 256, 0, s>>>(nh, bb.hmap.p, yh, gB);
    SPX_LAUNCH_CHECK();
    launches += (bb.Hm->nunits > 0 ? 3 : 2) + 1;
  }
  return launches;
}

template void block_boundary_build<double>(BlockBoundary&, const BoundaryDev&, const double*, int64_t, const int32_t*,
                                           int64_t, const DemagOptions&, cudaStream_t);
template void block_boundary_build<float>(BlockBoundary&, const BoundaryDev&, const double*, int64_t, const int32_t*,
                                          int64_t, const DemagOptions&, cudaStream_t);
template int block_boundary_apply<double, double>(BlockBoundary&, int64_t, const int32_t*, const double*, double*,
                                                  double*, double*, cudaStream_t);
template int block_boundary_apply<float, float>(BlockBoundary&, int64_t, const int32_t*, const float*, float*, float*,
                                                float*, cudaStream_t);
template int block_boundary_apply<double, float>(BlockBoundary&, int64_t, const int32_t*, const double*, double*,
                                                 double*, double*, cudaStream_t);

}  // namespace spx
