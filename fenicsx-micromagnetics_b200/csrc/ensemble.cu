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
// samples get an H-matrix built on the sample's own boundary; samples of the same geometry
// (coordinates equal up to a translation, same tetrahedra) share one H-matrix applied to all
// of them at once (HMatrix::apply_multi, every factor read once per batch of states), and
// the remaining ones are concatenated into one block-diagonal H-matrix (hmat_merge) applied
// by one k_hgather / k_far_z / k_rows sequence, the boundary gather / scatter fused through
// an index map.
#include <algorithm>

#include "fem.cuh"

namespace spx {

namespace {

// n x n FP64 block -> rows of ld TM entries (zero padded)
template <class TM>
__global__ void k_to_tm(int64_t n, int64_t ld, const double* __restrict__ src, TM* __restrict__ dst) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * ld) return;
  const int64_t i = t / ld, j = t % ld;
  dst[t] = j < n ? static_cast<TM>(src[i * n + j]) : TM(0);
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

// row stride of a dense block: the row length rounded up to 16 bytes (zero padding)
template <class TM>
constexpr int64_t block_ld(int64_t n) {
  return (n + (16 / sizeof(TM)) - 1) / (16 / sizeof(TM)) * (16 / sizeof(TM));
}

template <class TM> struct Vec16;
template <> struct Vec16<float> { using T = float4; static constexpr int E = 4; };
template <> struct Vec16<double> { using T = double2; static constexpr int E = 2; };
__device__ __forceinline__ void vec_elems(const float4& v, double e[4]) { e[0] = v.x; e[1] = v.y; e[2] = v.z; e[3] = v.w; }
__device__ __forceinline__ void vec_elems(const double2& v, double e[2]) { e[0] = v.x; e[1] = v.y; }

// CTA per tile of up to TILE_ROWS rows of one dense sample: the sample's boundary vector x
// is staged in shared memory (FP64, nb_s <= dense_max_nb entries), then each warp streams
// its rows of B_s as 16-byte vectors (rows padded to 16 bytes, four vectors in flight per
// lane):  g = B_s[i, :] . x,  gB[b0_s + i] = g,  phi[bverts[b0_s + i]] = u1 + g.
constexpr int TILE_ROWS = 64;
template <class TV, class TM>
__global__ void __launch_bounds__(256) k_block_gemv(const int32_t* __restrict__ tiles, const int64_t* __restrict__ b0,
                                                    const int64_t* __restrict__ nbv, const int64_t* __restrict__ off,
                                                    const TM* __restrict__ pool, const TV* __restrict__ xb,
                                                    const int32_t* __restrict__ bverts, const TV* __restrict__ u1,
                                                    TV* __restrict__ phi, TV* __restrict__ gB) {
  extern __shared__ double xs[];
  using VT = typename Vec16<TM>::T;
  constexpr int E = Vec16<TM>::E;
  const int q = tiles[2 * blockIdx.x], i0 = tiles[2 * blockIdx.x + 1];
  const int64_t n = nbv[q], base = b0[q];
  const int64_t nv = block_ld<TM>(n) / E;
  for (int64_t j = threadIdx.x; j < nv * E; j += blockDim.x) xs[j] = j < n ? static_cast<double>(xb[base + j]) : 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int64_t i1 = std::min<int64_t>(n, i0 + TILE_ROWS);
  for (int64_t i = i0 + wid; i < i1; i += nwarp) {
    const VT* row = reinterpret_cast<const VT*>(pool + off[q] + i * nv * E);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    int64_t v = lane;
    for (; v + 96 < nv; v += 128) {
      VT w[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) w[t] = __ldcs(row + v + 32 * t);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        double e[E];
        vec_elems(w[t], e);
        const double* xv = xs + (v + 32 * t) * E;  // padding entries of B are zero
#pragma unroll
        for (int u = 0; u < E; ++u) acc[t] += e[u] * xv[u];
      }
    }
    for (; v < nv; v += 32) {
      double e[E];
      vec_elems(__ldcs(row + v), e);
      const int64_t c = v * E;
#pragma unroll
      for (int u = 0; u < E; ++u)
        if (c + u < n) acc[0] += e[u] * xs[c + u];
    }
    const double g = warp_sum((acc[0] + acc[1]) + (acc[2] + acc[3]));
    if (lane == 0) {
      const TV y = static_cast<TV>(g);
      gB[base + i] = y;
      const int32_t vtx = bverts[base + i];
      phi[vtx] = u1[vtx] + y;
    }
  }
}

}  // namespace

int64_t BlockBoundary::device_bytes() const {
  int64_t t = static_cast<int64_t>(pool.bytes() + d_tiles.bytes() + d_b0.bytes() + d_nb.bytes() + d_off.bytes());
  for (const auto& h : H)
    if (h) t += h->device_bytes();
  if (Hm) t += Hm->device_bytes() + static_cast<int64_t>(hidx.bytes() + hmap.bytes() + gbh.bytes());
  for (const auto& sh : shared) t += sh.H->device_bytes();
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
  SPX_CHECK(o.dense_max_nb <= 27000, "dense_max_nb above 27000 (the staged boundary vector must fit in 216 KB of "
                                     "shared memory); larger samples use H-matrices");
  std::vector<int64_t> db0, dnb, doff;
  std::vector<int32_t> tiles;
  int64_t pos = 0, entries = 0, rows = 0;
  for (int64_t k = 0; k < ns; ++k)
    if (bb.dense[k]) {
      db0.push_back(bb.b0[k]);
      dnb.push_back(bb.nb[k]);
      doff.push_back(pos);
      pos += bb.nb[k] * block_ld<TM>(bb.nb[k]);
      entries += bb.nb[k] * bb.nb[k];
      rows += bb.nb[k];
      for (int64_t i0 = 0; i0 < bb.nb[k]; i0 += TILE_ROWS) {
        tiles.push_back(static_cast<int32_t>(db0.size() - 1));
        tiles.push_back(static_cast<int32_t>(i0));
      }
      bb.max_ld = std::max<int64_t>(bb.max_ld, block_ld<TM>(bb.nb[k]));
    }
  bb.ndense = static_cast<int64_t>(db0.size());
  bb.dense_rows = rows;
  bb.ntiles = static_cast<int64_t>(tiles.size() / 2);
  bb.dense_entries = entries;  // algorithmic (rows are stored padded to 16 bytes)
  bb.pool.alloc(std::max<int64_t>(pos, 1) * sizeof(TM));
  if (bb.ndense) {
    int64_t maxnb = 0;
    for (int64_t v : dnb) maxnb = std::max(maxnb, v);
    DevBuf<double> tmp(static_cast<size_t>(maxnb * maxnb));
    DevBuf<int32_t> rows_d(static_cast<size_t>(maxnb));
    std::vector<int32_t> hr(maxnb);
    for (int64_t q = 0; q < bb.ndense; ++q) {
      const int64_t n = dnb[q];
      for (int64_t i = 0; i < n; ++i) hr[i] = static_cast<int32_t>(db0[q] + i);
      SPX_CUDA(cudaMemcpyAsync(rows_d.p, hr.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
      bd.fill_block(rows_d.p, n, rows_d.p, n, tmp.p, s);
      launch_add_diag(n, bd.omega_sum.p + db0[q], tmp.p, s);
      const int64_t ld = block_ld<TM>(n);
      k_to_tm<TM><<<grid_for(n * ld, 256), 256, 0, s>>>(n, ld, tmp.p, reinterpret_cast<TM*>(bb.pool.p) + doff[q]);
      SPX_LAUNCH_CHECK();
    }
    bb.d_tiles.upload(tiles, s);
    bb.d_b0.upload(db0, s);
    bb.d_nb.upload(dnb, s);
    bb.d_off.upload(doff, s);
  }
  // H-matrix samples with the same geometry (node coordinates up to a translation, same
  // tetrahedra) share one H-matrix applied to all of them at once (HMatrix::apply_multi)
  std::vector<int64_t> group_of(ns, -1);
  std::vector<int64_t> reps;
  for (int64_t k = 0; k < ns; ++k) {
    if (bb.dense[k]) continue;
    const int64_t Nk = off[k + 1] - off[k];
    for (size_t g = 0; g < reps.size() && group_of[k] < 0; ++g) {
      const int64_t r = reps[g];
      if (off[r + 1] - off[r] != Nk || stets[r] != stets[k]) continue;
      bool same = true;
      for (int64_t i = 0; i < Nk && same; ++i)
        for (int c = 0; c < 3 && same; ++c)
          same = (X[3 * (off[k] + i) + c] - X[3 * off[k] + c]) == (X[3 * (off[r] + i) + c] - X[3 * off[r] + c]);
      if (same) group_of[k] = static_cast<int64_t>(g);
    }
    if (group_of[k] < 0) {
      group_of[k] = static_cast<int64_t>(reps.size());
      reps.push_back(k);
    }
  }
  std::vector<std::vector<int64_t>> members(reps.size());
  for (int64_t k = 0; k < ns; ++k)
    if (group_of[k] >= 0) members[group_of[k]].push_back(k);
  // H-matrix samples: built on the sample's own boundary (one per group)
  for (int64_t k = 0; k < ns; ++k) {
    if (bb.dense[k] || reps[group_of[k]] != k) continue;
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
  // groups of several samples: one H-matrix, all members in one multi-state apply
  for (size_t g = 0; g < reps.size(); ++g)
    if (members[g].size() > 1) {
      BlockBoundary::Shared sh;
      sh.H = std::move(bb.H[reps[g]]);
      for (int64_t k : members[g]) sh.b0.push_back(bb.b0[k]);
      bb.shared.push_back(std::move(sh));
    }
  // one block-diagonal H-matrix for the remaining (single) H-matrix samples
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
    const size_t smem = static_cast<size_t>(bb.max_ld) * sizeof(double);
    if (smem > 48 * 1024)
      SPX_CUDA(cudaFuncSetAttribute(k_block_gemv<TV, TM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    k_block_gemv<TV, TM><<<static_cast<unsigned>(bb.ntiles), 256, smem, s>>>(
        bb.d_tiles.p, bb.d_b0.p, bb.d_nb.p, bb.d_off.p, reinterpret_cast<const TM*>(bb.pool.p), xb, bverts, u1, phi,
        gB);
    SPX_LAUNCH_CHECK();
    launches += 2;
  }
  for (auto& sh : bb.shared) {
    const int R = static_cast<int>(sh.b0.size());
    sh.H->apply_multi<TV>(u1, bverts, sh.b0.data(), phi, u1, gB, sh.b0.data(), R, s);
    launches += ((R + 7) / 8) * (sh.H->nunits > 0 ? 3 : 2);
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
