// Boundary geometry upload and H-matrix construction on the GPU.
//
// Construction follows HMatrixBuilder (lindholm_hmatrix_gpu/builder.py:186-419):
//   admissible & dense bytes > max_temporary_block_bytes -> subdivide       (:338-341)
//   admissible -> fill, full-pivot ACA (compressors.py:35-99), then
//       accept if rank>0, relres <= eps(1+64 eps) and k(m+n) < 0.95 m n   (:343-356)
//       else subdivide if relres misses eps and a node can split          (:358-366)
//       else store dense                                                   (:368-370)
//   non-admissible leaf pair -> dense; otherwise subdivide the larger-diameter
//   node (:260-275).
// Every decision depends only on its own block, so blocks are processed in waves
// (all candidates of one recursion depth at once) instead of depth-first; the
// resulting partition is the same set of blocks.
//
// Device work per wave: all admissible candidates are filled by the tiled
// Lindholm kernel into a workspace and compressed by a batched ACA:
//   k_aca_update : one fused pass  R -= u v^T ; max|R| (first index on ties) ; ||R||_F^2
//                  over CHUNK-entry slices of every active block
//   k_aca_decide : one CTA per block: reduce the slices, apply the stopping rules of
//                  fullaca_dense, extract the next column u = R[:, j] and row
//                  v = R[i, :] / pivot.
// The residual update uses separately rounded multiply and subtract, as numpy's
// ``residual -= np.outer(u, v)`` does.  A block stops early once (k+1)(m+n) >= 0.95 m n
// with the tolerance unmet: its final rank could only be larger, so it ends up dense
// either way (the ACA reaches the tolerance at the latest at full rank).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "hmat.cuh"

namespace spx {

struct FillDesc {
  int64_t out_off, rows_off, cols_off;
  int32_t m, n;
};

// ------------------------------------------------------------------ boundary upload
void BoundaryDev::create(const double* X, int64_t N, const int32_t* tets, int64_t E) {
  SPX_CUDA(cudaGetDevice(&device));
  build_boundary(X, N, tets, E, host);
  const HostBoundary& h = host;
  SPX_CHECK(h.Nb > 0 && h.Nt > 0, "mesh has no boundary");
  std::vector<double> rec;
  pack_triangles(h, rec);
  std::vector<int32_t> ptr(h.Nb + 1, 0), tri(3 * h.Nt);
  for (int64_t t = 0; t < h.Nt; ++t)
    for (int v = 0; v < 3; ++v) ptr[h.tri_lid[3 * t + v] + 1]++;
  for (int64_t i = 0; i < h.Nb; ++i) {
    maxinc = std::max(maxinc, ptr[i + 1]);
    ptr[i + 1] += ptr[i];
  }
  {
    std::vector<int32_t> cur(ptr.begin(), ptr.end() - 1);
    for (int64_t t = 0; t < h.Nt; ++t)
      for (int v = 0; v < 3; ++v) tri[cur[h.tri_lid[3 * t + v]]++] = static_cast<int32_t>(t);
  }
  Xb.upload(h.Xb);
  T.upload(rec);
  omega_sum.upload(h.omega_sum);
  tri_lid.upload(h.tri_lid);
  inc_ptr.upload(ptr);
  inc_tri.upload(tri);
  bverts.upload(h.bverts);
  SPX_CUDA(cudaDeviceSynchronize());
}

void BoundaryDev::fill_block(const int32_t* rows_dev, int64_t m, const int32_t* cols_dev, int64_t n,
                             double* out, cudaStream_t s) const {
  if (m <= 0 || n <= 0) return;
  FillDesc d{0, 0, 0, static_cast<int32_t>(m), static_cast<int32_t>(n)};
  const int64_t ntiles = ((m + 127) / 128) * ((n + 31) / 32);
  DevBuf<FillDesc> dd(1);
  DevBuf<int64_t> ts(1);
  int64_t zero = 0;
  dd.upload(&d, 1, s);
  ts.upload(&zero, 1, s);
  launch_fill(dd.p, ts.p, 1, ntiles, rows_dev, cols_dev, Xb.p, tri_lid.p, T.p, inc_ptr.p, inc_tri.p,
              maxinc, host.Nb, out, s);
  SPX_CUDA(cudaStreamSynchronize(s));
}

void BoundaryDev::dense_B(double* B, cudaStream_t s) const {
  const int64_t Nb = host.Nb;
  std::vector<int32_t> id(Nb);
  for (int64_t i = 0; i < Nb; ++i) id[i] = static_cast<int32_t>(i);
  DevBuf<int32_t> idd;
  idd.upload(id, s);
  fill_block(idd.p, Nb, idd.p, Nb, B, s);
  launch_add_diag(Nb, omega_sum.p, B, s);
  SPX_CUDA(cudaStreamSynchronize(s));
}

// ------------------------------------------------------------------ batched ACA
struct AcaDesc {
  int64_t a_off, u_off, v_off;
  int64_t task0;   // first task of this block in the current update launch
  int64_t ptask0;  // first partial slot of this block (fixed for the batch)
  int32_t ntask, m, n, kmax, early, sidx;
};
struct AcaState {
  int32_t k, done, outcome, pad;
  double normA, rel;
};
struct Partial {
  double maxv;
  int64_t idx;
  double ss;
};
enum : int { OUT_RUN = 0, OUT_CONV = 1, OUT_KMAX = 2, OUT_PIVOT = 3, OUT_DENSE_EARLY = 4, OUT_ZERO = 5 };
constexpr int ACA_CHUNK = 8192;
constexpr int ACA_THREADS = 256;

__device__ __forceinline__ void better(double& v, int64_t& i, double v2, int64_t i2) {
  if (v2 > v || (v2 == v && i2 < i)) { v = v2; i = i2; }
}

__global__ void __launch_bounds__(ACA_THREADS) k_aca_update(
    const AcaDesc* __restrict__ D, int nb, const AcaState* __restrict__ st, double* __restrict__ Apool,
    const double* __restrict__ UV, Partial* __restrict__ part) {
  const int64_t task = blockIdx.x;
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (D[mid].task0 <= task) lo = mid; else hi = mid - 1;
  }
  const AcaDesc d = D[lo];
  if (st[d.sidx].done) return;
  const int k = st[d.sidx].k;
  const int64_t mn = (int64_t)d.m * d.n;
  const int64_t e0 = (task - d.task0) * ACA_CHUNK;
  const int64_t e1 = min(mn, e0 + ACA_CHUNK);
  double* R = Apool + d.a_off;
  const double* u = UV + d.u_off + (int64_t)(k - 1) * d.m;
  const double* v = UV + d.v_off + (int64_t)(k - 1) * d.n;
  double mv = -1.0, ss = 0.0;
  int64_t mi = INT64_MAX;
  for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    double r = R[e];
    if (k > 0) {
      const int64_t i = e / d.n, j = e - i * d.n;
      r = __dsub_rn(r, __dmul_rn(u[i], v[j]));
      R[e] = r;
    }
    better(mv, mi, fabs(r), e);
    ss += r * r;
  }
  __shared__ double sv[ACA_THREADS / 32], sss[ACA_THREADS / 32];
  __shared__ int64_t si[ACA_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_xor_sync(0xffffffffu, mv, o);
    const int64_t i2 = __shfl_xor_sync(0xffffffffu, mi, o);
    better(mv, mi, v2, i2);
    ss += __shfl_xor_sync(0xffffffffu, ss, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sv[w] = mv; si[w] = mi; sss[w] = ss; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double V = sv[0], S = sss[0];
    int64_t I = si[0];
    for (int q = 1; q < ACA_THREADS / 32; ++q) { better(V, I, sv[q], si[q]); S += sss[q]; }
    part[d.ptask0 + (task - d.task0)] = Partial{V, I, S};
  }
}

// one CTA per block of the batch (descriptors in original order, sidx == blockIdx.x)
__global__ void __launch_bounds__(ACA_THREADS) k_aca_decide(
    const AcaDesc* __restrict__ D, AcaState* __restrict__ st, const double* __restrict__ Apool,
    double* __restrict__ UV, const Partial* __restrict__ part, double rtol, double storage_factor,
    int* __restrict__ active) {
  const int b = blockIdx.x;
  if (st[b].done) return;
  const AcaDesc d = D[b];
  __shared__ double sv[ACA_THREADS], sss[ACA_THREADS];
  __shared__ int64_t si[ACA_THREADS];
  __shared__ int s_go;
  __shared__ double s_piv;
  __shared__ int64_t s_idx;
  double mv = -1.0, ss = 0.0;
  int64_t mi = INT64_MAX;
  for (int t = threadIdx.x; t < d.ntask; t += blockDim.x) {
    const Partial p = part[d.ptask0 + t];
    better(mv, mi, p.maxv, p.idx);
    ss += p.ss;
  }
  sv[threadIdx.x] = mv; si[threadIdx.x] = mi; sss[threadIdx.x] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double V = sv[0], S = sss[0];
    int64_t I = si[0];
    for (int q = 1; q < blockDim.x; ++q) { better(V, I, sv[q], si[q]); S += sss[q]; }
    AcaState s = st[b];
    int go = 1;
    if (s.k == 0) {
      s.normA = sqrt(S);
      if (s.normA == 0.0) { s.done = 1; s.outcome = OUT_ZERO; s.rel = 0.0; go = 0; }
    } else {
      s.rel = sqrt(S) / s.normA;
      if (s.rel <= rtol) { s.done = 1; s.outcome = OUT_CONV; go = 0; }
      else if (s.k >= d.kmax) { s.done = 1; s.outcome = OUT_KMAX; go = 0; }
      else if (d.early && (double)(s.k + 1) * (double)(d.m + d.n) >= storage_factor * (double)d.m * (double)d.n) {
        s.done = 1; s.outcome = OUT_DENSE_EARLY; go = 0;
      }
    }
    if (go && (I < 0 || I >= (int64_t)d.m * d.n || !(S == S))) {
      // no finite pivot (non-finite block entries): stop without extracting
      s.done = 1; s.outcome = OUT_PIVOT; go = 0;
    }
    if (go) {
      const double piv = Apool[d.a_off + I];
      if (fabs(piv) <= 2.220446049250313e-16 * s.normA) { s.done = 1; s.outcome = OUT_PIVOT; go = 0; }
      s_piv = piv;
      s_idx = I;
    }
    if (!go) atomicSub(active, 1);
    st[b] = s;
    s_go = go;
  }
  __syncthreads();
  if (!s_go) return;
  const int k = st[b].k;
  const int64_t i = s_idx / d.n, j = s_idx - i * d.n;
  const double piv = s_piv;
  const double* R = Apool + d.a_off;
  double* u = UV + d.u_off + (int64_t)k * d.m;
  double* v = UV + d.v_off + (int64_t)k * d.n;
  for (int r = threadIdx.x; r < d.m; r += blockDim.x) u[r] = R[(int64_t)r * d.n + j];
  for (int c = threadIdx.x; c < d.n; c += blockDim.x) v[c] = R[i * d.n + c] / piv;
  __syncthreads();
  if (threadIdx.x == 0) st[b].k = k + 1;
}

// copy jobs: dst[k] = src[k] for len doubles (one CTA per job)
struct CopyJob {
  const double* src;
  double* dst;
  int64_t len;
};
__global__ void k_copy_jobs(const CopyJob* __restrict__ jobs) {
  const CopyJob j = jobs[blockIdx.x];
  for (int64_t k = threadIdx.x; k < j.len; k += blockDim.x) j.dst[k] = j.src[k];
}

namespace {

struct GrowBuf {
  DevBuf<double> buf;
  int64_t used = 0;
  int64_t reserve(int64_t n) {
    if (used + n > static_cast<int64_t>(buf.n)) {
      int64_t cap = std::max<int64_t>(used + n, std::max<int64_t>(2 * (int64_t)buf.n, 1 << 20));
      DevBuf<double> nb(cap);
      if (used) SPX_CUDA(cudaMemcpy(nb.p, buf.p, used * sizeof(double), cudaMemcpyDeviceToDevice));
      buf = std::move(nb);
    }
    const int64_t off = used;
    used += n;
    return off;
  }
};

void run_copy_jobs(std::vector<CopyJob>& jobs, cudaStream_t s) {
  if (jobs.empty()) return;
  DevBuf<CopyJob> dj;
  for (size_t k0 = 0; k0 < jobs.size(); k0 += 65535) {
    const size_t cnt = std::min<size_t>(65535, jobs.size() - k0);
    dj.upload(jobs.data() + k0, cnt, s);
    k_copy_jobs<<<static_cast<unsigned>(cnt), 256, 0, s>>>(dj.p);
    SPX_LAUNCH_CHECK();
    SPX_CUDA(cudaStreamSynchronize(s));
  }
  jobs.clear();
}

}  // namespace

void HMatrix::build(const BoundaryDev& bd, const HBuildConfig& c, cudaStream_t s) {
  auto t_start = std::chrono::steady_clock::now();
  SPX_CUDA(cudaGetDevice(&device));
  cfg = c;
  Nb = bd.host.Nb;
  build_cluster_tree(bd.host.Xb.data(), Nb, c.leaf_size, tree);
  perm.upload(tree.perm, s);
  {
    std::vector<double> dj(Nb);
    for (int64_t i = 0; i < Nb; ++i)
      dj[i] = bd.host.omega_sum[tree.perm[i]] / (4.0 * 3.141592653589793) - 1.0;
    diag_perm.upload(dj, s);
  }
  stats = HStats{};
  blocks.clear();
  GrowBuf far_g, near_g;
  const double margin = 1.0 + 64.0 * 2.220446049250313e-16;
  const std::vector<TreeNode>& nodes = tree.nodes;

  std::vector<std::pair<int32_t, int32_t>> wave{{0, 0}}, next;
  auto subdivide = [&](int32_t r, int32_t cc, std::vector<std::pair<int32_t, int32_t>>& out,
                       std::vector<std::pair<int32_t, int32_t>>& near_out) {
    const TreeNode &R = nodes[r], &C = nodes[cc];
    const bool rs = !R.leaf(), cs = !C.leaf();
    if (!rs && !cs) { near_out.push_back({r, cc}); return; }
    if (rs && (!cs || R.diameter() >= C.diameter())) {
      out.push_back({R.left, cc});
      out.push_back({R.right, cc});
    } else {
      out.push_back({r, C.left});
      out.push_back({r, C.right});
    }
  };

  const int32_t* pool = perm.p;
  int* h_active = nullptr;
  SPX_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_active), sizeof(int)));
  DevBuf<int> d_active(1);

  while (!wave.empty()) {
    stats.waves++;
    next.clear();
    std::vector<std::pair<int32_t, int32_t>> adm, nearl;
    for (auto& pr : wave) {
      const TreeNode &R = nodes[pr.first], &C = nodes[pr.second];
      const bool a = admissible(R, C, c.eta);
      const int64_t bytes = (int64_t)R.size() * C.size() * 8;
      if (a && bytes > c.max_temporary_block_bytes) {
        stats.forced_subdivisions_memory++;
        subdivide(pr.first, pr.second, next, nearl);
      } else if (a) {
        adm.push_back(pr);
      } else if (R.leaf() && C.leaf()) {
        nearl.push_back(pr);
      } else {
        subdivide(pr.first, pr.second, next, nearl);
      }
    }
    // ---- near (non-admissible leaf pairs and unsplittable subdivisions): fill into near pool
    {
      std::vector<FillDesc> fd;
      std::vector<int64_t> ts;
      int64_t tiles = 0;
      auto flush = [&]() {
        if (fd.empty()) return;
        DevBuf<FillDesc> dfd;
        DevBuf<int64_t> dts;
        dfd.upload(fd, s);
        dts.upload(ts, s);
        launch_fill(dfd.p, dts.p, static_cast<int>(fd.size()), tiles, pool, pool, bd.Xb.p, bd.tri_lid.p,
                    bd.T.p, bd.inc_ptr.p, bd.inc_tri.p, bd.maxinc, bd.host.Nb, near_g.buf.p, s);
        SPX_CUDA(cudaStreamSynchronize(s));
        fd.clear();
        ts.clear();
        tiles = 0;
      };
      // reserve all first (pool may move), then fill
      std::vector<int64_t> offs;
      for (auto& pr : nearl) {
        const TreeNode &R = nodes[pr.first], &C = nodes[pr.second];
        offs.push_back(near_g.reserve((int64_t)R.size() * C.size()));
      }
      for (size_t q = 0; q < nearl.size(); ++q) {
        const TreeNode &R = nodes[nearl[q].first], &C = nodes[nearl[q].second];
        ts.push_back(tiles);
        fd.push_back(FillDesc{offs[q], R.start, C.start, R.size(), C.size()});
        tiles += (int64_t)((R.size() + 127) / 128) * ((C.size() + 31) / 32);
        HBlock hb{R.start, R.stop, C.start, C.stop, 0, 0, offs[q], 0, 0.0};
        blocks.push_back(hb);
        stats.dense_blocks++;
        stats.block_entry_evaluations += (int64_t)R.size() * C.size();
        if (tiles > (1ll << 28)) flush();
      }
      flush();
    }
    // ---- admissible candidates: batched fill + ACA
    std::sort(adm.begin(), adm.end(), [&](const std::pair<int32_t, int32_t>& x,
                                          const std::pair<int32_t, int32_t>& y) {
      const int64_t sx = (int64_t)nodes[x.first].size() * nodes[x.second].size();
      const int64_t sy = (int64_t)nodes[y.first].size() * nodes[y.second].size();
      if (sx != sy) return sx > sy;
      return x < y;
    });
    size_t q0 = 0;
    while (q0 < adm.size()) {
      // batch under the workspace budget
      std::vector<AcaDesc> ad;
      std::vector<FillDesc> fd;
      std::vector<int64_t> ts;
      int64_t a_tot = 0, uv_tot = 0, tasks = 0, tiles = 0;
      size_t q1 = q0;
      while (q1 < adm.size()) {
        const TreeNode &R = nodes[adm[q1].first], &C = nodes[adm[q1].second];
        const int64_t m = R.size(), n = C.size(), mn = m * n;
        const int64_t mnmin = std::min(m, n);
        int64_t kmax = c.max_rank < 0 ? mnmin : std::min<int64_t>(c.max_rank, mnmin);
        const bool early = (c.max_rank < 0) && (c.epsilon > 1e-10);
        int64_t kcap = kmax;
        if (early) {
          // largest k+1 extracted satisfies (k+1)(m+n) < 0.95 m n
          const int64_t kb = static_cast<int64_t>(std::floor(c.low_rank_storage_factor * (double)mn / (double)(m + n))) + 1;
          kcap = std::min(kcap, kb);
        }
        const int64_t need = (mn + kcap * (m + n)) * 8;
        if (q1 > q0 && (a_tot + uv_tot) * 8 + need > c.batch_bytes) break;
        ad.push_back(AcaDesc{a_tot, uv_tot, uv_tot + kcap * m, tasks, tasks,
                             static_cast<int32_t>((mn + ACA_CHUNK - 1) / ACA_CHUNK), (int32_t)m, (int32_t)n,
                             (int32_t)kmax, early ? 1 : 0, static_cast<int32_t>(ad.size())});
        fd.push_back(FillDesc{a_tot, R.start, C.start, (int32_t)m, (int32_t)n});
        ts.push_back(tiles);
        tiles += ((m + 127) / 128) * ((n + 31) / 32);
        tasks += ad.back().ntask;
        a_tot += mn;
        uv_tot += kcap * (m + n);
        ++q1;
      }
      const int nb = static_cast<int>(ad.size());
      DevBuf<double> A(a_tot), UV(std::max<int64_t>(uv_tot, 1));
      DevBuf<FillDesc> dfd;
      DevBuf<int64_t> dts;
      dfd.upload(fd, s);
      dts.upload(ts, s);
      launch_fill(dfd.p, dts.p, nb, tiles, pool, pool, bd.Xb.p, bd.tri_lid.p, bd.T.p, bd.inc_ptr.p,
                  bd.inc_tri.p, bd.maxinc, bd.host.Nb, A.p, s);
      stats.block_entry_evaluations += a_tot;
      DevBuf<AcaDesc> dad, dupd;
      dad.upload(ad, s);
      DevBuf<AcaState> dst(nb);
      {
        std::vector<AcaState> h0(nb, AcaState{0, 0, 0, 0, 0.0, 1.0});
        dst.upload(h0, s);
      }
      DevBuf<Partial> dpart(std::max<int64_t>(tasks, 1));
      int active = nb;
      SPX_CUDA(cudaMemcpyAsync(d_active.p, &active, sizeof(int), cudaMemcpyHostToDevice, s));
      // update launch list (compacted to the active blocks as they finish)
      const AcaDesc* upd = dad.p;
      int n_upd = nb;
      int64_t upd_tasks = tasks;
      int64_t max_steps = 1;
      for (auto& d : ad) max_steps = std::max<int64_t>(max_steps, (int64_t)d.kmax + 2);
      int64_t step = 0;
      const int check_every = 4;
      while (true) {
        k_aca_update<<<static_cast<unsigned>(upd_tasks), ACA_THREADS, 0, s>>>(upd, n_upd, dst.p, A.p, UV.p,
                                                                             dpart.p);
        SPX_LAUNCH_CHECK();
        k_aca_decide<<<nb, ACA_THREADS, 0, s>>>(dad.p, dst.p, A.p, UV.p, dpart.p, c.epsilon,
                                               c.low_rank_storage_factor, d_active.p);
        SPX_LAUNCH_CHECK();
        ++step;
        stats.aca_steps++;
        if (step % check_every == 0 || step >= max_steps) {
          SPX_CUDA(cudaMemcpyAsync(h_active, d_active.p, sizeof(int), cudaMemcpyDeviceToHost, s));
          SPX_CUDA(cudaStreamSynchronize(s));
          const int act = *h_active;
          if (act == 0) break;
          if (step >= max_steps) throw Error(ERR_INTERNAL, "ACA batch did not finish within kmax steps");
          if (2 * act < n_upd) {
            std::vector<AcaState> hs(nb);
            dst.download(hs.data(), nb, s);
            SPX_CUDA(cudaStreamSynchronize(s));
            std::vector<AcaDesc> sub;
            int64_t t0 = 0;
            for (int bq = 0; bq < nb; ++bq)
              if (!hs[bq].done) {
                AcaDesc d = ad[bq];
                d.task0 = t0;
                t0 += d.ntask;
                sub.push_back(d);
              }
            dupd.upload(sub, s);
            upd = dupd.p;
            n_upd = static_cast<int>(sub.size());
            upd_tasks = t0;
          }
        }
      }
      std::vector<AcaState> hs(nb);
      dst.download(hs.data(), nb, s);
      SPX_CUDA(cudaStreamSynchronize(s));
      // decisions (builder.py:343-370); reserve pool space before taking pointers
      std::vector<int> decision(nb, 0);  // 1 accept, 2 dense, 3 subdivide
      std::vector<int64_t> du(nb, -1), dv(nb, -1), dn(nb, -1);
      for (int bq = 0; bq < nb; ++bq) {
        const AcaDesc& d = ad[bq];
        const AcaState& st = hs[bq];
        const TreeNode &R = nodes[adm[q0 + bq].first], &C = nodes[adm[q0 + bq].second];
        const bool meets = std::isfinite(st.rel) && st.rel <= c.epsilon * margin;
        int dec;
        if (st.outcome == OUT_DENSE_EARLY) dec = 2;
        else if (st.k > 0 && meets &&
                 (double)st.k * (d.m + d.n) < c.low_rank_storage_factor * (double)d.m * d.n) dec = 1;
        else if (!meets && (!R.leaf() || !C.leaf())) dec = 3;
        else dec = 2;
        decision[bq] = dec;
        if (dec == 1) {
          du[bq] = far_g.reserve((int64_t)st.k * d.m);
          dv[bq] = far_g.reserve((int64_t)st.k * d.n);
        } else if (dec == 2) {
          dn[bq] = near_g.reserve((int64_t)d.m * d.n);
        }
      }
      std::vector<CopyJob> jobs;
      std::vector<FillDesc> rf;
      std::vector<int64_t> rts;
      int64_t rt = 0;
      for (int bq = 0; bq < nb; ++bq) {
        const AcaDesc& d = ad[bq];
        const AcaState& st = hs[bq];
        const int32_t rn = adm[q0 + bq].first, cn = adm[q0 + bq].second;
        const TreeNode &R = nodes[rn], &C = nodes[cn];
        if (decision[bq] == 1) {
          jobs.push_back(CopyJob{UV.p + d.u_off, far_g.buf.p + du[bq], (int64_t)st.k * d.m});
          jobs.push_back(CopyJob{UV.p + d.v_off, far_g.buf.p + dv[bq], (int64_t)st.k * d.n});
          blocks.push_back(HBlock{R.start, R.stop, C.start, C.stop, 1, st.k, du[bq], dv[bq], st.rel});
          stats.low_rank_blocks++;
          stats.max_observed_rank = std::max<int64_t>(stats.max_observed_rank, st.k);
          stats.sum_observed_rank += st.k;
        } else if (decision[bq] == 2) {
          // A now holds the residual: refill the original entries into the near pool
          rts.push_back(rt);
          rf.push_back(FillDesc{dn[bq], fd[bq].rows_off, fd[bq].cols_off, fd[bq].m, fd[bq].n});
          rt += (int64_t)((fd[bq].m + 127) / 128) * ((fd[bq].n + 31) / 32);
          blocks.push_back(HBlock{R.start, R.stop, C.start, C.stop, 0, 0, dn[bq], 0, st.rel});
          stats.dense_blocks++;
          stats.rejected_low_rank_blocks++;
          stats.block_entry_evaluations += (int64_t)d.m * d.n;
        } else {
          stats.compression_tolerance_subdivisions++;
          std::vector<std::pair<int32_t, int32_t>> none;
          subdivide(rn, cn, next, none);
          SPX_CHECK(none.empty(), "internal: subdivision of a splittable block produced a leaf pair");
        }
      }
      if (!rf.empty()) {
        DevBuf<FillDesc> drf;
        DevBuf<int64_t> drts;
        drf.upload(rf, s);
        drts.upload(rts, s);
        launch_fill(drf.p, drts.p, static_cast<int>(rf.size()), rt, pool, pool, bd.Xb.p, bd.tri_lid.p,
                    bd.T.p, bd.inc_ptr.p, bd.inc_tri.p, bd.maxinc, bd.host.Nb, near_g.buf.p, s);
      }
      run_copy_jobs(jobs, s);
      SPX_CUDA(cudaStreamSynchronize(s));
      q0 = q1;
    }
    wave.swap(next);
  }
  cudaFreeHost(h_active);
  far_pool64 = std::move(far_g.buf);
  near_pool64 = std::move(near_g.buf);
  stats.n_far = stats.low_rank_blocks;
  stats.n_near = stats.dense_blocks;
  for (auto& b : blocks) {
    if (b.type == 1) stats.far_entries += (int64_t)b.rank * ((b.re - b.rs) + (b.ce - b.cs));
    else stats.near_entries += (int64_t)(b.re - b.rs) * (b.ce - b.cs);
  }
  SPX_CUDA(cudaStreamSynchronize(s));
  packed = false;
  recompressed = false;
  sigma.clear();
  if (c.recompress) recompress(s);
  stats.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
}

}  // namespace spx
