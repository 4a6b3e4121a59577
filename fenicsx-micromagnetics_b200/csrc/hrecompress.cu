// Recompression of the ACA factors: every far block U V (U^T k x m, V k x n, FP64 pool) is
// rewritten as U' V' with U' = Q_u W_r Sigma_r and V' = Z_r^T Q_v^T from the SVD of its k x k
// core, truncated to the smallest rank r whose discarded singular values keep the block within
// the build tolerance: ||U V - U' V'||_F <= (epsilon - relres) ||U V||_F, relres the ACA
// residual of the block.  The block's guarantee ||A - U' V'||_F <= epsilon ||A||_F (the
// acceptance rule of HMatrixBuilder, builder.py:343-356) therefore still holds, and the
// stored relative residual becomes relres + the truncation error.  This is the
// ACA-plus-recompression of Bebendorf (M. Bebendorf, "Hierarchical Matrices", Springer 2008,
// sec. 1.1.5 / 3.4); the reference's truncated_svd compressor (compressors.py:102-235) is the
// same family applied to the dense block.
//
// Work split:
//   k_rc_gram  (device, one CTA per block): Gram matrices G_u = U^T U, G_v = V V^T (k x k);
//   host (all threads): equilibrated Cholesky G~ = L L^T, core C = L_u^T D_u^-1 D_v^-1 L_v,
//              one-sided Jacobi SVD of C, truncation, T_u = D_u L_u^-T W_r Sigma_r (k x r),
//              T_v = Z_r^T L_v^-1 D_v (r x k), and an a-posteriori check of the truncation
//              error ||U (I - T_u T_v) V||_F^2 = tr(M^T G_u M G_v) from the exact Grams; a block
//              whose check fails, or whose rank exceeds RC_KMAX, keeps its factors;
//   k_rc_apply (device, one CTA per block): U'^T = T_u^T U^T, V' = T_v V into a new pool.
// The new columns are ordered by decreasing singular value; column j of U' has norm
// sigma_j and row j of V' norm 1.  The sigmas are kept on the host (HMatrix::sigma) for the
// split-precision packing.
#include <algorithm>
#include <cmath>
#include <thread>

#include "hmat.cuh"

namespace spx {

namespace {

constexpr int RC_KMAX = 64;
constexpr int RC_THREADS = 256;
constexpr int RC_CHUNK = 64;  // columns of a factor streamed through shared memory at a time

struct RcBlock {
  int64_t off_u, off_v;  // FP64 pool: U^T (k x m), V (k x n)
  int64_t g_off;         // Grams: 2 k^2 doubles
  int32_t m, n, k, pad;
};

// G[p][q] = sum_c F[p][c] F[q][c] for a k x len row-major factor (p <= q, mirrored)
__device__ void gram_rows(const double* __restrict__ F, int k, int len, double* __restrict__ G, double* sm) {
  const int npair = k * (k + 1) / 2;
  constexpr int PPT = (RC_KMAX * (RC_KMAX + 1) / 2 + RC_THREADS - 1) / RC_THREADS;  // pairs per thread
  double acc[PPT];
  int pp[PPT], qq[PPT];
#pragma unroll
  for (int t = 0; t < PPT; ++t) {
    acc[t] = 0.0;
    const int idx = threadIdx.x + t * RC_THREADS;
    pp[t] = qq[t] = -1;
    if (idx < npair) {  // idx -> (p, q), p <= q, row-major upper triangle
      int p = 0, rem = idx;
      while (rem >= k - p) { rem -= k - p; ++p; }
      pp[t] = p;
      qq[t] = p + rem;
    }
  }
  for (int c0 = 0; c0 < len; c0 += RC_CHUNK) {
    const int w = min(RC_CHUNK, len - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < k * RC_CHUNK; e += blockDim.x) {
      const int p = e / RC_CHUNK, c = e - p * RC_CHUNK;
      sm[e] = c < w ? F[static_cast<int64_t>(p) * len + c0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < PPT; ++t) {
      if (pp[t] < 0) continue;
      const double* a = sm + pp[t] * RC_CHUNK;
      const double* b = sm + qq[t] * RC_CHUNK;
      double s = 0.0;
      for (int c = 0; c < w; ++c) s += a[c] * b[c];
      acc[t] += s;
    }
  }
#pragma unroll
  for (int t = 0; t < PPT; ++t)
    if (pp[t] >= 0) {
      G[pp[t] * k + qq[t]] = acc[t];
      G[qq[t] * k + pp[t]] = acc[t];
    }
}

__global__ void __launch_bounds__(RC_THREADS) k_rc_gram(const RcBlock* __restrict__ blk, const double* __restrict__ pool,
                                                       double* __restrict__ grams) {
  extern __shared__ double sm[];
  const RcBlock b = blk[blockIdx.x];
  gram_rows(pool + b.off_u, b.k, b.m, grams + b.g_off, sm);
  gram_rows(pool + b.off_v, b.k, b.n, grams + b.g_off + static_cast<int64_t>(b.k) * b.k, sm);
}

struct RcApply {
  int64_t src, dst, t_off;  // factor k x len at src -> r x len at dst; T: k x r at t_off (out[j] = sum_p T[p][j] in[p])
  int32_t k, r, len, pad;
};

__global__ void __launch_bounds__(RC_THREADS) k_rc_apply(const RcApply* __restrict__ jobs, const double* __restrict__ pool,
                                                        const double* __restrict__ T, double* __restrict__ out) {
  extern __shared__ double sm[];  // [RC_KMAX][RC_CHUNK] input chunk + [RC_KMAX][RC_KMAX] T
  const RcApply j = jobs[blockIdx.x];
  double* tin = sm;
  double* tt = sm + RC_KMAX * RC_CHUNK;
  for (int e = threadIdx.x; e < j.k * j.r; e += blockDim.x) tt[e] = T[j.t_off + e];
  for (int c0 = 0; c0 < j.len; c0 += RC_CHUNK) {
    const int w = min(RC_CHUNK, j.len - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < j.k * RC_CHUNK; e += blockDim.x) {
      const int p = e / RC_CHUNK, c = e - p * RC_CHUNK;
      tin[e] = c < w ? pool[j.src + static_cast<int64_t>(p) * j.len + c0 + c] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < j.r * RC_CHUNK; e += blockDim.x) {
      const int q = e / RC_CHUNK, c = e - q * RC_CHUNK;
      if (c >= w) continue;
      double s = 0.0;
      for (int p = 0; p < j.k; ++p) s += tt[p * j.r + q] * tin[p * RC_CHUNK + c];
      out[j.dst + static_cast<int64_t>(q) * j.len + c0 + c] = s;
    }
  }
}

// ---------------------------------------------------------------- host linear algebra
// lower Cholesky of the k x k SPD matrix A (row-major) in place; pivots below tol*max diag are
// treated as zero (rank-deficient factor): the row/column is dropped (L[i][i] = 0).
void cholesky(std::vector<double>& A, int k, std::vector<char>& live) {
  live.assign(k, 1);
  double dmax = 0.0;
  for (int i = 0; i < k; ++i) dmax = std::max(dmax, A[i * k + i]);
  const double tol = 1e-28 * std::max(dmax, 1e-300);
  for (int j = 0; j < k; ++j) {
    double d = A[j * k + j];
    for (int p = 0; p < j; ++p) d -= A[j * k + p] * A[j * k + p];
    if (!(d > tol)) {
      live[j] = 0;
      for (int i = j; i < k; ++i) A[i * k + j] = 0.0;
      continue;
    }
    const double l = std::sqrt(d);
    A[j * k + j] = l;
    for (int i = j + 1; i < k; ++i) {
      double s = A[i * k + j];
      for (int p = 0; p < j; ++p) s -= A[i * k + p] * A[j * k + p];
      A[i * k + j] = s / l;
    }
  }
  for (int i = 0; i < k; ++i)
    for (int j = i + 1; j < k; ++j) A[i * k + j] = 0.0;
}

// one-sided Jacobi: C (k x k, row-major) -> columns orthogonalised in place, Z (k x k) the
// accumulated rotations (C_in Z = C_out); returns false when it did not converge
bool jacobi_svd(std::vector<double>& C, std::vector<double>& Z, int k) {
  Z.assign(static_cast<size_t>(k) * k, 0.0);
  for (int i = 0; i < k; ++i) Z[i * k + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < k - 1; ++p)
      for (int q = p + 1; q < k; ++q) {
        double a = 0.0, b = 0.0, g = 0.0;
        for (int i = 0; i < k; ++i) {
          const double cp = C[i * k + p], cq = C[i * k + q];
          a += cp * cp;
          b += cq * cq;
          g += cp * cq;
        }
        if (g == 0.0 || std::fabs(g) <= 1e-15 * std::sqrt(a * b)) continue;
        off = std::max(off, std::fabs(g) / std::sqrt(a * b));
        const double zeta = (b - a) / (2.0 * g);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
        for (int i = 0; i < k; ++i) {
          const double cp = C[i * k + p], cq = C[i * k + q];
          C[i * k + p] = c * cp - s * cq;
          C[i * k + q] = s * cp + c * cq;
          const double zp = Z[i * k + p], zq = Z[i * k + q];
          Z[i * k + p] = c * zp - s * zq;
          Z[i * k + q] = s * zp + c * zq;
        }
      }
    if (off <= 1e-15) return true;
  }
  return false;
}

struct RcResult {
  int32_t r = 0;
  bool rewrite = false;
  double err = 0.0, norm = 0.0;
  std::vector<double> Tu, Tv, sigma;  // Tu: k x r, Tv stored transposed as k x r (out[j] = sum_p T[p][j] in[p])
};

void analyse_block(const double* Gu0, const double* Gv0, int k, double eps, double relres, RcResult& out) {
  out = RcResult();
  out.r = k;
  std::vector<double> Gu(Gu0, Gu0 + k * k), Gv(Gv0, Gv0 + k * k);
  std::vector<double> du(k), dv(k);
  for (int i = 0; i < k; ++i) {
    du[i] = Gu[i * k + i] > 0.0 ? 1.0 / std::sqrt(Gu[i * k + i]) : 0.0;
    dv[i] = Gv[i * k + i] > 0.0 ? 1.0 / std::sqrt(Gv[i * k + i]) : 0.0;
  }
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) {
      Gu[i * k + j] *= du[i] * du[j];
      Gv[i * k + j] *= dv[i] * dv[j];
    }
  std::vector<char> lu, lv;
  cholesky(Gu, k, lu);  // L~_u
  cholesky(Gv, k, lv);  // L~_v
  // C = L~_u^T diag(1 / (du dv)) L~_v ; U = Q_u L~_u^T D_u^-1, V = D_v^-1 L~_v Q_v^T
  std::vector<double> C(static_cast<size_t>(k) * k, 0.0);
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) {
      double s = 0.0;
      for (int p = 0; p < k; ++p) {
        const double w = (du[p] > 0.0 && dv[p] > 0.0) ? 1.0 / (du[p] * dv[p]) : 0.0;
        s += Gu[p * k + i] * w * Gv[p * k + j];
      }
      C[i * k + j] = s;
    }
  std::vector<double> Z;
  if (!jacobi_svd(C, Z, k)) return;
  std::vector<double> sig(k);
  for (int j = 0; j < k; ++j) {
    double s = 0.0;
    for (int i = 0; i < k; ++i) s += C[i * k + j] * C[i * k + j];
    sig[j] = std::sqrt(s);
  }
  std::vector<int> ord(k);
  for (int j = 0; j < k; ++j) ord[j] = j;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return sig[a] > sig[b]; });
  double nrm2 = 0.0;
  for (int j = 0; j < k; ++j) nrm2 += sig[j] * sig[j];
  const double nrm = std::sqrt(nrm2);
  out.norm = nrm;
  if (!(nrm > 0.0)) return;
  const double budget = std::max(0.0, eps - relres) * nrm * (1.0 - 4.0 * eps);
  // smallest r with sqrt(sum_{j >= r} sigma_j^2) <= budget
  std::vector<double> tail(k + 1, 0.0);
  for (int j = k - 1; j >= 0; --j) tail[j] = tail[j + 1] + sig[ord[j]] * sig[ord[j]];
  int r = k;
  for (int j = 0; j <= k; ++j)
    if (std::sqrt(tail[j]) <= budget) { r = j; break; }
  r = std::max(r, 1);
  // W = C Z / sigma (columns), T_u = D_u L~_u^-T W_r Sigma_r = D_u L~_u^-T (C Z)_r,
  // T_v^T (k x r) = D_v L~_v^-T Z_r
  auto solve_lt = [&](const std::vector<double>& L, const std::vector<char>& live, std::vector<double>& B, int nc) {
    // B (k x nc) <- L^-T B (back substitution on L^T, upper triangular); dropped pivots -> 0
    for (int c = 0; c < nc; ++c)
      for (int i = k - 1; i >= 0; --i) {
        if (!live[i]) { B[i * nc + c] = 0.0; continue; }
        double s = B[i * nc + c];
        for (int p = i + 1; p < k; ++p) s -= L[p * k + i] * B[p * nc + c];
        B[i * nc + c] = s / L[i * k + i];
      }
  };
  std::vector<double> Tu(static_cast<size_t>(k) * r), Tv(static_cast<size_t>(k) * r);
  for (int i = 0; i < k; ++i)
    for (int c = 0; c < r; ++c) {
      Tu[i * r + c] = C[i * k + ord[c]];  // (C Z)_{i, ord[c]} = W Sigma
      Tv[i * r + c] = Z[i * k + ord[c]];
    }
  solve_lt(Gu, lu, Tu, r);
  solve_lt(Gv, lv, Tv, r);
  for (int i = 0; i < k; ++i)
    for (int c = 0; c < r; ++c) {
      Tu[i * r + c] *= du[i];
      Tv[i * r + c] *= dv[i];
    }
  // a-posteriori truncation error: M = I - T_u T_v (T_v = Tv^T), err^2 = tr(M^T G_u M G_v)
  std::vector<double> M(static_cast<size_t>(k) * k);
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) {
      double s = 0.0;
      for (int c = 0; c < r; ++c) s += Tu[i * r + c] * Tv[j * r + c];
      M[i * k + j] = (i == j ? 1.0 : 0.0) - s;
    }
  // err^2 = tr(P G_v), P = M^T A1, A1 = G_u M
  std::vector<double> A1(static_cast<size_t>(k) * k);
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) {
      double s = 0.0;
      for (int p = 0; p < k; ++p) s += Gu0[i * k + p] * M[p * k + j];
      A1[i * k + j] = s;
    }
  double e2 = 0.0;
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < k; ++b) {
      double s = 0.0;
      for (int p = 0; p < k; ++p) s += M[p * k + a] * A1[p * k + b];
      e2 += s * Gv0[b * k + a];
    }
  const double err = std::sqrt(std::max(e2, 0.0));
  if (!(err <= std::max(budget, 0.0) * 1.01 + 1e-300) || r >= k) return;
  out.r = r;
  out.rewrite = true;
  out.err = err;
  out.Tu.swap(Tu);
  out.Tv.swap(Tv);
  out.sigma.resize(r);
  for (int c = 0; c < r; ++c) out.sigma[c] = sig[ord[c]];
}

}  // namespace

RecompressStats HMatrix::recompress(cudaStream_t s) {
  RecompressStats st;
  std::vector<int> fidx;
  for (size_t i = 0; i < blocks.size(); ++i)
    if (blocks[i].type == 1 && blocks[i].rank > 0 && blocks[i].rank <= RC_KMAX) fidx.push_back(static_cast<int>(i));
  for (const HBlock& b : blocks)
    if (b.type == 1) st.entries_before += static_cast<int64_t>(b.rank) * ((b.re - b.rs) + (b.ce - b.cs));
  const int nb = static_cast<int>(fidx.size());
  sigma.assign(blocks.size(), std::vector<double>());
  if (nb == 0) {
    st.entries_after = st.entries_before;
    return st;
  }
  // 1. Grams on the device
  std::vector<RcBlock> rb(nb);
  int64_t goff = 0;
  for (int q = 0; q < nb; ++q) {
    const HBlock& b = blocks[fidx[q]];
    rb[q] = RcBlock{b.off_u, b.off_v, goff, b.re - b.rs, b.ce - b.cs, b.rank, 0};
    goff += 2ll * b.rank * b.rank;
  }
  DevBuf<RcBlock> drb;
  drb.upload(rb, s);
  DevBuf<double> grams(goff);
  const size_t smem_gram = static_cast<size_t>(RC_KMAX) * RC_CHUNK * sizeof(double);
  SPX_CUDA(cudaFuncSetAttribute(k_rc_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_gram)));
  for (int q0 = 0; q0 < nb; q0 += 65535) {
    const int c = std::min(65535, nb - q0);
    k_rc_gram<<<c, RC_THREADS, smem_gram, s>>>(drb.p + q0, far_pool64.p, grams.p);
    SPX_LAUNCH_CHECK();
  }
  std::vector<double> hg(goff);
  grams.download(hg.data(), goff, s);
  SPX_CUDA(cudaStreamSynchronize(s));
  // 2. truncation on the host threads
  std::vector<RcResult> res(nb);
  const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nth; ++t)
      th.emplace_back([&, t]() {
        for (int q = static_cast<int>(t); q < nb; q += static_cast<int>(nth)) {
          const HBlock& b = blocks[fidx[q]];
          const int k = b.rank;
          analyse_block(hg.data() + rb[q].g_off, hg.data() + rb[q].g_off + static_cast<int64_t>(k) * k, k,
                        cfg.epsilon, b.relres, res[q]);
        }
      });
    for (auto& x : th) x.join();
  }
  // 3. new pool: rewritten blocks get T applied, the others are copied as they are (T = I)
  std::vector<RcApply> jobs;
  std::vector<double> hT;
  int64_t pos = 0;
  std::vector<int64_t> new_u(blocks.size(), -1), new_v(blocks.size(), -1);
  std::vector<int32_t> new_r(blocks.size(), 0);
  std::vector<char> in_set(blocks.size(), 0);
  for (int q = 0; q < nb; ++q) in_set[fidx[q]] = 1;
  int q = 0;
  for (size_t i = 0; i < blocks.size(); ++i) {
    const HBlock& b = blocks[i];
    if (b.type != 1) continue;
    const int m = b.re - b.rs, n = b.ce - b.cs, k = b.rank;
    int r = k;
    const RcResult* R = nullptr;
    if (in_set[i]) {
      R = &res[q++];
      if (R->rewrite) r = R->r;
    }
    new_r[i] = r;
    new_u[i] = pos;
    pos += static_cast<int64_t>(r) * m;
    new_v[i] = pos;
    pos += static_cast<int64_t>(r) * n;
    if (k == 0) continue;
    const int64_t toff = static_cast<int64_t>(hT.size());
    if (R && R->rewrite) {
      hT.insert(hT.end(), R->Tu.begin(), R->Tu.end());
      hT.insert(hT.end(), R->Tv.begin(), R->Tv.end());
      sigma[i] = R->sigma;
      st.rewritten++;
      st.truncation_error_max = std::max(st.truncation_error_max, R->err / std::max(R->norm, 1e-300));
    } else {  // identity
      for (int a = 0; a < k; ++a)
        for (int c = 0; c < k; ++c) hT.push_back(a == c ? 1.0 : 0.0);
      for (int a = 0; a < k; ++a)
        for (int c = 0; c < k; ++c) hT.push_back(a == c ? 1.0 : 0.0);
    }
    const int64_t tv = toff + static_cast<int64_t>(k) * r;
    jobs.push_back(RcApply{b.off_u, new_u[i], toff, k, r, m, 0});
    jobs.push_back(RcApply{b.off_v, new_v[i], tv, k, r, n, 0});
  }
  SPX_CHECK(static_cast<int64_t>(jobs.size()) < (int64_t(1) << 31), "too many recompression jobs");
  DevBuf<double> npool(std::max<int64_t>(pos, 1)), dT(std::max<size_t>(hT.size(), 1));
  dT.upload(hT, s);
  DevBuf<RcApply> dj;
  dj.upload(jobs, s);
  const size_t smem_apply = static_cast<size_t>(RC_KMAX) * (RC_CHUNK + RC_KMAX) * sizeof(double);
  SPX_CUDA(cudaFuncSetAttribute(k_rc_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_apply)));
  const int64_t nj = static_cast<int64_t>(jobs.size());
  for (int64_t j0 = 0; j0 < nj; j0 += 65535) {
    const int c = static_cast<int>(std::min<int64_t>(65535, nj - j0));
    k_rc_apply<<<c, RC_THREADS, smem_apply, s>>>(dj.p + j0, far_pool64.p, dT.p, npool.p);
    SPX_LAUNCH_CHECK();
  }
  SPX_CUDA(cudaStreamSynchronize(s));
  far_pool64 = std::move(npool);
  q = 0;
  stats.max_observed_rank = 0;
  stats.sum_observed_rank = 0;
  stats.far_entries = 0;
  for (size_t i = 0; i < blocks.size(); ++i) {
    HBlock& b = blocks[i];
    if (b.type != 1) continue;
    if (in_set[i]) {
      const RcResult& R = res[q++];
      if (R.rewrite) b.relres += R.err / std::max(R.norm, 1e-300);
    }
    b.rank = new_r[i];
    b.off_u = new_u[i];
    b.off_v = new_v[i];
    stats.max_observed_rank = std::max<int64_t>(stats.max_observed_rank, b.rank);
    stats.sum_observed_rank += b.rank;
    stats.far_entries += static_cast<int64_t>(b.rank) * ((b.re - b.rs) + (b.ce - b.cs));
  }
  st.entries_after = stats.far_entries;
  recompressed = true;
  packed = false;
  tr.reset();
  tc.reset();  // the tensor-core plan packs the old factors
  return st;
}

}  // namespace spx
