// Device side of the smoothed-aggregation AMG (amg.cuh): level upload, the FP32 V-cycle
// and the FP64 preconditioned CG that uses it, in one persistent cooperative kernel.
//
// Level layout: every level matrix (A_l, P_l, R_l = P_l^T) is SELL-32 (one thread per row,
// 32 rows per slice, padding entries point at column 0 with value 0), FP32 values, FP32
// vectors b, x, x2, d, r per level.  Levels with many nonzeros are swept by the whole grid
// (grid barrier between phases); small levels and the dense coarsest solve are swept by
// CTA 0 alone (__syncthreads between phases) while the other CTAs wait at the next grid
// barrier.
//
// PCG (FP64 vectors, scaled system A^ = D^-1/2 A D^-1/2, FP64 values):
//   z = V(r);  beta = (r,z)/(r,z)_old;  c = (w,z)/(w,w) (singular systems: remove the
//   null-vector component w = D^1/2 1 from z);  p = z - c w + beta p;
//   q = A^ z + beta q  (A^ w = 0, so q = A^ p without a second SpMV);  alpha = (r,z)/(p,q);
//   y += alpha p;  r -= alpha q.
// The recurrence residual is confirmed against the true FP64 residual before returning;
// stopping rule ||b - A x|| <= max(rtol ||b||, atol) in the unscaled norm, as the IR solver.
#include <algorithm>
#include <cmath>

#include "amg.cuh"
#include "fem.cuh"

namespace spx {

namespace {

void csr_to_sell(const CsrHost& A, HostSell& s, std::vector<float>& val) {
  const int64_t n = A.n;
  s.nrows = n;
  s.nslices = (n + SELL_C - 1) / SELL_C;
  s.slice_ptr.assign(s.nslices + 1, 0);
  for (int64_t sl = 0; sl < s.nslices; ++sl) {
    int64_t w = 0;
    for (int64_t r = sl * SELL_C; r < std::min(n, (sl + 1) * SELL_C); ++r) w = std::max(w, A.rp[r + 1] - A.rp[r]);
    s.slice_ptr[sl + 1] = s.slice_ptr[sl] + w * SELL_C;
  }
  const int64_t L = s.slice_ptr.back();
  s.col.assign(L, 0);
  val.assign(L, 0.0f);
  for (int64_t r = 0; r < n; ++r) {
    const int64_t sl = r / SELL_C, lane = r % SELL_C;
    int64_t q = 0;
    for (int64_t k = A.rp[r]; k < A.rp[r + 1]; ++k, ++q) {
      const int64_t pos = s.slice_ptr[sl] + q * SELL_C + lane;
      s.col[pos] = A.ci[k];
      val[pos] = static_cast<float>(A.v[k]);
    }
  }
  s.map.clear();
}

}  // namespace

void AmgDevice::upload(const AmgHost& h, cudaStream_t s) {
  nlev = static_cast<int>(h.lv.size());
  n0 = h.lv[0].A.n;
  nc = h.lv.back().A.n;
  A.clear(); P.clear(); R.clear(); val.clear(); pval.clear(); rval.clear(); dinv.clear(); vec.clear();
  A.resize(nlev); P.resize(nlev); R.resize(nlev);
  val.resize(nlev); pval.resize(nlev); rval.resize(nlev); dinv.resize(nlev); vec.resize(nlev);
  sizes.assign(nlev, 0);
  nnz.assign(nlev, 0);
  std::vector<AmgLevelDev> d(nlev);
  // grid levels: from the top while the level has enough nonzeros to fill the GPU
  nlev_grid = 0;
  for (int l = 0; l + 1 < nlev; ++l) {
    if (static_cast<int64_t>(h.lv[l].A.ci.size()) < 200000) break;
    nlev_grid = l + 1;
  }
  for (int l = 0; l < nlev; ++l) {
    const AmgHostLevel& L = h.lv[l];
    sizes[l] = L.A.n;
    nnz[l] = static_cast<int64_t>(L.A.ci.size());
    HostSell hs;
    std::vector<float> v;
    csr_to_sell(L.A, hs, v);
    A[l].upload(hs, s);
    val[l].upload(v, s);
    std::vector<float> di(L.dinv.begin(), L.dinv.end());
    dinv[l].upload(di, s);
    vec[l].alloc(5 * static_cast<size_t>(L.A.n));
    vec[l].zero(s);
    AmgLevelDev& D = d[l];
    D.n = L.A.n;
    D.nslices = hs.nslices;
    D.sp = A[l].slice_ptr.p;
    D.col = A[l].col.p;
    D.val = val[l].p;
    D.dinv = dinv[l].p;
    D.b = vec[l].p;
    D.x = vec[l].p + L.A.n;
    D.x2 = vec[l].p + 2 * L.A.n;
    D.d = vec[l].p + 3 * L.A.n;
    D.r = vec[l].p + 4 * L.A.n;
    D.p_nslices = D.r_nslices = 0;
    D.p_sp = D.r_sp = nullptr;
    D.p_col = D.r_col = nullptr;
    D.p_val = D.r_val = nullptr;
    if (l + 1 < nlev) {
      HostSell hp, hr;
      std::vector<float> vp, vr;
      csr_to_sell(L.P, hp, vp);
      csr_to_sell(L.R, hr, vr);
      P[l].upload(hp, s);
      R[l].upload(hr, s);
      pval[l].upload(vp, s);
      rval[l].upload(vr, s);
      D.p_nslices = hp.nslices;
      D.p_sp = P[l].slice_ptr.p;
      D.p_col = P[l].col.p;
      D.p_val = pval[l].p;
      D.r_nslices = hr.nslices;
      D.r_sp = R[l].slice_ptr.p;
      D.r_col = R[l].col.p;
      D.r_val = rval[l].p;
      const double b = 1.1 * L.lmax, a = 0.1 * L.lmax;
      D.theta = static_cast<float>(0.5 * (b + a));
      D.delta = static_cast<float>(0.5 * (b - a));
      D.sigma = static_cast<float>((b + a) / (b - a));
    } else {
      D.theta = D.delta = D.sigma = 1.0f;
    }
    D.cta = l >= nlev_grid ? 1 : 0;
  }
  lv.upload(d, s);
  std::vector<float> ci(h.coarse_inv.begin(), h.coarse_inv.end());
  cinv.upload(ci, s);
  SPX_CUDA(cudaStreamSynchronize(s));
}

int64_t AmgDevice::device_bytes() const {
  int64_t t = cinv.bytes() + lv.bytes();
  for (int l = 0; l < nlev; ++l) {
    t += A[l].slice_ptr.bytes() + A[l].col.bytes() + P[l].slice_ptr.bytes() + P[l].col.bytes() +
         R[l].slice_ptr.bytes() + R[l].col.bytes() + val[l].bytes() + pval[l].bytes() + rval[l].bytes() +
         dinv[l].bytes() + vec[l].bytes();
  }
  return t;
}

// ------------------------------------------------------------------ device phases
namespace {

constexpr int PCG_BLOCK = 1024;

struct RowRange {
  int64_t gw, nw;  // first warp, warp stride
  int lane;
};

__device__ __forceinline__ float sell_dot(const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                                          const float* __restrict__ val, int64_t sl, int lane,
                                          const float* __restrict__ v) {
  const int64_t base = sp[sl];
  const int width = static_cast<int>((sp[sl + 1] - base) >> 5);
  float acc = 0.0f;
  int k = 0;
  for (; k + 2 <= width; k += 2) {
    const int64_t i0 = base + (static_cast<int64_t>(k) << 5) + lane;
    const int64_t i1 = i0 + 32;
    const float a0 = val[i0], a1 = val[i1];
    const int32_t c0 = col[i0], c1 = col[i1];
    acc += a0 * v[c0];
    acc += a1 * v[c1];
  }
  if (k < width) {
    const int64_t i0 = base + (static_cast<int64_t>(k) << 5) + lane;
    acc += val[i0] * v[col[i0]];
  }
  return acc;
}

// pre-smoothing from x = 0, Chebyshev step 1 and 2 (one SpMV: A d0, d0 = D^-1 b / theta)
__device__ void pre_a(const AmgLevelDev& L, RowRange rr) {
  const float rho0 = 1.0f / L.sigma, rho1 = 1.0f / (2.0f * L.sigma - rho0);
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const int64_t base = L.sp[sl];
    const int width = static_cast<int>((L.sp[sl + 1] - base) >> 5);
    float t = 0.0f;
    for (int k = 0; k < width; ++k) {
      const int64_t idx = base + (static_cast<int64_t>(k) << 5) + rr.lane;
      const int32_t c = L.col[idx];
      t += L.val[idx] * (L.dinv[c] * L.b[c]);
    }
    if (i < L.n) {
      const float di = L.dinv[i], bi = L.b[i];
      const float d0 = di * bi / L.theta;
      const float r1 = di * (bi - t / L.theta);
      const float d1 = rho1 * rho0 * d0 + (2.0f * rho1 / L.delta) * r1;
      L.x[i] = d0 + d1;
      L.d[i] = d1;
      L.r[i] = r1;
    }
  }
}

// residual b - A x after pre-smoothing (A d1), stored in r
__device__ void pre_b(const AmgLevelDev& L, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const float t = sell_dot(L.sp, L.col, L.val, sl, rr.lane, L.d);
    if (i < L.n) {
      const float di = L.dinv[i];
      L.r[i] = (L.r[i] - di * t) / di;
    }
  }
}

__device__ void restrict_to(const AmgLevelDev& L, const AmgLevelDev& C, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.r_nslices; sl += rr.nw) {
    const int64_t a = sl * 32 + rr.lane;
    const float t = sell_dot(L.r_sp, L.r_col, L.r_val, sl, rr.lane, L.r);
    if (a < C.n) C.b[a] = t;
  }
}

__device__ void prolong_from(const AmgLevelDev& L, const AmgLevelDev& C, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.p_nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const float t = sell_dot(L.p_sp, L.p_col, L.p_val, sl, rr.lane, C.x);
    if (i < L.n) L.x[i] += t;
  }
}

// post-smoothing from x, Chebyshev step 1 (r0 = D^-1 (b - A x), x2 = x + r0 / theta)
__device__ void post_c(const AmgLevelDev& L, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const float t = sell_dot(L.sp, L.col, L.val, sl, rr.lane, L.x);
    if (i < L.n) {
      const float r0 = L.dinv[i] * (L.b[i] - t);
      const float d0 = r0 / L.theta;
      L.x2[i] = L.x[i] + d0;
      L.d[i] = d0;
      L.r[i] = r0;
    }
  }
}

// post-smoothing step 2; optionally the partial dots (r64, z) and (w, z) of the FP64 PCG
__device__ void post_d(const AmgLevelDev& L, RowRange rr, const double* __restrict__ r64,
                       const double* __restrict__ sdinv, double& rz, double& wz, bool dots) {
  const float rho0 = 1.0f / L.sigma, rho1 = 1.0f / (2.0f * L.sigma - rho0);
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const float t = sell_dot(L.sp, L.col, L.val, sl, rr.lane, L.d);
    if (i < L.n) {
      const float r1 = L.r[i] - L.dinv[i] * t;
      const float d1 = rho1 * rho0 * L.d[i] + (2.0f * rho1 / L.delta) * r1;
      const float z = L.x2[i] + d1;
      L.x[i] = z;
      if (dots) {
        rz += r64[i] * static_cast<double>(z);
        wz += static_cast<double>(z) / sdinv[i];
      }
    }
  }
}

// x = C^-1 b on the dense coarsest level (warps over rows, lanes over columns)
__device__ void coarse_solve(const AmgLevelDev& L, const float* __restrict__ cinv, int64_t nc) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int64_t i = warp; i < nc; i += nw) {
    float s = 0.0f;
    for (int64_t j = lane; j < nc; j += 32) s += cinv[i * nc + j] * L.b[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) L.x[i] = s;
  }
}

template <class TV>
struct PcgParams {
  int64_t n, nslices;
  const int64_t* sp;
  const int32_t* col;
  const double* v64;
  const double* sdinv;
  const double* diag;
  const TV* b;
  TV* x;
  double *bh, *y, *r, *p, *q;
  double* part;
  unsigned int* bar;
  int* err;
  int* iters;
  double* resid;
  unsigned long long* iters_acc;
  double* res_acc;
  double rtol, atol, ww;
  int maxit, max_outer, warm, project;
  const AmgLevelDev* lv;
  int nlev, nlev_grid;
  const float* cinv;
  int64_t nc;
};

#define PCG_ROWS_BEGIN                                              \
  for (int64_t sl = gw; sl < P.nslices; sl += nw) {                 \
    const int64_t row = sl * 32 + lane;                             \
    const int64_t base = P.sp[sl];                                  \
    const int width = static_cast<int>((P.sp[sl + 1] - base) >> 5); \
    (void)base; (void)width;                                        \
    if (row < n) {
#define PCG_ROWS_END \
  }                  \
  }

// z = V(r): lv[0].b holds r (FP32) on entry, lv[0].x holds z on exit; when the top level is
// a grid level its last phase also writes the partial dots (r, z), (w, z) to `slot`.
template <class TV>
__device__ bool vcycle(const PcgParams<TV>& P, int slot, double* sh, bool& dots_done) {
  const unsigned nb = gridDim.x;
  unsigned int* cnt = P.bar;
  unsigned int* gen = P.bar + 1;
  const int lane = threadIdx.x & 31;
  const RowRange grid_rr{static_cast<int64_t>((blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5),
                         static_cast<int64_t>((gridDim.x * static_cast<int64_t>(blockDim.x)) >> 5), lane};
  const RowRange cta_rr{static_cast<int64_t>(threadIdx.x >> 5), static_cast<int64_t>(blockDim.x >> 5), lane};
  const int G = P.nlev_grid, NL = P.nlev;
  for (int l = 0; l < G; ++l) {
    const AmgLevelDev& L = P.lv[l];
    pre_a(L, grid_rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pre_b(L, grid_rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    restrict_to(L, P.lv[l + 1], grid_rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
  }
  if (blockIdx.x == 0) {
    for (int l = G; l + 1 < NL; ++l) {
      const AmgLevelDev& L = P.lv[l];
      pre_a(L, cta_rr);
      __syncthreads();
      pre_b(L, cta_rr);
      __syncthreads();
      restrict_to(L, P.lv[l + 1], cta_rr);
      __syncthreads();
    }
    coarse_solve(P.lv[NL - 1], P.cinv, P.nc);
    __syncthreads();
    for (int l = NL - 2; l >= G; --l) {
      const AmgLevelDev& L = P.lv[l];
      prolong_from(L, P.lv[l + 1], cta_rr);
      __syncthreads();
      post_c(L, cta_rr);
      __syncthreads();
      double a = 0.0, b = 0.0;
      post_d(L, cta_rr, nullptr, nullptr, a, b, false);
      __syncthreads();
    }
  }
  if (!grid_barrier(cnt, gen, nb, P.err)) return false;
  dots_done = false;
  for (int l = G - 1; l >= 0; --l) {
    const AmgLevelDev& L = P.lv[l];
    prolong_from(L, P.lv[l + 1], grid_rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    post_c(L, grid_rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    double rz = 0.0, wz = 0.0;
    post_d(L, grid_rr, P.r, P.sdinv, rz, wz, l == 0);
    if (l == 0) {
      cta_partial(P.part, slot, rz, wz, 0.0, 0.0, sh);
      dots_done = true;
    }
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
  }
  return true;
}

template <class TV>
__global__ void __launch_bounds__(PCG_BLOCK, 1) k_pcg_amg(PcgParams<TV> P) {
  __shared__ double sh[160];
  const unsigned nb = gridDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  unsigned int* cnt = P.bar;
  unsigned int* gen = P.bar + 1;
  const int64_t n = P.n;
  float* b0 = P.lv[0].b;
  const float* z0 = P.lv[0].x;
  double tot[4];
  double meanb = 0.0;
  if (P.project) {
    double part = 0.0;
    PCG_ROWS_BEGIN part += static_cast<double>(P.b[row]);
    PCG_ROWS_END
    cta_partial(P.part, 0, part, 0.0, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
    cta_total(P.part, 0, tot, sh);
    meanb = tot[0] / static_cast<double>(n);
  }
  {
    double bb = 0.0;
    PCG_ROWS_BEGIN
      const double bv = static_cast<double>(P.b[row]) - meanb;
      P.bh[row] = bv * P.sdinv[row];
      if (!P.warm) P.y[row] = 0.0;
      bb += bv * bv;
    PCG_ROWS_END
    cta_partial(P.part, 1, bb, 0.0, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  cta_total(P.part, 1, tot, sh);
  const double bb = tot[0];
  const double tol2 = fmax(P.rtol * P.rtol * bb, P.atol * P.atol);
  int total = 0, outers = 0;
  double rr = 0.0, rr0 = -1.0;
  for (int outer = 0; outer < P.max_outer; ++outer) {
    ++outers;
    // true residual r = bh - A^ y (FP64), its unscaled norm, r -> level-0 right-hand side
    {
      double rh = 0.0;
      PCG_ROWS_BEGIN
        double acc = 0.0;
        for (int k = 0; k < width; ++k) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          acc += P.v64[idx] * P.y[P.col[idx]];
        }
        const double r = P.bh[row] - acc;
        P.r[row] = r;
        b0[row] = static_cast<float>(r);
        rh += P.diag[row] * r * r;
      PCG_ROWS_END
      cta_partial(P.part, 0, rh, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
    }
    cta_total(P.part, 0, tot, sh);
    rr = tot[0];
    if (rr0 < 0.0) rr0 = rr;
    if (rr <= tol2 || total >= P.maxit) break;
    double rz_old = 1.0;
    for (int it = 0;; ++it) {
      bool dots = false;
      if (!vcycle(P, 2, sh, dots)) return;
      if (!dots) {  // no grid level: dots over the whole grid after the CTA-0 cycle
        double rz = 0.0, wz = 0.0;
        PCG_ROWS_BEGIN
          const double z = static_cast<double>(z0[row]);
          rz += P.r[row] * z;
          wz += z / P.sdinv[row];
        PCG_ROWS_END
        cta_partial(P.part, 2, rz, wz, 0.0, 0.0, sh);
        if (!grid_barrier(cnt, gen, nb, P.err)) return;
      }
      cta_total(P.part, 2, tot, sh);
      const double rz = tot[0];
      const double c = P.project && P.ww > 0.0 ? tot[1] / P.ww : 0.0;
      const double beta = it == 0 ? 0.0 : rz / rz_old;
      double pq = 0.0;
      PCG_ROWS_BEGIN
        double acc = 0.0;
        for (int k = 0; k < width; ++k) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          acc += P.v64[idx] * static_cast<double>(z0[P.col[idx]]);
        }
        const double z = static_cast<double>(z0[row]);
        const double w = 1.0 / P.sdinv[row];
        const double pv = (z - c * w) + (it == 0 ? 0.0 : beta * P.p[row]);
        const double qv = acc + (it == 0 ? 0.0 : beta * P.q[row]);
        P.p[row] = pv;
        P.q[row] = qv;
        pq += pv * qv;
      PCG_ROWS_END
      cta_partial(P.part, 3, pq, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      cta_total(P.part, 3, tot, sh);
      const double pqt = tot[0];
      if (!(pqt > 0.0) || !(rz > 0.0)) break;
      const double alpha = rz / pqt;
      double rh = 0.0;
      PCG_ROWS_BEGIN
        P.y[row] += alpha * P.p[row];
        const double r = P.r[row] - alpha * P.q[row];
        P.r[row] = r;
        b0[row] = static_cast<float>(r);
        rh += P.diag[row] * r * r;
      PCG_ROWS_END
      cta_partial(P.part, 0, rh, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      cta_total(P.part, 0, tot, sh);
      rr = tot[0];
      ++total;
      rz_old = rz;
      // stop a little below the target so that the true residual confirms it
      if (rr <= 0.25 * tol2 || total >= P.maxit) break;
    }
  }
  double mx = 0.0;
  if (P.project) {
    double sx = 0.0;
    PCG_ROWS_BEGIN sx += P.y[row] * P.sdinv[row];
    PCG_ROWS_END
    cta_partial(P.part, 1, sx, 0.0, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
    cta_total(P.part, 1, tot, sh);
    mx = tot[0] / static_cast<double>(n);
  }
  PCG_ROWS_BEGIN
    const double xv = P.y[row] * P.sdinv[row] - mx;
    P.x[row] = static_cast<TV>(xv);
    P.y[row] = xv / P.sdinv[row];
  PCG_ROWS_END
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *P.iters = total;
    *P.resid = bb > 0.0 ? sqrt(rr / bb) : 0.0;
    atomicAdd(P.iters_acc, (unsigned long long)total);
    atomicAdd(P.iters_acc + 1, (unsigned long long)outers);
    atomicAdd(P.iters_acc + 2, 1ull);
    if (bb > 0.0) {
      atomicAdd(P.res_acc, sqrt(fmax(rr0, 0.0) / bb));
      atomicAdd(P.res_acc + 1, sqrt(rr / bb));
    }
  }
}

}  // namespace

// ------------------------------------------------------------------ host entry
template <class TM>
void CgSystem<TM>::enable_amg(const std::vector<int64_t>& rowptr, const std::vector<int32_t>& col,
                              const std::vector<double>& a, const std::vector<double>& d, bool singular,
                              cudaStream_t s) {
  CsrHost Ah;
  Ah.n = n;
  Ah.ncols = n;
  Ah.rp = rowptr;
  Ah.ci = col;
  Ah.v.resize(a.size());
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) Ah.v[k] = a[k] / std::sqrt(d[i] * d[col[k]]);
  std::vector<double> w(n);
  double ww = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    w[i] = std::sqrt(d[i]);
    ww += d[i];
  }
  AmgHost h;
  amg_build(Ah, w, singular, AmgOptions{}, h);
  amg = std::make_unique<AmgDevice>();
  amg->upload(h, s);
  amg_ww = ww;
  amg_singular = singular;
  if (!y64.n) {
    y64.alloc(n);
    y64.zero(s);
  }
  if (!bh64.n) bh64.alloc(n);
  amg_work.alloc(3 * static_cast<size_t>(n));
  if (!vals64.n) {  // FP64 scaled values (the FP64 CG keeps them in vals)
    std::vector<double> v(P.len);
    SPX_CUDA(cudaMemcpy(v.data(), vals.p, P.len * sizeof(double), cudaMemcpyDeviceToHost));
    vals64.upload(v, s);
  }
  int per_sm = 0;
  SPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_amg<double>, PCG_BLOCK, 0));
  SPX_CHECK(per_sm > 0, "AMG PCG kernel cannot be resident");
  int dev;
  SPX_CUDA(cudaGetDevice(&dev));
  const int64_t want = (P.nslices * 32 + PCG_BLOCK - 1) / PCG_BLOCK;
  amg_grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, num_sms(dev))));
  if (part.n < 4 * 4 * static_cast<size_t>(amg_grid)) part.alloc(4 * 4 * static_cast<size_t>(amg_grid));
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class TM>
template <class TV>
void CgSystem<TM>::launch_amg(const TV* b, TV* x, double rtol, double atol, int maxit, bool warm, bool project,
                              cudaStream_t st) {
  PcgParams<TV> q;
  q.n = n; q.nslices = P.nslices; q.sp = P.slice_ptr.p; q.col = P.col.p;
  q.v64 = vals64.p; q.sdinv = sdinv64.p; q.diag = diag64.p;
  q.b = b; q.x = x;
  q.bh = bh64.p; q.y = y64.p;
  q.r = amg_work.p; q.p = amg_work.p + n; q.q = amg_work.p + 2 * n;
  q.part = part.p; q.bar = bar.p; q.err = err.p; q.iters = iters.p; q.resid = resid.p;
  q.iters_acc = iters_acc.p; q.res_acc = res_acc.p;
  q.rtol = rtol; q.atol = atol; q.ww = amg_singular ? amg_ww : 0.0;
  q.maxit = maxit; q.max_outer = max_outer; q.warm = warm ? 1 : 0; q.project = project ? 1 : 0;
  q.lv = amg->lv.p; q.nlev = amg->nlev; q.nlev_grid = amg->nlev_grid; q.cinv = amg->cinv.p; q.nc = amg->nc;
  void* args[] = {&q};
  SPX_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_pcg_amg<TV>), dim3(amg_grid), dim3(PCG_BLOCK),
                                       args, 0, st));
}

template void CgSystem<double>::enable_amg(const std::vector<int64_t>&, const std::vector<int32_t>&,
                                           const std::vector<double>&, const std::vector<double>&, bool,
                                           cudaStream_t);
template void CgSystem<float>::enable_amg(const std::vector<int64_t>&, const std::vector<int32_t>&,
                                          const std::vector<double>&, const std::vector<double>&, bool,
                                          cudaStream_t);
template void CgSystem<double>::launch_amg<double>(const double*, double*, double, double, int, bool, bool,
                                                   cudaStream_t);
template void CgSystem<float>::launch_amg<double>(const double*, double*, double, double, int, bool, bool,
                                                  cudaStream_t);
template void CgSystem<float>::launch_amg<float>(const float*, float*, double, double, int, bool, bool,
                                                 cudaStream_t);

}  // namespace spx
