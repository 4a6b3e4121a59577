// Device side of the smoothed-aggregation AMG (amg.cuh): level upload, the FP32 V-cycle
// and the FP64 preconditioned CG that uses it, in one persistent cooperative kernel.
//
// Level layout: A_l and P_l are SELL-32 (one thread per row, 32 rows per slice, padding
// entries point at column 0 with value 0); R_l = P_l^T is CSR swept by `r_lanes` lanes per
// row (its rows are long); FP32 values; FP32 vectors b, D^-1 b, x, x2, d, r per level.  Every
// phase is swept by the whole grid with a grid barrier after it; the dense coarsest level
// (at most a few thousand unknowns) is one GEMV with its precomputed inverse, a warp per row.
//
// PCG (FP64 vectors, scaled system A^ = D^-1/2 A D^-1/2):
//   z = V(r);  beta = (r,z)/(r,z)_old;  c = (w,z)/(w,w) (singular systems: remove the
//   null-vector component w = D^1/2 1 from z);  p = z - c w + beta p;
//   q = A^ z + beta q  (A^ w = 0, so q = A^ p without a second SpMV), with A^ z evaluated as
//   D^-1/2 [sum_j a_ij (u_j - u_i) + (sum_j a_ij) u_i], u = D^-1/2 z, FP32 a_ij, FP64 sums
//   (the level-0 cycle works on the unscaled A and returns u directly, reading the same
//   FP32 a_ij and columns);
//   alpha = (r,z)/(p,q);  y += alpha p;  r -= alpha q.
// The recurrence residual is confirmed against the true FP64 residual (FP64 values) before
// returning; stopping rule ||b - A x|| <= max(rtol ||b||, atol) in the unscaled norm.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "amg.cuh"
#include "fem.cuh"

namespace spx {

std::atomic<int> g_pcg_timing{0};  // phase timing marks of the AMG-PCG kernel (spx_debug_pcg_timing)

// The cycle loads the matrices of its cycled levels with an L2 evict_last policy.  A larger L2
// set-aside for persisting lines (a limit of this process's context, not a GPU setting) can be
// requested with SPX_L2_PERSIST_MB (MiB, raised only, capped by the device's maximum).  It is
// off by default: measured on the 400 x 400 x 2 film, raising it from the context's 24 MB to
// 75 MB left the u1 solve unchanged and slowed the streaming boundary apply by 7 %.
void reserve_persisting_l2(int64_t bytes, int dev) {
  const char* e = std::getenv("SPX_L2_PERSIST_MB");
  if (!e) return;
  bytes = std::atoll(e) << 20;
  if (bytes <= 0) return;
  int mx = 0;
  SPX_CUDA(cudaDeviceGetAttribute(&mx, cudaDevAttrMaxPersistingL2CacheSize, dev));
  if (mx <= 0) return;
  size_t cur = 0;
  SPX_CUDA(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
  const size_t want = std::min<size_t>(static_cast<size_t>(mx), static_cast<size_t>(bytes));
  if (want > cur) SPX_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
}

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

// in-place Gauss-Jordan inverse of an SPD matrix (no pivoting), one pivot per step
__global__ void k_gj_pivot(double* __restrict__ M, double* __restrict__ colk, int64_t n, int64_t k) {
  const double p = M[k * n + k];
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) colk[i] = M[i * n + k];
  __syncthreads();
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) M[k * n + j] = (j == k) ? 1.0 / p : M[k * n + j] / p;
}
__global__ void k_gj_update(double* __restrict__ M, const double* __restrict__ colk, int64_t n, int64_t k) {
  const int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (e >= n * n) return;
  const int64_t i = e / n, j = e - i * n;
  if (i == k) return;
  const double f = colk[i];
  if (j == k)
    M[e] = -f * M[k * n + k];
  else
    M[e] -= f * M[k * n + j];
}
// FP32 copy of an n x n matrix into rows of ld >= n entries (zero padded)
__global__ void k_to_float_rows(const double* __restrict__ a, float* __restrict__ b, int64_t n, int64_t ld) {
  const int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (e >= n * ld) return;
  const int64_t i = e / ld, j = e - i * ld;
  b[e] = j < n ? static_cast<float>(a[i * n + j]) : 0.0f;
}

__global__ void k_f32_to_f16(int64_t n, const float* __restrict__ a, __half* __restrict__ b) {
  const int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (e < n) b[e] = __float2half_rn(a[e]);
}

}  // namespace

void AmgDevice::upload(const AmgHost& h, cudaStream_t s, const int64_t* sp0, const int32_t* col0, const float* val0,
                       int64_t nslices0, int nrep) {
  reps = nrep;
  nlev = static_cast<int>(h.lv.size());
  n0 = h.lv[0].A.n;
  nc = h.lv.back().A.n;
  A.clear(); P.clear(); rrp.clear(); rcol.clear();
  val.clear(); pval.clear(); rval.clear(); dinv.clear(); vec.clear(); val16.clear();
  A.resize(nlev); P.resize(nlev); rrp.resize(nlev); rcol.resize(nlev);
  val.resize(nlev); pval.resize(nlev); rval.resize(nlev); dinv.resize(nlev); vec.resize(nlev); val16.resize(nlev);
  // FP16 values for the cycle's sweeps (tuning option: half the value bytes of every sweep;
  // the PCG product keeps the FP32 values)
  const char* e16 = std::getenv("SPX_AMG_FP16");
  const bool fp16 = e16 && std::atoi(e16) != 0;
  sizes.assign(nlev, 0);
  nnz.assign(nlev, 0);
  pnnz.assign(nlev, 0);
  rnnz.assign(nlev, 0);
  std::vector<AmgLevelDev> d(nlev);
  for (int l = 0; l < nlev; ++l) {
    const AmgHostLevel& L = h.lv[l];
    sizes[l] = L.A.n;
    nnz[l] = static_cast<int64_t>(L.A.ci.size());
    pnnz[l] = static_cast<int64_t>(L.P.ci.size());
    rnnz[l] = static_cast<int64_t>(L.R.ci.size());
    AmgLevelDev& D = d[l];
    std::memset(&D, 0, sizeof(D));
    D.n = L.A.n;
    std::vector<float> di(L.dinv.begin(), L.dinv.end());
    dinv[l].upload(di, s);
    D.dinv = dinv[l].p;
    const int64_t nv = L.A.n * reps;  // every level vector holds the reps blocks one after the other
    vec[l].alloc(6 * static_cast<size_t>(nv));
    vec[l].zero(s);
    D.b = vec[l].p;
    D.db = vec[l].p + nv;
    D.x = vec[l].p + 2 * nv;
    D.x2 = vec[l].p + 3 * nv;
    D.d = vec[l].p + 4 * nv;
    D.r = vec[l].p + 5 * nv;
    if (l + 1 == nlev) break;  // dense coarsest: vectors only
    HostSell hs, hp;
    std::vector<float> v, vp;
    int64_t vlen = 0;
    if (l == 0 && sp0) {
      D.nslices = nslices0;
      D.sp = sp0;
      D.col = col0;
      D.val = val0;
      SPX_CUDA(cudaMemcpyAsync(&vlen, sp0 + nslices0, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      SPX_CUDA(cudaStreamSynchronize(s));
    } else {
      csr_to_sell(L.A, hs, v);
      A[l].upload(hs, s);
      val[l].upload(v, s);
      D.nslices = hs.nslices;
      D.sp = A[l].slice_ptr.p;
      D.col = A[l].col.p;
      D.val = val[l].p;
      vlen = static_cast<int64_t>(v.size());
    }
    D.val16 = nullptr;
    if (fp16 && vlen > 0) {
      val16[l].alloc(vlen);
      k_f32_to_f16<<<grid_for(vlen, 256), 256, 0, s>>>(vlen, D.val, val16[l].p);
      SPX_LAUNCH_CHECK();
      D.val16 = val16[l].p;
    }
    csr_to_sell(L.P, hp, vp);
    P[l].upload(hp, s);
    pval[l].upload(vp, s);
    D.p_nslices = hp.nslices;
    D.p_sp = P[l].slice_ptr.p;
    D.p_col = P[l].col.p;
    D.p_val = pval[l].p;
    rrp[l].upload(L.R.rp, s);
    rcol[l].upload(L.R.ci, s);
    std::vector<float> vr(L.R.v.begin(), L.R.v.end());
    rval[l].upload(vr, s);
    D.r_rp = rrp[l].p;
    D.r_col = rcol[l].p;
    D.r_val = rval[l].p;
    const double avg = static_cast<double>(L.R.ci.size()) / std::max<int64_t>(L.R.n, 1);
    int lanes = 1;  // about eight entries per lane
    while (lanes < 32 && lanes < avg / 8.0) lanes <<= 1;
    D.r_lanes = lanes;
    const double b = 1.1 * L.lmax, a = 0.1 * L.lmax;
    D.theta = static_cast<float>(0.5 * (b + a));
    D.delta = static_cast<float>(0.5 * (b - a));
    D.sigma = static_cast<float>((b + a) / (b - a));
  }
  lv.upload(d, s);
  // coarsest inverse: FP64 Gauss-Jordan on the device, stored FP32
  {
    DevBuf<double> M, colk;
    M.upload(h.coarse_dense, s);
    colk.alloc(std::max<int64_t>(nc, 1));
    const int64_t nn = nc * nc;
    for (int64_t k = 0; k < nc; ++k) {
      k_gj_pivot<<<1, 1024, 0, s>>>(M.p, colk.p, nc, k);
      k_gj_update<<<grid_for(nn, 256), 256, 0, s>>>(M.p, colk.p, nc, k);
    }
    SPX_LAUNCH_CHECK();
    ldc = (nc + 3) / 4 * 4;  // rows of 16-byte vectors
    cinv.alloc(std::max<int64_t>(nc * ldc, 1));
    k_to_float_rows<<<grid_for(nc * ldc, 256), 256, 0, s>>>(M.p, cinv.p, nc, ldc);
    SPX_LAUNCH_CHECK();
    SPX_CUDA(cudaStreamSynchronize(s));
  }
}

int64_t AmgDevice::device_bytes() const {
  int64_t t = cinv.bytes() + lv.bytes();
  for (int l = 0; l < nlev; ++l) {
    t += A[l].slice_ptr.bytes() + A[l].col.bytes() + P[l].slice_ptr.bytes() + P[l].col.bytes() + rrp[l].bytes() +
         rcol[l].bytes() + val[l].bytes() + pval[l].bytes() + rval[l].bytes() + dinv[l].bytes() + vec[l].bytes();
  }
  return t;
}

// ------------------------------------------------------------------ device phases
namespace {

#ifndef SPX_PCG_BLOCK
#define SPX_PCG_BLOCK 1024
#endif
#ifndef SPX_PCG_CTAS_PER_SM
#define SPX_PCG_CTAS_PER_SM 1
#endif
#ifndef SPX_PCG_BLOCK_R
#define SPX_PCG_BLOCK_R 512
#endif
constexpr int PCG_BLOCK = SPX_PCG_BLOCK;          // threads per CTA
// the R-block kernels keep R values per row in registers: fewer threads, more registers each
constexpr int PCG_BLOCK_R = SPX_PCG_BLOCK_R;
constexpr int PCG_CTAS_PER_SM = SPX_PCG_CTAS_PER_SM;  // resident CTAs per SM (all SMs filled)

struct RowRange {
  int64_t gw, nw;  // first warp, warp stride
  int lane;
};

// L2 residency hints.  The cycle's matrices (level 0: ~8 B per nonzero, read five times per
// PCG iteration together with the PCG product) are loaded with an evict_last policy so that
// they stay in L2 across the phases and iterations while vectors, transfer operators and the
// FP64 true-residual values stream past them (those use evict_first where read once).
__device__ __forceinline__ uint64_t l2_policy_keep() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_stream() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ float ld_hint(const float* a, uint64_t pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ int32_t ld_hint(const int32_t* a, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_hint(const double* a, uint64_t pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ float4 ld_hint4(const float4* a, uint64_t pol) {
  float4 v;
  asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(a), "l"(pol));
  return v;
}

__device__ __forceinline__ float ld_hint(const __half* a, uint64_t pol) {
  unsigned short v;
  asm("ld.global.nc.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(v) : "l"(a), "l"(pol));
  return __half2float(__ushort_as_half(v));
}

// row dot products of one SELL-32 slice (values and columns are read-only for the kernel's
// lifetime; loaded with the L2 policy `pol`); VT = float or __half values
template <class VT>
__device__ __forceinline__ float sell_dot(const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                                          const VT* __restrict__ val, int64_t sl, int lane,
                                          const float* __restrict__ v, uint64_t pol) {
  const int64_t base = sp[sl];
  const int width = static_cast<int>((sp[sl + 1] - base) >> 5);
  const VT* vv = val + base + lane;
  const int32_t* cc = col + base + lane;
  float a0 = 0.0f, a1 = 0.0f;
  int k = 0;
  for (; k + 8 <= width; k += 8) {  // eight gathers in flight per thread
    float w[8];
    int32_t c[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      w[u] = ld_hint(vv + (k + u) * 32, pol);
      c[u] = ld_hint(cc + (k + u) * 32, pol);
    }
#pragma unroll
    for (int u = 0; u < 8; u += 2) {
      a0 += w[u] * v[c[u]];
      a1 += w[u + 1] * v[c[u + 1]];
    }
  }
  for (; k + 2 <= width; k += 2) {
    const float w0 = ld_hint(vv + k * 32, pol), w1 = ld_hint(vv + (k + 1) * 32, pol);
    const int32_t c0 = ld_hint(cc + k * 32, pol), c1 = ld_hint(cc + (k + 1) * 32, pol);
    a0 += w0 * v[c0];
    a1 += w1 * v[c1];
  }
  if (k < width) a0 += ld_hint(vv + k * 32, pol) * v[ld_hint(cc + k * 32, pol)];
  return a0 + a1;
}

// Slice bounds of SELL-32 slice sl (zero width past the last slice); the PCG product phase
// loads the bounds of a warp's next slice while it works on the current one.
__device__ __forceinline__ void slice_bounds(const int64_t* __restrict__ sp, int64_t sl, int64_t ns, int64_t& base,
                                             int& width) {
  if (sl < ns) {
    base = sp[sl];
    width = static_cast<int>((sp[sl + 1] - base) >> 5);
  } else {
    base = 0;
    width = 0;
  }
}

// level matrix times a level vector for one slice, with the FP16 sweep values when present
__device__ __forceinline__ float lvl_dot(const AmgLevelDev& L, int64_t sl, int lane, const float* __restrict__ v) {
  return L.val16 ? sell_dot(L.sp, L.col, L.val16, sl, lane, v, l2_policy_keep())
                 : sell_dot(L.sp, L.col, L.val, sl, lane, v, l2_policy_keep());
}

// pre-smoothing from x = 0, Chebyshev steps 1 and 2 (one SpMV: A d0, d0 = D^-1 b / theta)
__device__ void pre_a(const AmgLevelDev& L, RowRange rr) {
  const float rho0 = 1.0f / L.sigma, rho1 = 1.0f / (2.0f * L.sigma - rho0);
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const float t = lvl_dot(L, sl, rr.lane, L.db);
    if (i < L.n) {
      const float di = L.dinv[i];
      const float d0 = L.db[i] / L.theta;
      const float r1 = L.db[i] - di * t / L.theta;
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
    const float t = lvl_dot(L, sl, rr.lane, L.d);
    if (i < L.n) {
      const float di = L.dinv[i];
      L.r[i] = (L.r[i] - di * t) / di;
    }
  }
}

// b_c = R r (CSR rows, `r_lanes` lanes per row), db_c = D_c^-1 b_c
__device__ void restrict_to(const AmgLevelDev& L, const AmgLevelDev& C, RowRange rr) {
  const int G = L.r_lanes;
  const int gl = rr.lane & (G - 1);
  const int64_t rows_per_warp = 32 / G;
  const int64_t first = rr.gw * rows_per_warp + rr.lane / G, stride = rr.nw * rows_per_warp;
  const int64_t nrows_pad = (C.n + rows_per_warp - 1) / rows_per_warp * rows_per_warp;
  for (int64_t a = first - rr.lane / G; a < nrows_pad; a += stride) {  // uniform per warp
    const int64_t row = a + rr.lane / G;
    float t = 0.0f;
    if (row < C.n) {
      const int64_t k1 = L.r_rp[row + 1];
      int64_t k = L.r_rp[row] + gl;
      for (; k + 3 * G < k1; k += 4 * G) {  // four gathers in flight per lane
        const float w0 = L.r_val[k], w1 = L.r_val[k + G], w2 = L.r_val[k + 2 * G], w3 = L.r_val[k + 3 * G];
        const int32_t c0 = L.r_col[k], c1 = L.r_col[k + G], c2 = L.r_col[k + 2 * G], c3 = L.r_col[k + 3 * G];
        t += w0 * L.r[c0] + w1 * L.r[c1] + w2 * L.r[c2] + w3 * L.r[c3];
      }
      for (; k < k1; k += G) t += L.r_val[k] * L.r[L.r_col[k]];
    }
    for (int o = G >> 1; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (row < C.n && gl == 0) {
      C.b[row] = t;
      C.db[row] = C.dinv[row] * t;
    }
  }
}

__device__ void prolong_from(const AmgLevelDev& L, const AmgLevelDev& C, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.p_nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const float t = sell_dot(L.p_sp, L.p_col, L.p_val, sl, rr.lane, C.x, l2_policy_stream());
    if (i < L.n) L.x[i] += t;
  }
}

// post-smoothing from x, Chebyshev step 1 (r0 = D^-1 (b - A x), x2 = x + r0 / theta)
__device__ void post_c(const AmgLevelDev& L, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const float t = lvl_dot(L, sl, rr.lane, L.x);
    if (i < L.n) {
      const float r0 = L.db[i] - L.dinv[i] * t;
      const float d0 = r0 / L.theta;
      L.x2[i] = L.x[i] + d0;
      L.d[i] = d0;
      L.r[i] = r0;
    }
  }
}

// post-smoothing step 2; on the top level also the partial dots (r64, z^), (w, z^) of the PCG
__device__ void post_d(const AmgLevelDev& L, RowRange rr, const double* __restrict__ r64,
                       const double* __restrict__ sdinv, double& rz, double& wz, bool top) {
  const float rho0 = 1.0f / L.sigma, rho1 = 1.0f / (2.0f * L.sigma - rho0);
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    const float t = lvl_dot(L, sl, rr.lane, L.d);
    if (i < L.n) {
      const float r1 = L.r[i] - L.dinv[i] * t;
      const float d1 = rho1 * rho0 * L.d[i] + (2.0f * rho1 / L.delta) * r1;
      const float z = L.x2[i] + d1;
      L.x[i] = z;
      if (top) {  // level 0 runs unscaled: z is u = D^-1/2 z^, z^ = u / sdinv
        const double zh = static_cast<double>(z) / sdinv[i];
        rz += r64[i] * zh;
        wz += zh / sdinv[i];
      }
    }
  }
}

// x = C^-1 b on the dense coarsest level: a warp per row over the grid, 16-byte loads of the
// zero-padded rows (ld = nc rounded up to 4; b is read up to ld, inside the level's vectors)
__device__ void coarse_solve(const AmgLevelDev& L, const float* __restrict__ cinv, int64_t nc, int64_t ldc,
                             RowRange rr) {
  const int64_t nv = ldc / 4;
  const uint64_t pol = l2_policy_keep();  // the inverse stays in L2 across iterations
  const float4* b4 = reinterpret_cast<const float4*>(L.b);
  for (int64_t i = rr.gw; i < nc; i += rr.nw) {
    const float4* row = reinterpret_cast<const float4*>(cinv + i * ldc);
    float s = 0.0f;
#pragma unroll 4
    for (int64_t j = rr.lane; j < nv; j += 32) {
      const float4 c = ld_hint4(row + j, pol);
      const float4 b = b4[j];
      s += c.x * b.x + c.y * b.y + c.z * b.z + c.w * b.w;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (rr.lane == 0) L.x[i] = s;
  }
}

// ---- R identical blocks (a batch of samples of one mesh): the matrix of one block and its
// hierarchy are stored once.  The cycle's level vectors and the PCG work vectors r, p, q hold
// the R blocks interleaved ([row][R]), so the R entries of a column are one vector load (8, 16
// or 32 bytes); the PCG's right-hand side, solution and iterate (b, x, y, bh) keep the
// ensemble's block order ([R][n]).  Each phase reads a matrix slice once.

template <int R> struct VecR;
template <> struct VecR<2> { using T = float2; };
template <> struct VecR<4> { using T = float4; };
template <int R>
__device__ __forceinline__ void load_r(const float* __restrict__ v, int64_t c, float (&g)[R]) {
  if constexpr (R == 8) {
    const float4 a = reinterpret_cast<const float4*>(v + c * 8)[0];
    const float4 b = reinterpret_cast<const float4*>(v + c * 8)[1];
    g[0] = a.x; g[1] = a.y; g[2] = a.z; g[3] = a.w; g[4] = b.x; g[5] = b.y; g[6] = b.z; g[7] = b.w;
  } else if constexpr (R == 4) {
    const float4 a = reinterpret_cast<const float4*>(v)[c];
    g[0] = a.x; g[1] = a.y; g[2] = a.z; g[3] = a.w;
  } else if constexpr (R == 2) {
    const float2 a = reinterpret_cast<const float2*>(v)[c];
    g[0] = a.x; g[1] = a.y;
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r) g[r] = v[c * R + r];
  }
}

template <int R>
__device__ __forceinline__ void store_r(float* __restrict__ v, int64_t c, const float (&g)[R]) {
  if constexpr (R == 8) {
    reinterpret_cast<float4*>(v + c * 8)[0] = make_float4(g[0], g[1], g[2], g[3]);
    reinterpret_cast<float4*>(v + c * 8)[1] = make_float4(g[4], g[5], g[6], g[7]);
  } else if constexpr (R == 4) {
    reinterpret_cast<float4*>(v)[c] = make_float4(g[0], g[1], g[2], g[3]);
  } else if constexpr (R == 2) {
    reinterpret_cast<float2*>(v)[c] = make_float2(g[0], g[1]);
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r) v[c * R + r] = g[r];
  }
}

// R interleaved FP64 entries of row c ([row][R], R even): 16-byte loads and stores
template <int R>
__device__ __forceinline__ void load_r64(const double* __restrict__ v, int64_t c, double (&g)[R]) {
  static_assert(R % 2 == 0, "R even");
  const double2* p = reinterpret_cast<const double2*>(v + c * R);
#pragma unroll
  for (int h = 0; h < R / 2; ++h) {
    const double2 a = p[h];
    g[2 * h] = a.x;
    g[2 * h + 1] = a.y;
  }
}
template <int R>
__device__ __forceinline__ void store_r64(double* __restrict__ v, int64_t c, const double (&g)[R]) {
  double2* p = reinterpret_cast<double2*>(v + c * R);
#pragma unroll
  for (int h = 0; h < R / 2; ++h) p[h] = make_double2(g[2 * h], g[2 * h + 1]);
}

template <int R>
__device__ __forceinline__ void sell_dot_r(const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                                           const float* __restrict__ val, int64_t sl, int lane,
                                           const float* __restrict__ v, uint64_t pol, float (&t)[R]) {
  constexpr int KB = R >= 8 ? 4 : 8;  // columns in flight per thread
  const int64_t base = sp[sl];
  const int width = static_cast<int>((sp[sl + 1] - base) >> 5);
  const float* vv = val + base + lane;
  const int32_t* cc = col + base + lane;
#pragma unroll
  for (int r = 0; r < R; ++r) t[r] = 0.0f;
  for (int k = 0; k < width; k += KB) {  // the last round predicated
    float w[KB];
    int32_t c[KB];
#pragma unroll
    for (int u = 0; u < KB; ++u) {
      const bool in = k + u < width;
      w[u] = in ? ld_hint(vv + (k + u) * 32, pol) : 0.0f;
      c[u] = in ? ld_hint(cc + (k + u) * 32, pol) : 0;
    }
    float g[KB][R];
#pragma unroll
    for (int u = 0; u < KB; ++u) load_r<R>(v, c[u], g[u]);
#pragma unroll
    for (int u = 0; u < KB; ++u)
#pragma unroll
      for (int r = 0; r < R; ++r) t[r] += w[u] * g[u][r];
  }
}

template <int R>
__device__ void pre_a_r(const AmgLevelDev& L, RowRange rr) {
  const float rho0 = 1.0f / L.sigma, rho1 = 1.0f / (2.0f * L.sigma - rho0);
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    float t[R];
    sell_dot_r<R>(L.sp, L.col, L.val, sl, rr.lane, L.db, l2_policy_keep(), t);
    if (i < L.n) {
      const float di = L.dinv[i];
      float db[R], xo[R], dd[R], ro[R];
      load_r<R>(L.db, i, db);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float d0 = db[r] / L.theta;
        const float r1 = db[r] - di * t[r] / L.theta;
        const float d1 = rho1 * rho0 * d0 + (2.0f * rho1 / L.delta) * r1;
        xo[r] = d0 + d1;
        dd[r] = d1;
        ro[r] = r1;
      }
      store_r<R>(L.x, i, xo);
      store_r<R>(L.d, i, dd);
      store_r<R>(L.r, i, ro);
    }
  }
}

template <int R>
__device__ void pre_b_r(const AmgLevelDev& L, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    float t[R];
    sell_dot_r<R>(L.sp, L.col, L.val, sl, rr.lane, L.d, l2_policy_keep(), t);
    if (i < L.n) {
      const float di = L.dinv[i];
      float rv[R];
      load_r<R>(L.r, i, rv);
#pragma unroll
      for (int r = 0; r < R; ++r) rv[r] = (rv[r] - di * t[r]) / di;
      store_r<R>(L.r, i, rv);
    }
  }
}

template <int R>
__device__ void restrict_to_r(const AmgLevelDev& L, const AmgLevelDev& C, RowRange rr) {
  const int G = L.r_lanes;
  const int gl = rr.lane & (G - 1);
  const int64_t rows_per_warp = 32 / G;
  const int64_t first = rr.gw * rows_per_warp + rr.lane / G, stride = rr.nw * rows_per_warp;
  const int64_t nrows_pad = (C.n + rows_per_warp - 1) / rows_per_warp * rows_per_warp;
  for (int64_t a = first - rr.lane / G; a < nrows_pad; a += stride) {  // uniform per warp
    const int64_t row = a + rr.lane / G;
    float t[R];
#pragma unroll
    for (int r = 0; r < R; ++r) t[r] = 0.0f;
    if (row < C.n) {
      const int64_t k1 = L.r_rp[row + 1];
      int64_t k = L.r_rp[row] + gl;
      for (; k + G < k1; k += 2 * G) {  // two gathers in flight per lane
        const float w0 = L.r_val[k], w1 = L.r_val[k + G];
        const int32_t c0 = L.r_col[k], c1 = L.r_col[k + G];
        float g0[R], g1[R];
        load_r<R>(L.r, c0, g0);
        load_r<R>(L.r, c1, g1);
#pragma unroll
        for (int r = 0; r < R; ++r) t[r] += w0 * g0[r] + w1 * g1[r];
      }
      for (; k < k1; k += G) {
        const float w = L.r_val[k];
        float g[R];
        load_r<R>(L.r, L.r_col[k], g);
#pragma unroll
        for (int r = 0; r < R; ++r) t[r] += w * g[r];
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
      for (int o = G >> 1; o > 0; o >>= 1) t[r] += __shfl_xor_sync(0xffffffffu, t[r], o);
    if (row < C.n && gl == 0) {
      const float dc = C.dinv[row];
      float dbv[R];
#pragma unroll
      for (int r = 0; r < R; ++r) dbv[r] = dc * t[r];
      store_r<R>(C.b, row, t);
      store_r<R>(C.db, row, dbv);
    }
  }
}

template <int R>
__device__ void prolong_from_r(const AmgLevelDev& L, const AmgLevelDev& C, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.p_nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    float t[R];
    sell_dot_r<R>(L.p_sp, L.p_col, L.p_val, sl, rr.lane, C.x, l2_policy_stream(), t);
    if (i < L.n) {
      float xv[R];
      load_r<R>(L.x, i, xv);
#pragma unroll
      for (int r = 0; r < R; ++r) xv[r] += t[r];
      store_r<R>(L.x, i, xv);
    }
  }
}

template <int R>
__device__ void post_c_r(const AmgLevelDev& L, RowRange rr) {
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    float t[R];
    sell_dot_r<R>(L.sp, L.col, L.val, sl, rr.lane, L.x, l2_policy_keep(), t);
    if (i < L.n) {
      const float di = L.dinv[i];
      float db[R], xv[R], x2[R], dd[R], ro[R];
      load_r<R>(L.db, i, db);
      load_r<R>(L.x, i, xv);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float r0 = db[r] - di * t[r];
        const float d0 = r0 / L.theta;
        x2[r] = xv[r] + d0;
        dd[r] = d0;
        ro[r] = r0;
      }
      store_r<R>(L.x2, i, x2);
      store_r<R>(L.d, i, dd);
      store_r<R>(L.r, i, ro);
    }
  }
}

// on the top level also the partial dots (r64, z^), (w, z^) over all R blocks; r64 is the
// interleaved PCG residual, sdinv the block-ordered (replicated) scaling
template <int R>
__device__ void post_d_r(const AmgLevelDev& L, RowRange rr, const double* __restrict__ r64,
                         const double* __restrict__ sdinv, double& rz, double& wz, bool top) {
  const float rho0 = 1.0f / L.sigma, rho1 = 1.0f / (2.0f * L.sigma - rho0);
  for (int64_t sl = rr.gw; sl < L.nslices; sl += rr.nw) {
    const int64_t i = sl * 32 + rr.lane;
    float t[R];
    sell_dot_r<R>(L.sp, L.col, L.val, sl, rr.lane, L.d, l2_policy_keep(), t);
    if (i < L.n) {
      const float di = L.dinv[i];
      const double sd = top ? sdinv[i] : 1.0;
      float rv[R], dv[R], x2[R], zo[R];
      load_r<R>(L.r, i, rv);
      load_r<R>(L.d, i, dv);
      load_r<R>(L.x2, i, x2);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float r1 = rv[r] - di * t[r];
        const float d1 = rho1 * rho0 * dv[r] + (2.0f * rho1 / L.delta) * r1;
        const float z = x2[r] + d1;
        zo[r] = z;
        if (top) {
          const double zh = static_cast<double>(z) / sd;
          rz += r64[i * R + r] * zh;
          wz += zh / sd;
        }
      }
      store_r<R>(L.x, i, zo);
    }
  }
}

// dense coarsest level for R blocks (interleaved vectors; b entries past nc are taken as 0)
// the right-hand sides of the dense coarsest level, transposed to [R][nc], for k_pcg_amg_r's
// coarse phase (dynamic shared memory of nc x R floats)
extern __shared__ float pcg_coarse_smem[];

// dense coarsest level for R blocks (interleaved vectors): the CTA stages the R right-hand
// sides in shared memory ([R][nc], one coalesced pass), then a warp per row of the inverse
// reads the row once (L2 evict_last policy, coalesced) against all R of them
template <int R>
__device__ void coarse_solve_r(const AmgLevelDev& L, const float* __restrict__ cinv, int64_t nc, int64_t ldc,
                               RowRange rr) {
  float* sb = pcg_coarse_smem;
  for (int64_t e = threadIdx.x; e < nc * R; e += blockDim.x) {
    const int64_t j = e / R;
    sb[(e - j * R) * nc + j] = L.b[e];
  }
  __syncthreads();
  const uint64_t pol = l2_policy_keep();  // the inverse stays in L2 across iterations
  for (int64_t i = rr.gw; i < nc; i += rr.nw) {
    const float* row = cinv + i * ldc;
    float s[R];
#pragma unroll
    for (int r = 0; r < R; ++r) s[r] = 0.0f;
#pragma unroll 4
    for (int64_t j = rr.lane; j < nc; j += 32) {
      const float c = ld_hint(row + j, pol);
#pragma unroll
      for (int r = 0; r < R; ++r) s[r] += c * sb[r * nc + j];
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      for (int o = 16; o > 0; o >>= 1) s[r] += __shfl_xor_sync(0xffffffffu, s[r], o);
      if (rr.lane == 0) L.x[i * R + r] = s[r];
    }
  }
}

template <class TV>
struct PcgParams {
  int64_t n, nslices;
  const int64_t* sp;
  const int32_t* col;
  const double* v64;   // scaled FP64 values (true residual)
  const float* a32;    // unscaled FP32 values (difference-form SpMV)
  const double* rsum;  // row sums of the unscaled matrix
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
  int bh_given;  // bh already holds the scaled, projected right-hand side (FP64)
  const AmgLevelDev* lv;
  int nlev;
  const float* cinv;
  int64_t nc, ldc;
  int reps;  // identical blocks: vectors hold reps x n entries, the matrix n rows
  int timing;  // phase timing marks on (spx_debug_pcg_timing)
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
// SpMV phases: the bounds of the warp's next slice are loaded while it works on this one
#define PCG_SLICES_BEGIN                                     \
  {                                                          \
    int64_t base, nbase_;                                    \
    int width, nwidth_;                                      \
    slice_bounds(P.sp, gw, P.nslices, base, width);          \
    for (int64_t sl = gw; sl < P.nslices; sl += nw) {        \
      slice_bounds(P.sp, sl + nw, P.nslices, nbase_, nwidth_); \
      const int64_t row = sl * 32 + lane;                    \
      if (row < n) {
#define PCG_SLICES_END \
  }                    \
  base = nbase_;       \
  width = nwidth_;     \
  }                    \
  }

// Phase timing of k_pcg_amg and k_pcg_amg_r (switched on by spx_debug_pcg_timing): CTA 0 adds the globaltimer interval
// since its previous mark to the slot of the phase that just ended (the phase's slowest CTA
// plus the barrier); read and cleared by pcg_phase_times.  Slots: V-cycle phases in order
// (3 per level down, the coarse solve, 3 per level up), 28 the PCG product, 29 the update,
// 30 the true residual.
__device__ unsigned long long g_pcg_phase_ns[32];
__device__ unsigned long long g_pcg_phase_n[32];
__device__ __forceinline__ void pcg_mark(unsigned long long& t_prev, int slot, int on) {
  if (on && blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t_prev != 0ull && slot >= 0 && slot < 32) {
      g_pcg_phase_ns[slot] += t - t_prev;
      g_pcg_phase_n[slot] += 1ull;
    }
    t_prev = t;
  }
}

// z^ = V(r^): lv[0].b / lv[0].db hold the unscaled residual D^1/2 r^ (FP32) on entry, lv[0].x
// holds u = D^-1/2 z^ on exit, and slot `slot` of the partials holds (r^, z^), (w, z^).  nlev >= 2.
template <class TV>
__device__ bool vcycle(const PcgParams<TV>& P, int slot, double* sh, unsigned long long& tm) {
  const unsigned nb = gridDim.x;
  unsigned int* cnt = P.bar;
  unsigned int* gen = P.bar + 1;
  const RowRange rr{static_cast<int64_t>((blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5),
                    static_cast<int64_t>((gridDim.x * static_cast<int64_t>(blockDim.x)) >> 5),
                    static_cast<int>(threadIdx.x & 31)};
  const int NL = P.nlev;
  int ph = 0;
  for (int l = 0; l + 1 < NL; ++l) {
    const AmgLevelDev& L = P.lv[l];
    pre_a(L, rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
    pre_b(L, rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
    restrict_to(L, P.lv[l + 1], rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
  }
  coarse_solve(P.lv[NL - 1], P.cinv, P.nc, P.ldc, rr);
  if (!grid_barrier(cnt, gen, nb, P.err)) return false;
  pcg_mark(tm, ph++, P.timing);
  for (int l = NL - 2; l >= 0; --l) {
    const AmgLevelDev& L = P.lv[l];
    prolong_from(L, P.lv[l + 1], rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
    post_c(L, rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
    double rz = 0.0, wz = 0.0;
    post_d(L, rr, P.r, P.sdinv, rz, wz, l == 0);
    if (l == 0) cta_partial(P.part, slot, rz, wz, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
  }
  return true;
}

template <class TV>
__global__ void __launch_bounds__(PCG_BLOCK, PCG_CTAS_PER_SM) k_pcg_amg(PcgParams<TV> P) {
  unsigned long long tm = 0ull;
  __shared__ double sh[160];
  const unsigned nb = gridDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  unsigned int* cnt = P.bar;
  unsigned int* gen = P.bar + 1;
  const int64_t n = P.n;
  float* b0 = P.lv[0].b;
  float* db0 = P.lv[0].db;
  const float* dinv0 = P.lv[0].dinv;
  double tot[4];
  double meanb = 0.0;
  if (P.project && !P.bh_given) {
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
      double bv;
      if (P.bh_given) {
        bv = P.bh[row] / P.sdinv[row];
      } else {
        bv = static_cast<double>(P.b[row]) - meanb;
        P.bh[row] = bv * P.sdinv[row];
      }
      if (!P.warm) P.y[row] = 0.0;
      bb += bv * bv;
    PCG_ROWS_END
    cta_partial(P.part, 1, bb, 0.0, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  cta_total(P.part, 1, tot, sh);
  const double bb = tot[0];
  if (P.warm && !(bb > 0.0)) {  // b = 0: the solution is 0
    PCG_ROWS_BEGIN P.y[row] = 0.0;
    PCG_ROWS_END
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  const double tol2 = fmax(P.rtol * P.rtol * bb, P.atol * P.atol);
  int total = 0, outers = 0;
  double rr = 0.0, rr0 = -1.0;
  for (int outer = 0; outer < P.max_outer; ++outer) {
    ++outers;
    // true residual r = bh - A^ y (FP64), its unscaled norm, r -> level-0 right-hand side
    {
      double rh = 0.0;
      PCG_ROWS_BEGIN
        double acc = 0.0, acc2 = 0.0;
        const uint64_t pst = l2_policy_stream(), pkeep = l2_policy_keep();
        int k = 0;
        for (; k + 2 <= width; k += 2) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          acc += ld_hint(P.v64 + idx, pst) * P.y[ld_hint(P.col + idx, pkeep)];
          acc2 += ld_hint(P.v64 + idx + 32, pst) * P.y[ld_hint(P.col + idx + 32, pkeep)];
        }
        if (k < width) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          acc += ld_hint(P.v64 + idx, pst) * P.y[ld_hint(P.col + idx, pkeep)];
        }
        const double r = P.bh[row] - (acc + acc2);
        P.r[row] = r;
        const float rf = static_cast<float>(r / P.sdinv[row]);
        b0[row] = rf;
        db0[row] = dinv0[row] * rf;
        rh += P.diag[row] * r * r;
      PCG_ROWS_END
      cta_partial(P.part, 0, rh, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      pcg_mark(tm, 30, P.timing);
    }
    cta_total(P.part, 0, tot, sh);
    rr = tot[0];
    if (rr0 < 0.0) rr0 = rr;
    if (rr <= tol2 || total >= P.maxit) break;
    double rz_old = 1.0;
    for (int it = 0;; ++it) {
      if (!vcycle(P, 2, sh, tm)) return;
      cta_total(P.part, 2, tot, sh);
      const double rz = tot[0];
      const double c = P.project && P.ww > 0.0 ? tot[1] / P.ww : 0.0;
      const double beta = it == 0 ? 0.0 : rz / rz_old;
      const float* u0 = P.lv[0].x;  // u = D^-1/2 z^ from the unscaled level-0 cycle
      double pq = 0.0;
      PCG_SLICES_BEGIN
        const double ui = static_cast<double>(u0[row]);
        const uint64_t pkeep = l2_policy_keep();
        double acc = 0.0, acc2 = 0.0;
        int k = 0;
        for (; k + 4 <= width; k += 4) {
          const int64_t i0 = base + ((int64_t)k << 5) + lane;
          const float w0 = ld_hint(P.a32 + i0, pkeep), w1 = ld_hint(P.a32 + i0 + 32, pkeep),
                      w2 = ld_hint(P.a32 + i0 + 64, pkeep), w3 = ld_hint(P.a32 + i0 + 96, pkeep);
          const int32_t c0 = ld_hint(P.col + i0, pkeep), c1 = ld_hint(P.col + i0 + 32, pkeep),
                        c2 = ld_hint(P.col + i0 + 64, pkeep), c3 = ld_hint(P.col + i0 + 96, pkeep);
          acc += static_cast<double>(w0) * (static_cast<double>(u0[c0]) - ui);
          acc2 += static_cast<double>(w1) * (static_cast<double>(u0[c1]) - ui);
          acc += static_cast<double>(w2) * (static_cast<double>(u0[c2]) - ui);
          acc2 += static_cast<double>(w3) * (static_cast<double>(u0[c3]) - ui);
        }
        if (k < width) {  // up to three remaining columns, loaded together, summed in order
          float wt[3];
          int32_t ct[3];
#pragma unroll
          for (int u = 0; u < 3; ++u) {
            const int64_t idx = base + ((int64_t)(k + u) << 5) + lane;
            const bool in = k + u < width;
            wt[u] = in ? ld_hint(P.a32 + idx, pkeep) : 0.0f;
            ct[u] = in ? ld_hint(P.col + idx, pkeep) : 0;
          }
#pragma unroll
          for (int u = 0; u < 3; ++u)
            if (k + u < width) acc += static_cast<double>(wt[u]) * (static_cast<double>(u0[ct[u]]) - ui);
        }
        const double rsi = P.rsum[row], sdi = P.sdinv[row];
        const double pold = it == 0 ? 0.0 : P.p[row], qold = it == 0 ? 0.0 : P.q[row];
        acc = (acc + acc2 + rsi * ui) * sdi;
        const double z = ui / sdi;
        const double w = 1.0 / sdi;
        const double pv = (z - c * w) + (it == 0 ? 0.0 : beta * pold);
        const double qv = acc + (it == 0 ? 0.0 : beta * qold);
        P.p[row] = pv;
        P.q[row] = qv;
        pq += pv * qv;
      PCG_SLICES_END
      cta_partial(P.part, 3, pq, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      pcg_mark(tm, 28, P.timing);
      cta_total(P.part, 3, tot, sh);
      const double pqt = tot[0];
      if (!(pqt > 0.0) || !(rz > 0.0)) break;
      const double alpha = rz / pqt;
      double rh = 0.0;
      PCG_ROWS_BEGIN
        P.y[row] += alpha * P.p[row];
        const double r = P.r[row] - alpha * P.q[row];
        P.r[row] = r;
        const float rf = static_cast<float>(r / P.sdinv[row]);
        b0[row] = rf;
        db0[row] = dinv0[row] * rf;
        rh += P.diag[row] * r * r;
      PCG_ROWS_END
      cta_partial(P.part, 0, rh, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      pcg_mark(tm, 29, P.timing);
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

// the V-cycle of k_pcg_amg for R identical blocks (same phases and barriers)
template <class TV, int R>
__device__ bool vcycle_r(const PcgParams<TV>& P, int slot, double* sh, unsigned long long& tm) {
  const unsigned nb = gridDim.x;
  unsigned int* cnt = P.bar;
  unsigned int* gen = P.bar + 1;
  const RowRange rr{static_cast<int64_t>((blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5),
                    static_cast<int64_t>((gridDim.x * static_cast<int64_t>(blockDim.x)) >> 5),
                    static_cast<int>(threadIdx.x & 31)};
  const int NL = P.nlev;
  int ph = 0;
  for (int l = 0; l + 1 < NL; ++l) {
    const AmgLevelDev& L = P.lv[l];
    pre_a_r<R>(L, rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
    pre_b_r<R>(L, rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
    restrict_to_r<R>(L, P.lv[l + 1], rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
  }
  coarse_solve_r<R>(P.lv[NL - 1], P.cinv, P.nc, P.ldc, rr);
  if (!grid_barrier(cnt, gen, nb, P.err)) return false;
  pcg_mark(tm, ph++, P.timing);
  for (int l = NL - 2; l >= 0; --l) {
    const AmgLevelDev& L = P.lv[l];
    prolong_from_r<R>(L, P.lv[l + 1], rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
    post_c_r<R>(L, rr);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
    double rz = 0.0, wz = 0.0;
    post_d_r<R>(L, rr, P.r, P.sdinv, rz, wz, l == 0);
    if (l == 0) cta_partial(P.part, slot, rz, wz, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return false;
    pcg_mark(tm, ph++, P.timing);
  }
  return true;
}

// k_pcg_amg on R identical blocks: one CG on the block-diagonal system (the scalars are those of
// the whole system, as for a disjoint union), with the block's matrix and hierarchy stored once.
// Per-row data (rsum, sdinv, diag, level dinv) are those of block row i (identical blocks); b, x,
// y, bh are indexed in block order (r n + i), the work vectors r, p, q and the level vectors
// interleaved (i R + r).
template <class TV, int R>
__global__ void __launch_bounds__(PCG_BLOCK_R, PCG_CTAS_PER_SM) k_pcg_amg_r(PcgParams<TV> P) {
  unsigned long long tm = 0ull;
  __shared__ double sh[160];
  const unsigned nb = gridDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  unsigned int* cnt = P.bar;
  unsigned int* gen = P.bar + 1;
  const int64_t n = P.n;
  float* b0 = P.lv[0].b;
  float* db0 = P.lv[0].db;
  const float* dinv0 = P.lv[0].dinv;
  double tot[4];
  double meanb = 0.0;
  if (P.project && !P.bh_given) {
    double part = 0.0;
    PCG_ROWS_BEGIN
#pragma unroll
      for (int r = 0; r < R; ++r) part += static_cast<double>(P.b[r * n + row]);
    PCG_ROWS_END
    cta_partial(P.part, 0, part, 0.0, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
    cta_total(P.part, 0, tot, sh);
    meanb = tot[0] / static_cast<double>(R * n);
  }
  {
    double bb = 0.0;
    PCG_ROWS_BEGIN
      const double sd = P.sdinv[row];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int64_t j = r * n + row;
        double bv;
        if (P.bh_given) {
          bv = P.bh[j] / sd;
        } else {
          bv = static_cast<double>(P.b[j]) - meanb;
          P.bh[j] = bv * sd;
        }
        if (!P.warm) P.y[j] = 0.0;
        bb += bv * bv;
      }
    PCG_ROWS_END
    cta_partial(P.part, 1, bb, 0.0, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  cta_total(P.part, 1, tot, sh);
  const double bb = tot[0];
  if (P.warm && !(bb > 0.0)) {  // b = 0: the solution is 0
    PCG_ROWS_BEGIN
#pragma unroll
      for (int r = 0; r < R; ++r) P.y[r * n + row] = 0.0;
    PCG_ROWS_END
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  const double tol2 = fmax(P.rtol * P.rtol * bb, P.atol * P.atol);
  int total = 0, outers = 0;
  double rr = 0.0, rr0 = -1.0;
  for (int outer = 0; outer < P.max_outer; ++outer) {
    ++outers;
    // true residual r = bh - A^ y (FP64) of every block, its unscaled norm, r -> level-0 rhs
    {
      double rh = 0.0;
      const uint64_t pst = l2_policy_stream(), pkeep = l2_policy_keep();
      PCG_SLICES_BEGIN
        double acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0.0;
        int k = 0;
        for (; k + 2 <= width; k += 2) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          const double v0 = ld_hint(P.v64 + idx, pst), v1 = ld_hint(P.v64 + idx + 32, pst);
          const int32_t c0 = ld_hint(P.col + idx, pkeep), c1 = ld_hint(P.col + idx + 32, pkeep);
#pragma unroll
          for (int r = 0; r < R; ++r) acc[r] += v0 * P.y[r * n + c0] + v1 * P.y[r * n + c1];
        }
        if (k < width) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          const double v = ld_hint(P.v64 + idx, pst);
          const int32_t c = ld_hint(P.col + idx, pkeep);
#pragma unroll
          for (int r = 0; r < R; ++r) acc[r] += v * P.y[r * n + c];
        }
        const float di0 = dinv0[row];
        const double sd = P.sdinv[row], dg = P.diag[row];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const double rv = P.bh[r * n + row] - acc[r];
          const int64_t j = row * R + r;
          P.r[j] = rv;
          const float rf = static_cast<float>(rv / sd);
          b0[j] = rf;
          db0[j] = di0 * rf;
          rh += dg * rv * rv;
        }
      PCG_SLICES_END
      cta_partial(P.part, 0, rh, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      pcg_mark(tm, 30, P.timing);
    }
    cta_total(P.part, 0, tot, sh);
    rr = tot[0];
    if (rr0 < 0.0) rr0 = rr;
    if (rr <= tol2 || total >= P.maxit) break;
    double rz_old = 1.0;
    for (int it = 0;; ++it) {
      if (!vcycle_r<TV, R>(P, 2, sh, tm)) return;
      cta_total(P.part, 2, tot, sh);
      const double rz = tot[0];
      const double c = P.project && P.ww > 0.0 ? tot[1] / P.ww : 0.0;
      const double beta = it == 0 ? 0.0 : rz / rz_old;
      const float* u0 = P.lv[0].x;  // u = D^-1/2 z^ of every block (interleaved)
      double pq = 0.0;
      const uint64_t pkeep = l2_policy_keep();
      PCG_SLICES_BEGIN
        float uf[R];
        load_r<R>(u0, row, uf);
        const double rs = P.rsum[row];
        const double sd = P.sdinv[row];
        double ui[R], acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          ui[r] = static_cast<double>(uf[r]);
          acc[r] = 0.0;
        }
        for (int k = 0; k < width; k += 4) {  // rounds of four columns, the last predicated
          const int64_t i0 = base + ((int64_t)k << 5) + lane;
          float w[4];
          int32_t cc[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const bool in = k + u < width;
            w[u] = in ? ld_hint(P.a32 + i0 + 32 * u, pkeep) : 0.0f;
            cc[u] = in ? ld_hint(P.col + i0 + 32 * u, pkeep) : 0;
          }
          float g[4][R];
#pragma unroll
          for (int u = 0; u < 4; ++u) load_r<R>(u0, cc[u], g[u]);
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (k + u < width) {
#pragma unroll
              for (int r = 0; r < R; ++r)
                acc[r] += static_cast<double>(w[u]) * (static_cast<double>(g[u][r]) - ui[r]);
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int64_t j = row * R + r;
          const double av = (acc[r] + rs * ui[r]) * sd;
          const double z = ui[r] / sd;
          const double w = 1.0 / sd;
          const double pv = (z - c * w) + (it == 0 ? 0.0 : beta * P.p[j]);
          const double qv = av + (it == 0 ? 0.0 : beta * P.q[j]);
          P.p[j] = pv;
          P.q[j] = qv;
          pq += pv * qv;
        }
      PCG_SLICES_END
      cta_partial(P.part, 3, pq, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      pcg_mark(tm, 28, P.timing);
      cta_total(P.part, 3, tot, sh);
      const double pqt = tot[0];
      if (!(pqt > 0.0) || !(rz > 0.0)) break;
      const double alpha = rz / pqt;
      double rh = 0.0;
      PCG_ROWS_BEGIN
        const float di0 = dinv0[row];
        const double sd = P.sdinv[row], dg = P.diag[row];
        double pv[R], rv[R], qv[R];
        load_r64<R>(P.p, row, pv);
        load_r64<R>(P.r, row, rv);
        load_r64<R>(P.q, row, qv);
        float bf[R], dbf[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          P.y[r * n + row] += alpha * pv[r];
          rv[r] -= alpha * qv[r];
          const float rf = static_cast<float>(rv[r] / sd);
          bf[r] = rf;
          dbf[r] = di0 * rf;
          rh += dg * rv[r] * rv[r];
        }
        store_r64<R>(P.r, row, rv);
        store_r<R>(b0, row, bf);
        store_r<R>(db0, row, dbf);
      PCG_ROWS_END
      cta_partial(P.part, 0, rh, 0.0, 0.0, 0.0, sh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      pcg_mark(tm, 29, P.timing);
      cta_total(P.part, 0, tot, sh);
      rr = tot[0];
      ++total;
      rz_old = rz;
      if (rr <= 0.25 * tol2 || total >= P.maxit) break;
    }
  }
  double mx = 0.0;
  if (P.project) {
    double sx = 0.0;
    PCG_ROWS_BEGIN
      const double sd = P.sdinv[row];
#pragma unroll
      for (int r = 0; r < R; ++r) sx += P.y[r * n + row] * sd;
    PCG_ROWS_END
    cta_partial(P.part, 1, sx, 0.0, 0.0, 0.0, sh);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
    cta_total(P.part, 1, tot, sh);
    mx = tot[0] / static_cast<double>(R * n);
  }
  PCG_ROWS_BEGIN
    const double sd = P.sdinv[row];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t j = r * n + row;
      const double xv = P.y[j] * sd - mx;
      P.x[j] = static_cast<TV>(xv);
      P.y[j] = xv / sd;
    }
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
void CgSystem<TM>::enable_amg(const HostSell& hs, const std::vector<int64_t>& rowptr, const std::vector<int32_t>& col,
                              const std::vector<double>& a, const std::vector<double>& d, bool singular,
                              cudaStream_t s) {
  const int64_t n = n1;  // the stored block (reps copies of it form the system)
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
  ww *= reps;  // the null vector of the whole system repeats w in every block
  AmgHost h;
  amg_build(Ah, w, singular, AmgOptions{}, h);
  if (h.lv.size() < 2) {  // no coarsening possible: keep the Jacobi solver
    amg.reset();
    return;
  }
  // unscaled FP32 values on the SELL pattern and FP64 row sums (difference-form SpMV); the
  // finest level of the cycle uses the same values
  {
    std::vector<float> v(P.len, 0.0f);
    std::vector<double> rs(n, 0.0);
    for (int64_t i = 0; i < n; ++i)
      for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
        rs[i] += a[k];
        if (hs.map[k] >= 0) v[hs.map[k]] = static_cast<float>(a[k]);
      }
    amg_a32.upload(v, s);
    amg_rsum.upload(rs, s);
  }
  // level 0 in the unscaled space: D^-1 of A, P_0 = D^-1/2 P^_0, R_0 = P^_0^T D^-1/2
  {
    AmgHostLevel& L0 = h.lv[0];
    for (int64_t i = 0; i < n; ++i) L0.dinv[i] = 1.0 / d[i];
    for (int64_t i = 0; i < n; ++i)
      for (int64_t k = L0.P.rp[i]; k < L0.P.rp[i + 1]; ++k) L0.P.v[k] /= std::sqrt(d[i]);
    for (int64_t k = 0; k < static_cast<int64_t>(L0.R.v.size()); ++k) L0.R.v[k] /= std::sqrt(d[L0.R.ci[k]]);
  }
  amg = std::make_unique<AmgDevice>();
  amg->upload(h, s, P.slice_ptr.p, P.col.p, amg_a32.p, P.nslices, reps);
  amg_ww = ww;
  amg_singular = singular;
  if (!y64.n) {
    y64.alloc(this->n);
    y64.zero(s);
  }
  if (!bh64.n) bh64.alloc(this->n);
  amg_work.alloc(3 * static_cast<size_t>(this->n));
  amg_work.zero(s);
  if (!vals64.n) {  // FP64 scaled values (the FP64 CG keeps them in vals)
    std::vector<double> v(P.len);
    SPX_CUDA(cudaMemcpy(v.data(), vals.p, P.len * sizeof(double), cudaMemcpyDeviceToHost));
    vals64.upload(v, s);
  }
  SPX_CHECK(reps == 1 || reps == 2 || reps == 4 || reps == 8, "repeated blocks: 1, 2, 4 or 8");
  int per_sm = 0;
  SPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_amg<double>, PCG_BLOCK, 0));
  SPX_CHECK(per_sm >= PCG_CTAS_PER_SM, "AMG PCG kernel cannot be resident");
  if (reps > 1) {
    const void* kr = reps == 2 ? reinterpret_cast<const void*>(k_pcg_amg_r<double, 2>)
                     : reps == 4 ? reinterpret_cast<const void*>(k_pcg_amg_r<double, 4>)
                                 : reinterpret_cast<const void*>(k_pcg_amg_r<double, 8>);
    // the coarse phase stages the R right-hand sides in dynamic shared memory
    const size_t dyn = static_cast<size_t>(amg->nc) * reps * sizeof(float);
    SPX_CHECK(dyn <= 200 * 1024, "AMG coarsest level too large for the repeated-block kernel");
    const void* kall[] = {reinterpret_cast<const void*>(k_pcg_amg_r<double, 2>),
                          reinterpret_cast<const void*>(k_pcg_amg_r<double, 4>),
                          reinterpret_cast<const void*>(k_pcg_amg_r<double, 8>),
                          reinterpret_cast<const void*>(k_pcg_amg_r<float, 2>),
                          reinterpret_cast<const void*>(k_pcg_amg_r<float, 4>),
                          reinterpret_cast<const void*>(k_pcg_amg_r<float, 8>)};
    for (const void* kk : kall)
      SPX_CUDA(cudaFuncSetAttribute(kk, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn)));
    SPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kr, PCG_BLOCK_R, dyn));
    SPX_CHECK(per_sm >= PCG_CTAS_PER_SM, "AMG PCG kernel (repeated blocks) cannot be resident");
  }
  int dev;
  SPX_CUDA(cudaGetDevice(&dev));
  amg_grid = num_sms(dev) * PCG_CTAS_PER_SM;
  {
    int64_t keep = P.len * static_cast<int64_t>(sizeof(float) + sizeof(int32_t));  // level 0 (shared pattern)
    for (int l = 1; l + 1 < amg->nlev; ++l) keep += amg->A[l].len * static_cast<int64_t>(sizeof(float) + sizeof(int32_t));
    keep += amg->cinv.bytes();  // the dense coarsest inverse
    reserve_persisting_l2(keep + keep / 8, dev);
  }
  if (part.n < 4 * 4 * static_cast<size_t>(amg_grid)) part.alloc(4 * 4 * static_cast<size_t>(amg_grid));
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class TM>
template <class TV>
void CgSystem<TM>::launch_amg(const TV* b, TV* x, double rtol, double atol, int maxit, bool warm, bool project,
                              cudaStream_t st, bool bh_given) {
  PcgParams<TV> q;
  q.n = n1; q.nslices = P.nslices; q.sp = P.slice_ptr.p; q.col = P.col.p; q.reps = reps;
  q.v64 = vals64.p; q.a32 = amg_a32.p; q.rsum = amg_rsum.p; q.sdinv = sdinv64.p; q.diag = diag64.p;
  q.b = b; q.x = x;
  q.bh = bh64.p; q.y = y64.p;
  q.r = amg_work.p; q.p = amg_work.p + n; q.q = amg_work.p + 2 * n;
  q.part = part.p; q.bar = bar.p; q.err = err.p; q.iters = iters.p; q.resid = resid.p;
  q.iters_acc = iters_acc.p; q.res_acc = res_acc.p;
  q.rtol = rtol; q.atol = atol; q.ww = amg_singular ? amg_ww : 0.0;
  q.maxit = maxit; q.max_outer = max_outer; q.warm = warm ? 1 : 0; q.project = project ? 1 : 0;
  q.bh_given = bh_given ? 1 : 0;
  q.lv = amg->lv.p; q.nlev = amg->nlev; q.cinv = amg->cinv.p; q.nc = amg->nc; q.ldc = amg->ldc;
  q.timing = g_pcg_timing.load(std::memory_order_relaxed);
  void* args[] = {&q};
  void* k = reinterpret_cast<void*>(k_pcg_amg<TV>);
  if (reps == 2) k = reinterpret_cast<void*>(k_pcg_amg_r<TV, 2>);
  if (reps == 4) k = reinterpret_cast<void*>(k_pcg_amg_r<TV, 4>);
  if (reps == 8) k = reinterpret_cast<void*>(k_pcg_amg_r<TV, 8>);
  const size_t dyn = reps > 1 ? static_cast<size_t>(amg->nc) * reps * sizeof(float) : 0;
  SPX_CUDA(cudaLaunchCooperativeKernel(k, dim3(amg_grid), dim3(reps > 1 ? PCG_BLOCK_R : PCG_BLOCK), args, dyn, st));
}

// per-slot sums (ns) and counts of the phase timing marks since the last call
void pcg_phase_times(double* ns32, int64_t* n32) {
  unsigned long long a[32], b[32], z[32] = {};
  SPX_CUDA(cudaDeviceSynchronize());
  SPX_CUDA(cudaMemcpyFromSymbol(a, g_pcg_phase_ns, sizeof(a)));
  SPX_CUDA(cudaMemcpyFromSymbol(b, g_pcg_phase_n, sizeof(b)));
  SPX_CUDA(cudaMemcpyToSymbol(g_pcg_phase_ns, z, sizeof(z)));
  SPX_CUDA(cudaMemcpyToSymbol(g_pcg_phase_n, z, sizeof(z)));
  for (int i = 0; i < 32; ++i) {
    ns32[i] = static_cast<double>(a[i]);
    n32[i] = static_cast<int64_t>(b[i]);
  }
}

template void CgSystem<double>::enable_amg(const HostSell&, const std::vector<int64_t>&, const std::vector<int32_t>&,
                                           const std::vector<double>&, const std::vector<double>&, bool,
                                           cudaStream_t);
template void CgSystem<float>::enable_amg(const HostSell&, const std::vector<int64_t>&, const std::vector<int32_t>&,
                                          const std::vector<double>&, const std::vector<double>&, bool,
                                          cudaStream_t);
template void CgSystem<double>::launch_amg<double>(const double*, double*, double, double, int, bool, bool,
                                                   cudaStream_t, bool);
template void CgSystem<float>::launch_amg<double>(const double*, double*, double, double, int, bool, bool,
                                                  cudaStream_t, bool);
template void CgSystem<float>::launch_amg<float>(const float*, float*, double, double, int, bool, bool,
                                                 cudaStream_t, bool);

}  // namespace spx
