// H-matrix apply: y = P^-1 [diag o x~ + Near x~ + sum_b U_b (V_b x~_{J_b})],  x~ = x[perm]
// (HMatrixGPUPackedFused.matvec, lindholm_hmatrix_gpu/backend_fused.py:496-512).
//
// B200 layout.  Far factors are packed per block as U^T (k x m, each column of U
// contiguous) followed by V (k x n, each row of V contiguous) in the storage type TF
// (FP64, FP32 or BF16).  Near blocks are dense tiles stored column-major (n x m) in
// TN.  Three kernels, no atomics, every output row written by exactly one CTA:
//   k_hgather : x~[i] = src[g(perm[i])]             (fused boundary gather + perm)
//   k_far_z   : z_b = V_b x~_{J_b}, one CTA per far block, lanes over columns
//   k_rows    : one CTA per leaf row cluster; threads over the cluster's rows walk
//               the cluster's item list (near tiles and far blocks covering it),
//               read U^T / tile columns coalesced across rows, add diag o x~, and
//               scatter y to dst[g(perm[i])].
// Near tiles may use compensated (Kahan) accumulation in the mixed-precision form.
#include <algorithm>
#include <mutex>
#include <string>

#include "hmat.cuh"

namespace spx {

template <class T> __device__ __forceinline__ T from_d(double v) { return static_cast<T>(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_d<__nv_bfloat16>(double v) {
  return __float2bfloat16_rn(static_cast<float>(v));
}
template <class T> __device__ __forceinline__ double to_d(T v) { return static_cast<double>(v); }
template <> __device__ __forceinline__ double to_d<__nv_bfloat16>(__nv_bfloat16 v) {
  return static_cast<double>(__bfloat162float(v));
}
template <class A, class T> __device__ __forceinline__ A cvt(T v) { return static_cast<A>(v); }
template <> __device__ __forceinline__ float cvt<float, __nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ double cvt<double, __nv_bfloat16>(__nv_bfloat16 v) {
  return static_cast<double>(__bfloat162float(v));
}

// ------------------------------------------------------------------ packing
struct PackFar {
  int64_t src_u, src_v, dst_u, dst_v;  // element offsets
  int32_t m, n, k, ldv;
};
// U^T (k x m) as is; V (k x n) into rows of ldv elements (ldv = n rounded up to 8), zero padded
template <class TF>
__global__ void k_pack_far(const PackFar* __restrict__ jobs, const double* __restrict__ pool, TF* __restrict__ out) {
  const PackFar j = jobs[blockIdx.x];
  const int64_t lu = (int64_t)j.k * j.m, lv = (int64_t)j.k * j.ldv;
  for (int64_t e = threadIdx.x; e < lu; e += blockDim.x) out[j.dst_u + e] = from_d<TF>(pool[j.src_u + e]);
  for (int64_t e = threadIdx.x; e < lv; e += blockDim.x) {
    const int64_t q = e / j.ldv, c = e - q * j.ldv;
    out[j.dst_v + e] = (c < j.n) ? from_d<TF>(pool[j.src_v + q * j.n + c]) : from_d<TF>(0.0);
  }
}
struct PackNear {
  int64_t src, dst;
  int32_t m, n;
};
template <class TN>
__global__ void k_pack_near(const PackNear* __restrict__ jobs, const double* __restrict__ pool, TN* __restrict__ out) {
  const PackNear j = jobs[blockIdx.x];
  const int64_t L = (int64_t)j.m * j.n;
  // out[c * m + r] = in[r * n + c]
  for (int64_t e = threadIdx.x; e < L; e += blockDim.x) {
    const int64_t c = e / j.m, r = e - c * j.m;
    out[j.dst + e] = from_d<TN>(pool[j.src + r * j.n + c]);
  }
}

// ------------------------------------------------------------------ apply kernels
template <class TS, class TX>
__global__ void k_hgather(int64_t Nb, const TS* __restrict__ src, const int32_t* __restrict__ gidx,
                          const int32_t* __restrict__ perm, TX* __restrict__ xp) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= Nb) return;
  const int32_t b = perm[i];
  const int64_t o = gidx ? gidx[b] : b;
  xp[i] = static_cast<TX>(src[o]);
}

// 16-byte vector loads of far factors
template <class TF> struct V16;
template <> struct V16<double> { using T = double2; static constexpr int E = 2; };
template <> struct V16<float> { using T = float4; static constexpr int E = 4; };
template <> struct V16<__nv_bfloat16> { using T = uint4; static constexpr int E = 8; };

template <class TA, class TF>
__device__ __forceinline__ void v16_elems(const typename V16<TF>::T& v, TA out[V16<TF>::E]);
template <>
__device__ __forceinline__ void v16_elems<double, double>(const double2& v, double out[2]) { out[0] = v.x; out[1] = v.y; }
template <>
__device__ __forceinline__ void v16_elems<float, double>(const double2& v, float out[2]) {
  out[0] = static_cast<float>(v.x); out[1] = static_cast<float>(v.y);
}
template <>
__device__ __forceinline__ void v16_elems<double, float>(const float4& v, double out[4]) {
  out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
}
template <>
__device__ __forceinline__ void v16_elems<float, float>(const float4& v, float out[4]) {
  out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
}
template <class TA>
__device__ __forceinline__ void bf16x8(const uint4& v, TA out[8]) {
  const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    out[2 * q] = static_cast<TA>(__uint_as_float(w[q] << 16));
    out[2 * q + 1] = static_cast<TA>(__uint_as_float(w[q] & 0xffff0000u));
  }
}
template <>
__device__ __forceinline__ void v16_elems<double, __nv_bfloat16>(const uint4& v, double out[8]) { bf16x8<double>(v, out); }
template <>
__device__ __forceinline__ void v16_elems<float, __nv_bfloat16>(const uint4& v, float out[8]) { bf16x8<float>(v, out); }

// z_b = V_b x~_{J_b}: one CTA per far block; V rows (ldv elements, zero padded, 16-byte aligned)
// are read as 16-byte vectors by groups of G lanes (G = chunks per row rounded to a power of
// two, at most 32), groups reduce with shuffles.
template <class TF, class TA, class TX>
__global__ void __launch_bounds__(128) k_far_z(const int32_t* __restrict__ meta, const int64_t* __restrict__ voff,
                                               const int64_t* __restrict__ zoff, const TF* __restrict__ F,
                                               const TX* __restrict__ xp, TA* __restrict__ z) {
  constexpr int E = V16<TF>::E;
  using VT = typename V16<TF>::T;
  const int b = blockIdx.x;
  const int cs = meta[6 * b + 2], n = meta[6 * b + 3], k = meta[6 * b + 4], ldv = meta[6 * b + 5];
  const VT* V = reinterpret_cast<const VT*>(F + voff[b]);
  const TX* x = xp + cs;
  const int nch = ldv / E;
  int G = 1;
  while (G < nch && G < 32) G <<= 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int gpw = 32 / G;                // groups per warp
  const int gl = lane % G, gw = lane / G;
  for (int qb = warp * gpw; qb < k; qb += nwarps * gpw) {
    const int q = qb + gw;
    TA acc = 0;
    if (q < k) {
      const VT* row = V + (int64_t)q * nch;
      for (int c = gl; c < nch; c += G) {
        const VT v = row[c];
        TA e[E];
        v16_elems<TA, TF>(v, e);
        const int j0 = c * E;
#pragma unroll
        for (int t = 0; t < E; ++t)
          if (j0 + t < n) acc += e[t] * static_cast<TA>(x[j0 + t]);
      }
    }
    for (int o = G >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (q < k && gl == 0) z[zoff[b] + q] = acc;
  }
}

constexpr int ROWS_GROUPS = 4;
constexpr int ROWS_GSIZE = 64;

template <class TF, class TN, class TA, class TX, class TD>
__global__ void __launch_bounds__(ROWS_GROUPS * ROWS_GSIZE) k_rows(
    const int32_t* __restrict__ leaf_start, const int64_t* __restrict__ item_ptr,
    const int32_t* __restrict__ items, const int32_t* __restrict__ far_meta,
    const int64_t* __restrict__ far_uoff, const int64_t* __restrict__ far_zoff,
    const TF* __restrict__ F, const int32_t* __restrict__ near_meta, const int64_t* __restrict__ near_off,
    const TN* __restrict__ Nt, const TA* __restrict__ z, const TX* __restrict__ xp,
    const double* __restrict__ diag, const int32_t* __restrict__ perm, const int32_t* __restrict__ gidx,
    TD* __restrict__ dst, const TD* __restrict__ add, TD* __restrict__ yb, int kahan) {
  extern __shared__ unsigned char smem_raw[];
  const int leaf = blockIdx.x;
  const int r0 = leaf_start[leaf], nr = leaf_start[leaf + 1] - r0;
  TA* acc = reinterpret_cast<TA*>(smem_raw);             // [GROUPS][nr]
  TA* cmp = acc + ROWS_GROUPS * nr;                       // [GROUPS][nr] Kahan compensation
  const int g = threadIdx.x / ROWS_GSIZE, t = threadIdx.x % ROWS_GSIZE;
  for (int r = t; r < nr; r += ROWS_GSIZE) {
    acc[g * nr + r] = 0;
    cmp[g * nr + r] = 0;
  }
  const int64_t i0 = item_ptr[leaf], i1 = item_ptr[leaf + 1];
  for (int64_t it = i0 + g; it < i1; it += ROWS_GROUPS) {
    const int32_t code = items[it];
    const int32_t bi = code >> 1;
    if (code & 1) {
      const int rs = far_meta[6 * bi], m = far_meta[6 * bi + 1], k = far_meta[6 * bi + 4];
      const TF* Ut = F + far_uoff[bi];
      const TA* zb = z + far_zoff[bi];
      for (int r = t; r < nr; r += ROWS_GSIZE) {
        const TF* u = Ut + (r0 + r - rs);
        TA s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        int q = 0;
        for (; q + 4 <= k; q += 4) {
          s0 += cvt<TA>(u[(int64_t)q * m]) * zb[q];
          s1 += cvt<TA>(u[(int64_t)(q + 1) * m]) * zb[q + 1];
          s2 += cvt<TA>(u[(int64_t)(q + 2) * m]) * zb[q + 2];
          s3 += cvt<TA>(u[(int64_t)(q + 3) * m]) * zb[q + 3];
        }
        for (; q < k; ++q) s0 += cvt<TA>(u[(int64_t)q * m]) * zb[q];
        acc[g * nr + r] += (s0 + s1) + (s2 + s3);
      }
    } else {
      const int rs = near_meta[4 * bi], m = near_meta[4 * bi + 1], cs = near_meta[4 * bi + 2],
                n = near_meta[4 * bi + 3];
      const TN* tile = Nt + near_off[bi];
      const TX* x = xp + cs;
      for (int r = t; r < nr; r += ROWS_GSIZE) {
        const TN* u = tile + (r0 + r - rs);
        TA s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        int c = 0;
        for (; c + 4 <= n; c += 4) {
          s0 += cvt<TA>(u[(int64_t)c * m]) * static_cast<TA>(x[c]);
          s1 += cvt<TA>(u[(int64_t)(c + 1) * m]) * static_cast<TA>(x[c + 1]);
          s2 += cvt<TA>(u[(int64_t)(c + 2) * m]) * static_cast<TA>(x[c + 2]);
          s3 += cvt<TA>(u[(int64_t)(c + 3) * m]) * static_cast<TA>(x[c + 3]);
        }
        for (; c < n; ++c) s0 += cvt<TA>(u[(int64_t)c * m]) * static_cast<TA>(x[c]);
        const TA s = (s0 + s1) + (s2 + s3);
        if (kahan) {
          const TA y = s - cmp[g * nr + r];
          const TA tt = acc[g * nr + r] + y;
          cmp[g * nr + r] = (tt - acc[g * nr + r]) - y;
          acc[g * nr + r] = tt;
        } else {
          acc[g * nr + r] += s;
        }
      }
    }
  }
  __syncthreads();
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    const int64_t i = r0 + r;
    TA y = static_cast<TA>(diag[i]) * static_cast<TA>(xp[i]);
    for (int q = 0; q < ROWS_GROUPS; ++q) y += acc[q * nr + r] - cmp[q * nr + r];
    const int32_t b = perm[i];
    const int64_t o = gidx ? gidx[b] : b;
    const TD yv = static_cast<TD>(y);
    dst[o] = add ? static_cast<TD>(add[o] + yv) : yv;
    if (yb) yb[b] = yv;
  }
}

// ------------------------------------------------------------------ host side
namespace {
template <class TF, class TN>
void do_pack(HMatrix& H, cudaStream_t s) {
  std::vector<PackFar> pf;
  std::vector<PackNear> pn;
  std::vector<int32_t> fmeta, nmeta;
  std::vector<int64_t> fu, fv, fz, noff;
  std::vector<int32_t> code_of(H.blocks.size());
  int64_t fpos = 0, npos = 0, zpos = 0;
  int32_t nf = 0, nn = 0;
  for (size_t q = 0; q < H.blocks.size(); ++q) {
    const HBlock& b = H.blocks[q];
    const int32_t m = b.re - b.rs, n = b.ce - b.cs;
    if (b.type == 1) {
      const int32_t ldv = (n + 7) / 8 * 8;
      const int64_t pu = fpos;
      const int64_t pv = (pu + (int64_t)b.rank * m + 7) / 8 * 8;  // 16-byte aligned V rows
      pf.push_back(PackFar{b.off_u, b.off_v, pu, pv, m, n, b.rank, ldv});
      fmeta.insert(fmeta.end(), {b.rs, m, b.cs, n, b.rank, ldv});
      fu.push_back(pu);
      fv.push_back(pv);
      fz.push_back(zpos);
      fpos = pv + (int64_t)b.rank * ldv;
      zpos += b.rank;
      code_of[q] = (nf++ << 1) | 1;
    } else {
      pn.push_back(PackNear{b.off_u, npos, m, n});
      nmeta.insert(nmeta.end(), {b.rs, m, b.cs, n});
      noff.push_back(npos);
      npos += (int64_t)m * n;
      code_of[q] = (nn++ << 1);
    }
  }
  H.n_far = nf;
  H.n_near = nn;
  H.zlen = zpos;
  H.far_f.alloc(std::max<int64_t>(fpos, 1) * sizeof(TF));
  H.near_f.alloc(std::max<int64_t>(npos, 1) * sizeof(TN));
  H.bytes_far = fpos * (int64_t)sizeof(TF);
  H.bytes_near = npos * (int64_t)sizeof(TN);
  for (size_t k0 = 0; k0 < pf.size(); k0 += 65535) {
    const size_t c = std::min<size_t>(65535, pf.size() - k0);
    DevBuf<PackFar> d;
    d.upload(pf.data() + k0, c, s);
    k_pack_far<TF><<<static_cast<unsigned>(c), 256, 0, s>>>(d.p, H.far_pool64.p, reinterpret_cast<TF*>(H.far_f.p));
    SPX_LAUNCH_CHECK();
    SPX_CUDA(cudaStreamSynchronize(s));
  }
  for (size_t k0 = 0; k0 < pn.size(); k0 += 65535) {
    const size_t c = std::min<size_t>(65535, pn.size() - k0);
    DevBuf<PackNear> d;
    d.upload(pn.data() + k0, c, s);
    k_pack_near<TN><<<static_cast<unsigned>(c), 256, 0, s>>>(d.p, H.near_pool64.p, reinterpret_cast<TN*>(H.near_f.p));
    SPX_LAUNCH_CHECK();
    SPX_CUDA(cudaStreamSynchronize(s));
  }
  H.far_meta.upload(fmeta, s);
  H.far_uoff.upload(fu, s);
  H.far_voff.upload(fv, s);
  H.far_zoff.upload(fz, s);
  H.near_meta.upload(nmeta, s);
  H.near_off.upload(noff, s);
  // leaf row clusters: tree leaves in permutation order
  std::vector<int32_t> ls;
  for (const TreeNode& nd : H.tree.nodes)
    if (nd.leaf()) ls.push_back(nd.start);
  std::sort(ls.begin(), ls.end());
  ls.push_back(static_cast<int32_t>(H.Nb));
  const int64_t nleaf = static_cast<int64_t>(ls.size()) - 1;
  std::vector<std::vector<int32_t>> per(nleaf);
  for (size_t q = 0; q < H.blocks.size(); ++q) {
    const HBlock& b = H.blocks[q];
    int64_t l = std::upper_bound(ls.begin(), ls.end(), b.rs) - ls.begin() - 1;
    for (; l < nleaf && ls[l] < b.re; ++l) per[l].push_back(code_of[q]);
  }
  std::vector<int64_t> ip(nleaf + 1, 0);
  std::vector<int32_t> items;
  for (int64_t l = 0; l < nleaf; ++l) {
    items.insert(items.end(), per[l].begin(), per[l].end());
    ip[l + 1] = static_cast<int64_t>(items.size());
  }
  H.nleaf = nleaf;
  H.leaf_start.upload(ls, s);
  H.item_ptr.upload(ip, s);
  H.items.upload(items, s);
  int max_leaf = 0;
  for (int64_t l = 0; l < nleaf; ++l) max_leaf = std::max(max_leaf, ls[l + 1] - ls[l]);
  SPX_CHECK(max_leaf <= 2048, "leaf clusters larger than 2048 rows are not supported by the apply kernel");
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class TF, class TN, class TA, class TX, class TS>
void do_apply(HMatrix& H, const TS* src, const int32_t* gidx, TS* dst, const TS* add, TS* yb, cudaStream_t s) {
  const int64_t Nb = H.Nb;
  if (H.xperm.n < Nb * sizeof(TX)) H.xperm.alloc(Nb * sizeof(TX));
  if (H.z.n < std::max<int64_t>(H.zlen, 1) * sizeof(TA)) H.z.alloc(std::max<int64_t>(H.zlen, 1) * sizeof(TA));
  TX* xp = reinterpret_cast<TX*>(H.xperm.p);
  TA* z = reinterpret_cast<TA*>(H.z.p);
  k_hgather<TS, TX><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, src, gidx, H.perm.p, xp);
  SPX_LAUNCH_CHECK();
  if (H.n_far > 0) {
    k_far_z<TF, TA, TX><<<static_cast<unsigned>(H.n_far), 128, 0, s>>>(
        H.far_meta.p, H.far_voff.p, H.far_zoff.p, reinterpret_cast<const TF*>(H.far_f.p), xp, z);
    SPX_LAUNCH_CHECK();
  }
  int max_leaf = H.cfg.leaf_size;
  const size_t smem = 2 * ROWS_GROUPS * static_cast<size_t>(std::max(max_leaf, 1)) * sizeof(TA);
  k_rows<TF, TN, TA, TX, TS><<<static_cast<unsigned>(H.nleaf), ROWS_GROUPS * ROWS_GSIZE, smem, s>>>(
      H.leaf_start.p, H.item_ptr.p, H.items.p, H.far_meta.p, H.far_uoff.p, H.far_zoff.p,
      reinterpret_cast<const TF*>(H.far_f.p), H.near_meta.p, H.near_off.p,
      reinterpret_cast<const TN*>(H.near_f.p), z, xp, H.diag_perm.p, H.perm.p, gidx, dst, add, yb,
      (H.prec == Prec::MIXED && sizeof(TA) == sizeof(float)) ? 1 : 0);
  SPX_LAUNCH_CHECK();
}
}  // namespace

void HMatrix::pack(Prec p, cudaStream_t s) {
  prec = p;
  switch (p) {
    case Prec::F64: do_pack<double, double>(*this, s); break;
    case Prec::F32: do_pack<float, float>(*this, s); break;
    case Prec::MIXED: do_pack<__nv_bfloat16, float>(*this, s); break;
  }
  packed = true;
}

template <class T>
void HMatrix::apply_gather(const T* src, const int32_t* gidx, T* dst, const T* add, T* yb, cudaStream_t s) {
  SPX_CHECK(packed, "H-matrix is not packed");
  // FP64 vectors accumulate in FP64 whatever the factor storage; FP32 vectors in FP32
  if (sizeof(T) == sizeof(double)) {
    switch (prec) {
      case Prec::F64: do_apply<double, double, double, double, T>(*this, src, gidx, dst, add, yb, s); break;
      case Prec::F32: do_apply<float, float, double, double, T>(*this, src, gidx, dst, add, yb, s); break;
      case Prec::MIXED: do_apply<__nv_bfloat16, float, double, double, T>(*this, src, gidx, dst, add, yb, s); break;
    }
  } else {
    switch (prec) {
      case Prec::F64: do_apply<double, double, float, float, T>(*this, src, gidx, dst, add, yb, s); break;
      case Prec::F32: do_apply<float, float, float, float, T>(*this, src, gidx, dst, add, yb, s); break;
      case Prec::MIXED: do_apply<__nv_bfloat16, float, float, float, T>(*this, src, gidx, dst, add, yb, s); break;
    }
  }
}
template void HMatrix::apply_gather<double>(const double*, const int32_t*, double*, const double*, double*, cudaStream_t);
template void HMatrix::apply_gather<float>(const float*, const int32_t*, float*, const float*, float*, cudaStream_t);

void HMatrix::apply_f64(const double* x, double* y, cudaStream_t s) {
  apply_gather<double>(x, nullptr, y, nullptr, nullptr, s);
}

int64_t HMatrix::device_bytes() const {
  return static_cast<int64_t>(far_f.bytes() + near_f.bytes() + far_uoff.bytes() + far_voff.bytes() +
                              far_zoff.bytes() + far_meta.bytes() + near_off.bytes() + near_meta.bytes() +
                              leaf_start.bytes() + item_ptr.bytes() + items.bytes() + z.bytes() +
                              xperm.bytes() + diag_perm.bytes() + perm.bytes());
}

}  // namespace spx

// ------------------------------------------------------------------ apply without allocation
// spx_hmat_apply_noalloc runs the same three kernels as spx_hmat_apply, but its scratch
// (x in permuted order, then the far-field z vectors) lives in this fixed device array
// instead of buffers allocated on first use.  Every device that loads the library holds
// the array until the process exits.  In host code the symbol is only a stand-in: the
// device address comes from cudaGetSymbolAddress, looked up once per device.
namespace spx {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

void* noalloc_scratch_address() {
  static std::mutex mu;
  static std::vector<void*> addr;
  int dev = 0;
  SPX_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (static_cast<size_t>(dev) >= addr.size()) addr.resize(dev + 1, nullptr);
  if (!addr[dev]) {
    void* p = nullptr;
    SPX_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    addr[dev] = p;
  }
  return addr[dev];
}

template <class TF, class TN, class TA, class TX>
void apply_noalloc_impl(HMatrix& H, const double* x, double* y, cudaStream_t s) {
  const int64_t Nb = H.Nb;
  const size_t xbytes = ((static_cast<size_t>(Nb) * sizeof(TX) + 255) / 256) * 256;
  const size_t zbytes = static_cast<size_t>(std::max<int64_t>(H.zlen, 1)) * sizeof(TA);
  if (xbytes + zbytes > kNoAllocScratchBytes)
    throw Error(ERR_INVALID, "H-matrix too large for the 32 MiB static scratch of spx_hmat_apply_noalloc "
                             "(needs " + std::to_string(xbytes + zbytes) + " bytes); use spx_hmat_apply");
  unsigned char* base = static_cast<unsigned char*>(noalloc_scratch_address());
  TX* xp = reinterpret_cast<TX*>(base);
  TA* z = reinterpret_cast<TA*>(base + xbytes);
  k_hgather<double, TX><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, x, nullptr, H.perm.p, xp);
  SPX_LAUNCH_CHECK();
  if (H.n_far > 0) {
    k_far_z<TF, TA, TX><<<static_cast<unsigned>(H.n_far), 128, 0, s>>>(
        H.far_meta.p, H.far_voff.p, H.far_zoff.p, reinterpret_cast<const TF*>(H.far_f.p), xp, z);
    SPX_LAUNCH_CHECK();
  }
  const size_t smem = 2 * ROWS_GROUPS * static_cast<size_t>(std::max(H.cfg.leaf_size, 1)) * sizeof(TA);
  k_rows<TF, TN, TA, TX, double><<<static_cast<unsigned>(H.nleaf), ROWS_GROUPS * ROWS_GSIZE, smem, s>>>(
      H.leaf_start.p, H.item_ptr.p, H.items.p, H.far_meta.p, H.far_uoff.p, H.far_zoff.p,
      reinterpret_cast<const TF*>(H.far_f.p), H.near_meta.p, H.near_off.p,
      reinterpret_cast<const TN*>(H.near_f.p), z, xp, H.diag_perm.p, H.perm.p, nullptr, y, nullptr, nullptr,
      (H.prec == Prec::MIXED && sizeof(TA) == sizeof(float)) ? 1 : 0);
  SPX_LAUNCH_CHECK();
}

}  // namespace

void hmat_apply_noalloc(HMatrix& H, const double* x, double* y, cudaStream_t s) {
  SPX_CHECK(H.packed, "H-matrix is not packed");
  switch (H.prec) {
    case Prec::F64: apply_noalloc_impl<double, double, double, double>(H, x, y, s); break;
    case Prec::F32: apply_noalloc_impl<float, float, double, double>(H, x, y, s); break;
    case Prec::MIXED: apply_noalloc_impl<__nv_bfloat16, float, double, double>(H, x, y, s); break;
  }
}

}  // namespace spx
