// H-matrix apply: y = P^-1 [diag o x~ + Near x~ + sum_b U_b (V_b x~_{J_b})],  x~ = x[perm]
// (HMatrixGPUPackedFused.matvec, lindholm_hmatrix_gpu/backend_fused.py:496-512).
//
// B200 layout (built by pack() from the FP64 pools of the builder, in the storage type TF of
// the far factors -- FP64, FP32 or BF16 -- and TN of the near tiles -- FP64 or FP32):
//   * row segments: the leaf clusters in permutation order, split into pieces of at most
//     64 rows; every output row belongs to exactly one segment.
//   * V_b^T of each far block: n rows of ldk = k rounded up to 16 bytes (row c holds
//     V_b[0..k-1, c]), cut into units of at most ~16 KB of rows.
//   * U_b of each far block, cut at the segments it covers: per segment a tile of k rows of
//     ld = rows rounded up to a 16-byte multiple (row q holds U[rows, q]).
//   * near blocks, cut the same way: per segment a tile of n columns of ld entries.
// Every tile and row starts 16-byte aligned and is zero padded, so all factor traffic is
// 16-byte vector loads of contiguous memory.
//
// Kernels (no atomics on data, every output written by exactly one warp or CTA):
//   k_hgather : x~[i] = src[g(perm[i])]             (fused boundary gather + perm)
//   k_far_z   : z_b = V_b x~_{J_b} = sum_c x~_c V_b^T[c, :].  Persistent warps over contiguous,
//               byte-balanced unit ranges; lanes = (16-byte vector of outputs q, phase over
//               rows c), accumulating in registers across the units of a block; at the
//               block's last unit in the warp a shuffle sum over the phases writes z_b.  A
//               block shared by several warps (only at range ends) adds the warps' partials
//               through an arrival counter: the last arriving warp sums them in contributor
//               order and resets the counter, so z does not depend on scheduling.
//   k_rows    : one CTA per row segment; its warps take the segment's items (U tiles with z_b,
//               near tiles with x~) round-robin, lanes over 16-byte row vectors x phases over
//               the tile rows, then a fixed-order sum over warps, + diag o x~, scattered to
//               dst[g(perm[i])].
// Each warp keeps the factor data of its next units / items moving into L2 with
// cp.async.bulk.prefetch.L2 (a few units ahead), so its own 16-byte loads mostly hit L2.
// Near tiles use compensated (Kahan) accumulation when FP32 accumulates BF16/FP32 data in
// the mixed-precision form.
#include <algorithm>
#include <mutex>
#include <string>

#include <cuda_fp16.h>

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
namespace {
constexpr int Z_WARPS = 8;      // warps per far_z CTA
constexpr int Z_CTAS_PER_SM = 4;
constexpr int SEG_MAX = 64;     // rows per segment
constexpr int ROWS_WARPS = 8;   // warps per k_rows CTA
inline int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }
}  // namespace

// dst[q * ld + r] = pool[src + q * sq + r * sr] * (scaled by qscale[qs + q] when qs >= 0, or
// by rscale[qs + r] when rs != 0) for r < nr, 0 for nr <= r < ld, q < nq
struct PackJob {
  int64_t src, dst;
  int32_t nq, nr, ld, sq, sr;
  int64_t qs = -1;  // first scale factor of this job (-1: none)
  int32_t rs = 0;   // 1: the scale runs along r instead of q
};
template <class T> __device__ __forceinline__ T from_d_s(double v) { return from_d<T>(v); }
template <> __device__ __forceinline__ __half from_d_s<__half>(double v) { return __double2half(v); }
template <class T>
__global__ void k_pack(const PackJob* __restrict__ jobs, int64_t njobs, const double* __restrict__ pool,
                       const double* __restrict__ scale, T* __restrict__ out) {
  for (int64_t jb = blockIdx.x; jb < njobs; jb += gridDim.x) {
    const PackJob j = jobs[jb];
    const int64_t L = static_cast<int64_t>(j.nq) * j.ld;
    for (int64_t e = threadIdx.x; e < L; e += blockDim.x) {
      const int64_t q = e / j.ld, r = e - q * j.ld;
      double v = r < j.nr ? pool[j.src + q * j.sq + r * j.sr] : 0.0;
      if (j.qs >= 0 && r < j.nr) v *= scale[j.qs + (j.rs ? r : q)];
      out[j.dst + e] = from_d_s<T>(v);
    }
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
template <> struct V16<__half> { using T = uint4; static constexpr int E = 8; };

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
template <class TA>
__device__ __forceinline__ void h16x8(const uint4& v, TA out[8]) {
  const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[q]));
    out[2 * q] = static_cast<TA>(f.x);
    out[2 * q + 1] = static_cast<TA>(f.y);
  }
}
template <>
__device__ __forceinline__ void v16_elems<double, __half>(const uint4& v, double out[8]) { h16x8<double>(v, out); }
template <>
__device__ __forceinline__ void v16_elems<float, __half>(const uint4& v, float out[8]) { h16x8<float>(v, out); }
template <>
__device__ __forceinline__ void v16_elems<double, __nv_bfloat16>(const uint4& v, double out[8]) { bf16x8<double>(v, out); }
template <>
__device__ __forceinline__ void v16_elems<float, __nv_bfloat16>(const uint4& v, float out[8]) { bf16x8<float>(v, out); }


__device__ __forceinline__ int log2_ceil_le5(int n) {
  int l = 0;
  while ((1 << l) < n && l < 5) ++l;
  return l;
}

// asynchronous prefetch of a contiguous range into L2 (cp.async.bulk.prefetch.L2; 16-byte
// aligned address, size a multiple of 16)
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

#ifndef SPX_Z_PF
#define SPX_Z_PF 1
#endif
#ifndef SPX_R_PF
#define SPX_R_PF 1
#endif
constexpr int Z_PF = SPX_Z_PF;  // units prefetched ahead by each far_z warp
constexpr int R_PF = SPX_R_PF;  // items prefetched ahead by each rows warp

template <class TF, class TA, class TX>
__global__ void __launch_bounds__(Z_WARPS * 32, Z_CTAS_PER_SM)
    k_far_z(const FarUnit* __restrict__ units, const int32_t* __restrict__ warp_first, int nwarps,
            const TF* __restrict__ F, const TX* __restrict__ xp, TA* __restrict__ z, TA* __restrict__ zpart,
            const FarGroup* __restrict__ groups, unsigned int* __restrict__ gcnt) {
  constexpr int E = V16<TF>::E;
  using VT = typename V16<TF>::T;
  using TP = TA;
  const int wg = static_cast<int>((blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5);
  if (wg >= nwarps) return;  // uniform per warp
  const int lane = threadIdx.x & 31;
  const int u1 = warp_first[wg + 1];
  int u = warp_first[wg];
  FarUnit nxt;
  if (u < u1) {
    nxt = units[u];
    if (lane == 0) prefetch_l2(F + nxt.voff, static_cast<uint32_t>(nxt.nc) * nxt.ldk * sizeof(TF));
  }
  TA acc[E];
#pragma unroll
  for (int t = 0; t < E; ++t) acc[t] = TA(0);
  for (; u < u1; ++u) {
    const FarUnit U = nxt;
    if (u + 1 < u1) nxt = units[u + 1];  // descriptor of the next unit in flight
    const int nvq = U.ldk / E;
    const int lg = log2_ceil_le5(nvq);
    const int G = 1 << lg, P = 32 >> lg;
    const int vl = lane & (G - 1), ph = lane >> lg;
    if (vl < nvq) {
      const VT* tile = reinterpret_cast<const VT*>(F + U.voff) + vl;
      const TX* x = xp + U.xc;
      int c = ph;
      for (; c + 3 * P < U.nc; c += 4 * P) {
        VT w[4];
        TP a[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          w[i] = tile[static_cast<int64_t>(c + i * P) * nvq];
          a[i] = static_cast<TP>(x[c + i * P]);
        }
        TP ps[E];
#pragma unroll
        for (int t = 0; t < E; ++t) ps[t] = TP(0);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          TP e[E];
          v16_elems<TP, TF>(w[i], e);
#pragma unroll
          for (int t = 0; t < E; ++t) ps[t] += e[t] * a[i];
        }
#pragma unroll
        for (int t = 0; t < E; ++t) acc[t] += static_cast<TA>(ps[t]);
      }
      for (; c < U.nc; c += P) {
        TP e[E];
        v16_elems<TP, TF>(tile[static_cast<int64_t>(c) * nvq], e);
        const TP a = static_cast<TP>(x[c]);
#pragma unroll
        for (int t = 0; t < E; ++t) acc[t] += static_cast<TA>(e[t] * a);
      }
    }
    if (lane == 0 && u + 1 < u1)  // the next unit's V^T rows into L2
      prefetch_l2(F + nxt.voff, static_cast<uint32_t>(nxt.nc) * nxt.ldk * sizeof(TF));
    const int fl = U.flags & 3;
    if (fl == 0) continue;
    // the block ends in this warp: sum over the phases, write its k rows
#pragma unroll
    for (int t = 0; t < E; ++t)
      for (int o = G; o < 32; o <<= 1) acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], o);
    TA* out = fl == 1 ? z : zpart;
    if (ph == 0 && vl < nvq) {
#pragma unroll
      for (int t = 0; t < E; ++t) {
        const int q = vl * E + t;
        if (q < U.k) out[U.zout + q] = acc[t];
      }
    }
#pragma unroll
    for (int t = 0; t < E; ++t) acc[t] = TA(0);
    if (fl == 2) {  // block shared between warps: the last contributor sums the partials in order
      __threadfence();
      __syncwarp();
      const FarGroup Gp = groups[U.grp];
      unsigned last = 0;
      if (lane == 0) last = atomicAdd(gcnt + U.grp, 1u) == static_cast<unsigned>(Gp.ncontrib) - 1u ? 1u : 0u;
      last = __shfl_sync(0xffffffffu, last, 0);
      if (last) {
        __threadfence();
        for (int q = lane; q < Gp.k; q += 32) {
          TA sum = TA(0);
          for (int cc = 0; cc < Gp.ncontrib; ++cc) sum += __ldcg(zpart + Gp.pbase + cc * U.ldk + q);
          z[Gp.zdst + q] = sum;
        }
        if (lane == 0) atomicExch(gcnt + U.grp, 0u);
      }
    }
  }
}

// Accumulate one warp's share of a segment's items: item it covers tile rows q < len of
// ld = round_up(nr, E) entries; row q is multiplied by vs[item.src + q].
template <class T, class TA, class TV>
__device__ __forceinline__ void rows_items(const RowItem* __restrict__ items, int64_t first, int64_t end,
                                           const T* __restrict__ base, const TV* __restrict__ vs, int nr,
                                           TA* __restrict__ part, int lane, bool kahan,
                                           const double* __restrict__ vscale = nullptr) {
  constexpr int E = V16<T>::E;
  using VT = typename V16<T>::T;
  const int nvec = (nr + E - 1) / E;
  const int lg = log2_ceil_le5(nvec);
  const int G = 1 << lg, P = 32 >> lg;
  const int vl = lane & (G - 1), ph = lane >> lg;
  TA acc[E], cmp[E];
#pragma unroll
  for (int t = 0; t < E; ++t) acc[t] = cmp[t] = TA(0);
  using TP = TA;
  const bool active = vl < nvec;
  RowItem nxt;
  if (first < end) nxt = items[first];
  if (lane < R_PF) {  // the first items' tiles into L2
    const int64_t f = first + static_cast<int64_t>(lane) * ROWS_WARPS;
    if (f < end) {
      const RowItem P = items[f];
      prefetch_l2(base + P.off, static_cast<uint32_t>(P.len) * static_cast<uint32_t>(nvec) * 16u);
    }
  }
  for (int64_t it = first; it < end; it += ROWS_WARPS) {
    const RowItem I = nxt;
    if (it + ROWS_WARPS < end) nxt = items[it + ROWS_WARPS];
    const int64_t fp = it + static_cast<int64_t>(R_PF) * ROWS_WARPS;
    if (lane == 0 && fp < end) {
      const RowItem P = items[fp];
      prefetch_l2(base + P.off, static_cast<uint32_t>(P.len) * static_cast<uint32_t>(nvec) * 16u);
    }
    if (!active) continue;
    const VT* tile = reinterpret_cast<const VT*>(base + I.off) + vl;
    const TV* v = vs + I.src;
    const double* sc = vscale ? vscale + I.src : nullptr;
    int q = ph;
    for (; q + 3 * P < I.len; q += 4 * P) {
      VT w[4];
      TA a[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        w[u] = tile[static_cast<int64_t>(q + u * P) * nvec];
        a[u] = static_cast<TA>(v[q + u * P]);
        if (sc) a[u] *= static_cast<TA>(sc[q + u * P]);
      }
      if (kahan) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          TA e[E];
          v16_elems<TA, T>(w[u], e);
#pragma unroll
          for (int t = 0; t < E; ++t) {
            const TA y = e[t] * a[u] - cmp[t];
            const TA s = acc[t] + y;
            cmp[t] = (s - acc[t]) - y;
            acc[t] = s;
          }
        }
      } else {
        TP ps[E];
#pragma unroll
        for (int t = 0; t < E; ++t) ps[t] = TP(0);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          TP e[E];
          v16_elems<TP, T>(w[u], e);
          const TP au = static_cast<TP>(a[u]);
#pragma unroll
          for (int t = 0; t < E; ++t) ps[t] += e[t] * au;
        }
#pragma unroll
        for (int t = 0; t < E; ++t) acc[t] += static_cast<TA>(ps[t]);
      }
    }
    for (; q < I.len; q += P) {
      const VT w = tile[static_cast<int64_t>(q) * nvec];
      const TA a = static_cast<TA>(v[q]) * (sc ? static_cast<TA>(sc[q]) : TA(1));
      TA e[E];
      v16_elems<TA, T>(w, e);
      if (kahan) {
#pragma unroll
        for (int t = 0; t < E; ++t) {
          const TA y = e[t] * a - cmp[t];
          const TA s = acc[t] + y;
          cmp[t] = (s - acc[t]) - y;
          acc[t] = s;
        }
      } else {
#pragma unroll
        for (int t = 0; t < E; ++t) acc[t] += e[t] * a;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < E; ++t) {
    TA y = acc[t] - cmp[t];
    for (int o = G; o < 32; o <<= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
    acc[t] = y;
  }
  if (ph == 0 && active) {
#pragma unroll
    for (int t = 0; t < E; ++t) {
      const int r = vl * E + t;
      if (r < nr) part[r] += acc[t];
    }
  }
  __syncwarp();
}

template <class TF, class TN, class TA, class TX, class TD>
__global__ void __launch_bounds__(ROWS_WARPS * 32) k_rows(
    const int32_t* __restrict__ seg_start, const int64_t* __restrict__ item_ptr,
    const int64_t* __restrict__ near_begin, const RowItem* __restrict__ items, const TF* __restrict__ F,
    const TN* __restrict__ Nt, const TA* __restrict__ z, const TX* __restrict__ xp,
    const double* __restrict__ diag, const int32_t* __restrict__ perm, const int32_t* __restrict__ gidx,
    TD* __restrict__ dst, const TD* __restrict__ add, TD* __restrict__ yb, int kahan,
    const int64_t* __restrict__ half_begin, const __half* __restrict__ Fh, const double* __restrict__ zscale) {
  __shared__ TA part[ROWS_WARPS][SEG_MAX];
  const int sgm = blockIdx.x;
  const int r0 = seg_start[sgm], nr = seg_start[sgm + 1] - r0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = lane; r < SEG_MAX; r += 32) part[warp][r] = TA(0);
  __syncwarp();
  const int64_t i0 = item_ptr[sgm], im = near_begin[sgm], i1 = item_ptr[sgm + 1];
  const int64_t ih = half_begin ? half_begin[sgm] : im;
  rows_items<TF, TA, TA>(items, i0 + warp, ih, F, z, nr, part[warp], lane, false);
  if (ih < im) rows_items<__half, TA, TA>(items, ih + warp, im, Fh, z, nr, part[warp], lane, false, zscale);
  rows_items<TN, TA, TX>(items, im + warp, i1, Nt, xp, nr, part[warp], lane, kahan != 0);
  __syncthreads();
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    const int64_t i = r0 + r;
    TA y = static_cast<TA>(diag[i]) * static_cast<TA>(xp[i]);
#pragma unroll
    for (int w = 0; w < ROWS_WARPS; ++w) y += part[w][r];
    const int32_t b = perm[i];
    const int64_t o = gidx ? gidx[b] : b;
    const TD yv = static_cast<TD>(y);
    dst[o] = add ? static_cast<TD>(add[o] + yv) : yv;
    if (yb) yb[b] = yv;
  }
}

// ------------------------------------------------------------------ host side
namespace {

template <class T>
void run_pack_jobs(const std::vector<PackJob>& jobs, const double* pool, const double* scale, char* out,
                   cudaStream_t s) {
  if (jobs.empty()) return;
  constexpr size_t CH = size_t(1) << 20;
  for (size_t k0 = 0; k0 < jobs.size(); k0 += CH) {
    const size_t c = std::min(CH, jobs.size() - k0);
    DevBuf<PackJob> d;
    d.upload(jobs.data() + k0, c, s);
    const unsigned grid = static_cast<unsigned>(std::min<size_t>(c, 65535));
    k_pack<T><<<grid, 128, 0, s>>>(d.p, static_cast<int64_t>(c), pool, scale, reinterpret_cast<T*>(out));
    SPX_LAUNCH_CHECK();
    SPX_CUDA(cudaStreamSynchronize(s));
  }
}

// far_z units dealt to warps in contiguous ranges of about equal cost; the last unit of a
// block in each warp writes the block (flags 1), or contributes partials to a group (flags 2)
// whose slots start at *ppos.  Returns the warp ranges.
std::vector<int32_t> plan_units(std::vector<FarUnit>& units, size_t elem_bytes, int nsm, int64_t& nw_out,
                                std::vector<FarGroup>& groups, int64_t& ppos) {
  const int64_t nw = std::max<int64_t>(1, std::min<int64_t>(static_cast<int64_t>(nsm) * Z_CTAS_PER_SM * Z_WARPS,
                                                            static_cast<int64_t>(units.size())));
  std::vector<double> cost(units.size() + 1, 0.0);
  for (size_t u = 0; u < units.size(); ++u) {
    const FarUnit& U = units[u];
    cost[u + 1] = cost[u] + static_cast<double>(U.nc) * U.ldk * elem_bytes + 8.0 * U.nc + 512.0;
  }
  std::vector<int32_t> wf(nw + 1, 0);
  {
    size_t u = 0;
    for (int64_t w = 0; w <= nw; ++w) {
      const double target = cost.back() * static_cast<double>(w) / static_cast<double>(nw);
      while (u < units.size() && cost[u] < target) ++u;
      wf[w] = static_cast<int32_t>(u);
    }
    wf[nw] = static_cast<int32_t>(units.size());
  }
  std::vector<int32_t> warp_of(units.size());
  for (int64_t w = 0; w < nw; ++w)
    for (int32_t u = wf[w]; u < wf[w + 1]; ++u) warp_of[u] = static_cast<int32_t>(w);
  size_t u = 0;
  while (u < units.size()) {
    size_t e = u;
    while (e < units.size() && units[e].zout == units[u].zout) ++e;  // block = units [u, e)
    std::vector<size_t> lasts;
    for (size_t v = u; v < e; ++v)
      if (v + 1 == e || warp_of[v + 1] != warp_of[v]) lasts.push_back(v);
    if (lasts.size() == 1) {
      units[lasts[0]].flags = 1;
    } else {
      const int32_t g = static_cast<int32_t>(groups.size());
      groups.push_back(FarGroup{static_cast<int32_t>(ppos), static_cast<int32_t>(lasts.size()), units[u].zout,
                                units[u].k});
      for (size_t c = 0; c < lasts.size(); ++c) {
        FarUnit& L = units[lasts[c]];
        L.flags = 2;
        L.grp = g;
        L.zout = static_cast<int32_t>(ppos + static_cast<int64_t>(c) * L.ldk);
      }
      ppos += static_cast<int64_t>(lasts.size()) * units[u].ldk;
    }
    u = e;
  }
  nw_out = units.empty() ? 0 : nw;
  return wf;
}

// FP32 columns kept by a recompressed block under the split packing: the trailing columns go
// to FP16 when their rounding (relative 2^-11 in U and in V) stays within a tenth of the
// block's error budget, sqrt(sum_{j>=c} 2 (sigma_j 2^-11)^2) <= 0.1 eps ||A||; rounded up to
// a multiple of 4 (the FP32 vector width); k (all FP32) without singular values.
int split_head(const std::vector<double>& sig, int k, double eps) {
  if (static_cast<int>(sig.size()) != k || k == 0) return k;
  double n2 = 0.0;
  for (double v : sig) n2 += v * v;
  const double bud = 0.1 * eps * std::sqrt(n2);
  const double u16 = std::ldexp(1.0, -11);
  double acc = 0.0;
  int c = k;
  for (int j = k - 1; j >= 0; --j) {
    acc += 2.0 * (sig[j] * u16) * (sig[j] * u16);
    if (std::sqrt(acc) > bud) break;
    c = j;
  }
  const int c4 = static_cast<int>(round_up(c, 4));
  return c4 >= k ? k : c4;
}

template <class TF, class TN>
void do_pack(HMatrix& H, cudaStream_t s, bool split = false) {
  constexpr int EF = 16 / static_cast<int>(sizeof(TF));
  constexpr int EN = 16 / static_cast<int>(sizeof(TN));
  constexpr int EH = 8;  // FP16 elements per 16 bytes
  // row segments: leaf clusters in permutation order, cut into pieces of <= SEG_MAX rows
  std::vector<int32_t> ls;
  for (const TreeNode& nd : H.tree.nodes)
    if (nd.leaf()) ls.push_back(nd.start);
  std::sort(ls.begin(), ls.end());
  ls.push_back(static_cast<int32_t>(H.Nb));
  std::vector<int32_t> seg;
  for (size_t l = 0; l + 1 < ls.size(); ++l) {
    const int32_t a = ls[l], n = ls[l + 1] - ls[l];
    const int32_t pieces = (n + SEG_MAX - 1) / SEG_MAX;
    for (int32_t p = 0; p < pieces; ++p) seg.push_back(a + static_cast<int32_t>((int64_t)n * p / pieces));
  }
  seg.push_back(static_cast<int32_t>(H.Nb));
  const int64_t nseg = static_cast<int64_t>(seg.size()) - 1;

  std::vector<PackJob> jf, jn, jh;
  std::vector<FarUnit> units, units_h;
  std::vector<std::vector<RowItem>> far_items(nseg), half_items(nseg), near_items(nseg);
  std::vector<double> scale;  // 1 / sigma of the FP16 columns of U (pack), sigma per z entry (apply)
  std::vector<double> zsc;
  int64_t fpos = 0, hpos = 0, npos = 0, zpos = 0, nf = 0, nn = 0;
  for (size_t bi = 0; bi < H.blocks.size(); ++bi) {
    const HBlock& b = H.blocks[bi];
    const int32_t m = b.re - b.rs, n = b.ce - b.cs;
    int64_t sg = std::upper_bound(seg.begin(), seg.end(), b.rs) - seg.begin() - 1;
    SPX_CHECK(sg >= 0 && seg[sg] == b.rs, "block rows do not start at a segment boundary");
    if (b.type == 1) {
      const int32_t k = b.rank;
      const int32_t kh = split ? split_head(H.sigma.empty() ? std::vector<double>() : H.sigma[bi], k,
                                            H.cfg.epsilon) : k;  // FP32 columns
      const int32_t kt = k - kh;                                 // FP16 columns
      const int32_t ldk = static_cast<int32_t>(round_up(std::max(kh, 1), EF));
      const int64_t pv = fpos;
      // V^T head: n rows of ldk (row c = V[0..kh-1, c]); units of at most ~16 KB of rows
      jf.push_back(PackJob{b.off_v, pv, n, kh, ldk, 1, n});
      fpos = pv + static_cast<int64_t>(n) * ldk;
      if (kh > 0) {
        const int32_t uc = std::max<int32_t>(8, static_cast<int32_t>(16384 / (static_cast<int64_t>(ldk) * sizeof(TF))));
        for (int32_t c0 = 0; c0 < n; c0 += uc)
          units.push_back(FarUnit{pv + static_cast<int64_t>(c0) * ldk, ldk, std::min(uc, n - c0), b.cs + c0, kh,
                                  static_cast<int32_t>(zpos), -1, 0, 0});
      }
      int64_t sgu = sg;
      for (; sgu < nseg && seg[sgu] < b.re; ++sgu) {
        const int32_t a = seg[sgu], nr = seg[sgu + 1] - seg[sgu];
        const int32_t ld = static_cast<int32_t>(round_up(nr, EF));
        jf.push_back(PackJob{b.off_u + (a - b.rs), fpos, kh, nr, ld, m, 1});
        far_items[sgu].push_back(RowItem{fpos, kh, static_cast<int32_t>(zpos)});
        fpos = round_up(fpos + (int64_t)kh * ld, EF);
      }
      for (int32_t q = 0; q < kh; ++q) zsc.push_back(1.0);
      if (kt > 0) {
        // tail: unit columns of U (scaled by 1 / sigma) and unit rows of V in FP16; z of the
        // tail is scaled back by sigma in the row kernel
        const std::vector<double>& sig = H.sigma[bi];
        const int64_t s0 = static_cast<int64_t>(scale.size());
        for (int32_t q = 0; q < kt; ++q) scale.push_back(1.0 / sig[kh + q]);
        const int32_t ldh = static_cast<int32_t>(round_up(kt, EH));
        const int64_t ph = hpos;
        jh.push_back(PackJob{b.off_v + static_cast<int64_t>(kh) * n, ph, n, kt, ldh, 1, n});
        hpos = ph + static_cast<int64_t>(n) * ldh;
        const int32_t uc = std::max<int32_t>(8, static_cast<int32_t>(16384 / (static_cast<int64_t>(ldh) * 2)));
        for (int32_t c0 = 0; c0 < n; c0 += uc)
          units_h.push_back(FarUnit{ph + static_cast<int64_t>(c0) * ldh, ldh, std::min(uc, n - c0), b.cs + c0, kt,
                                    static_cast<int32_t>(zpos + kh), -1, 0, 0});
        for (sgu = sg; sgu < nseg && seg[sgu] < b.re; ++sgu) {
          const int32_t a = seg[sgu], nr = seg[sgu + 1] - seg[sgu];
          const int32_t ld = static_cast<int32_t>(round_up(nr, EH));
          PackJob J{b.off_u + static_cast<int64_t>(kh) * m + (a - b.rs), hpos, kt, nr, ld, m, 1};
          J.qs = s0;
          jh.push_back(J);
          half_items[sgu].push_back(RowItem{hpos, kt, static_cast<int32_t>(zpos + kh)});
          hpos = round_up(hpos + (int64_t)kt * ld, EH);
        }
        for (int32_t q = 0; q < kt; ++q) zsc.push_back(sig[kh + q]);
      }
      zpos += k;
      ++nf;
    } else {
      for (; sg < nseg && seg[sg] < b.re; ++sg) {
        const int32_t a = seg[sg], nr = seg[sg + 1] - seg[sg];
        const int32_t ld = static_cast<int32_t>(round_up(nr, EN));
        jn.push_back(PackJob{b.off_u + (int64_t)(a - b.rs) * n, npos, n, nr, ld, 1, n});
        near_items[sg].push_back(RowItem{npos, n, b.cs});
        npos = round_up(npos + (int64_t)n * ld, EN);
      }
      ++nn;
    }
  }
  SPX_CHECK(zpos < (int64_t(1) << 31), "far-field rank sum exceeds 2^31");
  H.n_far = nf;
  H.n_near = nn;
  H.zlen = zpos;
  H.far_f.alloc(std::max<int64_t>(fpos, 1) * sizeof(TF));
  H.near_f.alloc(std::max<int64_t>(npos, 1) * sizeof(TN));
  H.far_h.alloc(hpos > 0 ? hpos * 2 : 0);
  H.bytes_far = fpos * (int64_t)sizeof(TF) + hpos * 2;
  H.bytes_near = npos * (int64_t)sizeof(TN);
  const bool bf = (H.prec == Prec::MIXED);
  if (sizeof(TF) == 8) run_pack_jobs<double>(jf, H.far_pool64.p, nullptr, H.far_f.p, s);
  else if (bf) run_pack_jobs<__nv_bfloat16>(jf, H.far_pool64.p, nullptr, H.far_f.p, s);
  else run_pack_jobs<float>(jf, H.far_pool64.p, nullptr, H.far_f.p, s);
  if (sizeof(TN) == 8) run_pack_jobs<double>(jn, H.near_pool64.p, nullptr, H.near_f.p, s);
  else run_pack_jobs<float>(jn, H.near_pool64.p, nullptr, H.near_f.p, s);
  if (!jh.empty()) {
    DevBuf<double> dsc;
    dsc.upload(scale, s);
    run_pack_jobs<__half>(jh, H.far_pool64.p, dsc.p, H.far_h.p, s);
  }

  const int nsm = num_sms(H.device);
  std::vector<FarGroup> groups;
  int64_t ppos = 0, nw = 0, nwh = 0;
  std::vector<int32_t> wf = plan_units(units, sizeof(TF), nsm, nw, groups, ppos);
  const int32_t g_h0 = static_cast<int32_t>(groups.size());
  std::vector<int32_t> wfh = plan_units(units_h, 2, nsm, nwh, groups, ppos);
  (void)g_h0;
  SPX_CHECK(ppos < (int64_t(1) << 31), "far-field partial slots exceed 2^31");
  auto check_units = [&](const std::vector<FarUnit>& us, int64_t cap, int E) {
    for (const FarUnit& U : us)
      SPX_CHECK(U.voff % E == 0 && U.nc >= 1 && U.k >= 1 && U.ldk % E == 0 && U.ldk >= U.k &&
                    U.voff + static_cast<int64_t>(U.nc) * U.ldk <= cap && U.xc >= 0 &&
                    U.xc + static_cast<int64_t>(U.nc) <= H.Nb &&
                    ((U.flags & 3) != 2 || (U.grp >= 0 && U.grp < static_cast<int64_t>(groups.size()) &&
                                            U.zout + static_cast<int64_t>(U.k) <= ppos)),
                "far_z plan: unit out of range");
  };
  check_units(units, fpos, EF);
  check_units(units_h, hpos, EH);
  H.zpart_len = ppos;
  H.nunits = static_cast<int64_t>(units.size());
  H.nwarps_z = nw;
  H.nunits_h = static_cast<int64_t>(units_h.size());
  H.nwarps_z_h = nwh;
  H.units.upload(units, s);
  H.warp_first.upload(wf, s);
  H.units_h.upload(units_h, s);
  H.warp_first_h.upload(wfh, s);
  H.groups.upload(groups, s);
  H.gcnt.alloc(std::max<size_t>(groups.size(), 1));
  H.gcnt.zero(s);

  std::vector<int64_t> ip(nseg + 1, 0), nb(nseg, 0), hb(nseg, 0);
  std::vector<RowItem> items;
  for (int64_t g = 0; g < nseg; ++g) {
    items.insert(items.end(), far_items[g].begin(), far_items[g].end());
    hb[g] = static_cast<int64_t>(items.size());
    items.insert(items.end(), half_items[g].begin(), half_items[g].end());
    nb[g] = static_cast<int64_t>(items.size());
    items.insert(items.end(), near_items[g].begin(), near_items[g].end());
    ip[g + 1] = static_cast<int64_t>(items.size());
  }
  H.nseg = nseg;
  H.seg_start.upload(seg, s);
  H.item_ptr.upload(ip, s);
  H.near_begin.upload(nb, s);
  H.items.upload(items, s);
  if (H.nunits_h > 0) {
    H.half_begin.upload(hb, s);
    H.zscale.upload(zsc, s);
  } else {
    H.half_begin.release();
    H.zscale.release();
  }
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class TF, class TN, class TA, class TX, class TS>
void launch_apply(HMatrix& H, const TS* src, const int32_t* gidx, TS* dst, const TS* add, TS* yb, TX* xp, TA* z,
                  TA* zpart, cudaStream_t s) {
  const int64_t Nb = H.Nb;
  k_hgather<TS, TX><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, src, gidx, H.perm.p, xp);
  SPX_LAUNCH_CHECK();
  if (H.nunits > 0) {
    const unsigned ctas = static_cast<unsigned>((H.nwarps_z + Z_WARPS - 1) / Z_WARPS);
    k_far_z<TF, TA, TX><<<ctas, Z_WARPS * 32, 0, s>>>(H.units.p, H.warp_first.p, static_cast<int>(H.nwarps_z),
                                                       reinterpret_cast<const TF*>(H.far_f.p), xp, z, zpart,
                                                       H.groups.p, H.gcnt.p);
    SPX_LAUNCH_CHECK();
  }
  if (H.nunits_h > 0) {  // FP16 trailing columns of the split packing
    const unsigned ctas = static_cast<unsigned>((H.nwarps_z_h + Z_WARPS - 1) / Z_WARPS);
    k_far_z<__half, TA, TX><<<ctas, Z_WARPS * 32, 0, s>>>(
        H.units_h.p, H.warp_first_h.p, static_cast<int>(H.nwarps_z_h), reinterpret_cast<const __half*>(H.far_h.p),
        xp, z, zpart, H.groups.p, H.gcnt.p);
    SPX_LAUNCH_CHECK();
  }
  const bool half = H.nunits_h > 0;
  k_rows<TF, TN, TA, TX, TS><<<static_cast<unsigned>(H.nseg), ROWS_WARPS * 32, 0, s>>>(
      H.seg_start.p, H.item_ptr.p, H.near_begin.p, H.items.p, reinterpret_cast<const TF*>(H.far_f.p),
      reinterpret_cast<const TN*>(H.near_f.p), z, xp, H.diag_perm.p, H.perm.p, gidx, dst, add, yb,
      (H.prec != Prec::F64 && sizeof(TA) == sizeof(float)) ? 1 : 0, half ? H.half_begin.p : nullptr,
      half ? reinterpret_cast<const __half*>(H.far_h.p) : nullptr, half ? H.zscale.p : nullptr);
  SPX_LAUNCH_CHECK();
}

template <class TF, class TN, class TA, class TX, class TS>
void do_apply(HMatrix& H, const TS* src, const int32_t* gidx, TS* dst, const TS* add, TS* yb, cudaStream_t s) {
  const int64_t Nb = H.Nb;
  if (H.xperm.n < Nb * sizeof(TX)) H.xperm.alloc(Nb * sizeof(TX));
  if (H.z.n < std::max<int64_t>(H.zlen, 1) * sizeof(TA)) H.z.alloc(std::max<int64_t>(H.zlen, 1) * sizeof(TA));
  if (H.zpart.n < std::max<int64_t>(H.zpart_len, 1) * sizeof(TA))
    H.zpart.alloc(std::max<int64_t>(H.zpart_len, 1) * sizeof(TA));
  launch_apply<TF, TN, TA, TX, TS>(H, src, gidx, dst, add, yb, reinterpret_cast<TX*>(H.xperm.p),
                                   reinterpret_cast<TA*>(H.z.p), reinterpret_cast<TA*>(H.zpart.p), s);
}
}  // namespace

void HMatrix::pack(Prec p, cudaStream_t s) {
  if (p == Prec::SPLIT && !recompressed) recompress(s);  // the split needs SVD-ordered columns
  tr.reset();
  prec = p;
  switch (p) {
    case Prec::F64: do_pack<double, double>(*this, s); break;
    case Prec::F32: do_pack<float, float>(*this, s); break;
    case Prec::MIXED: do_pack<__nv_bfloat16, float>(*this, s); break;
    case Prec::SPLIT: do_pack<float, float>(*this, s, true); break;
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
      case Prec::F32:
      case Prec::SPLIT: do_apply<float, float, double, double, T>(*this, src, gidx, dst, add, yb, s); break;
      case Prec::MIXED: do_apply<__nv_bfloat16, float, double, double, T>(*this, src, gidx, dst, add, yb, s); break;
    }
  } else {
    switch (prec) {
      case Prec::F64: do_apply<double, double, float, float, T>(*this, src, gidx, dst, add, yb, s); break;
      case Prec::F32:
      case Prec::SPLIT: do_apply<float, float, float, float, T>(*this, src, gidx, dst, add, yb, s); break;
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
  return static_cast<int64_t>(far_f.bytes() + near_f.bytes() + units.bytes() + warp_first.bytes() + groups.bytes() +
                              gcnt.bytes() + seg_start.bytes() + item_ptr.bytes() + near_begin.bytes() +
                              items.bytes() + z.bytes() + zpart.bytes() + xperm.bytes() + diag_perm.bytes() +
                              perm.bytes() + far_h.bytes() + units_h.bytes() + warp_first_h.bytes() +
                              half_begin.bytes() + zscale.bytes());
}

}  // namespace spx

// ------------------------------------------------------------------ apply without allocation
// spx_hmat_apply_noalloc runs the same three kernels as spx_hmat_apply, but its scratch
// (x in permuted order, the far-field z vectors and the partial sums of long rows) lives in
// this fixed device array instead of buffers allocated on first use.  Every device that
// loads the library holds the array until the process exits.  In host code the symbol is
// only a stand-in: the device address comes from cudaGetSymbolAddress, looked up once per
// device.
namespace spx {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
std::atomic<int64_t> g_noalloc_cap{0};  // test cap on the accepted scratch size (0: none)

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
  const size_t zbytes = ((static_cast<size_t>(std::max<int64_t>(H.zlen, 1)) * sizeof(TA) + 255) / 256) * 256;
  const size_t pbytes = static_cast<size_t>(std::max<int64_t>(H.zpart_len, 1)) * sizeof(TA);
  const int64_t cap = g_noalloc_cap.load();
  const size_t limit = cap > 0 ? std::min(kNoAllocScratchBytes, static_cast<size_t>(cap)) : kNoAllocScratchBytes;
  if (xbytes + zbytes + pbytes > limit)
    throw Error(ERR_INVALID, "H-matrix too large for the " + std::to_string(limit) +
                             "-byte static scratch of spx_hmat_apply_noalloc (needs " +
                             std::to_string(xbytes + zbytes + pbytes) + " bytes); use spx_hmat_apply");
  unsigned char* base = static_cast<unsigned char*>(noalloc_scratch_address());
  launch_apply<TF, TN, TA, TX, double>(H, x, nullptr, y, nullptr, nullptr, reinterpret_cast<TX*>(base),
                                       reinterpret_cast<TA*>(base + xbytes),
                                       reinterpret_cast<TA*>(base + xbytes + zbytes), s);
}

}  // namespace

void hmat_apply_noalloc(HMatrix& H, const double* x, double* y, cudaStream_t s) {
  SPX_CHECK(H.packed, "H-matrix is not packed");
  switch (H.prec) {
    case Prec::F64: apply_noalloc_impl<double, double, double, double>(H, x, y, s); break;
    case Prec::F32:
    case Prec::SPLIT: apply_noalloc_impl<float, float, double, double>(H, x, y, s); break;
    case Prec::MIXED: apply_noalloc_impl<__nv_bfloat16, float, double, double>(H, x, y, s); break;
  }
}

}  // namespace spx
