// H-matrix apply to R right-hand sides at once: Y = H X for R states on one boundary (the
// same geometry: a batch of films, samples of an ensemble that share a mesh, tangent
// directions).  The packed factors are those of the single-vector apply (hmat.cu); every
// 16-byte factor vector read from HBM now feeds R accumulators, so the factor traffic of an
// apply is shared by the R states and the per-state cost falls towards the vector traffic.
//
// Layout: the permuted inputs, the far-field z vectors and the partial sums of shared blocks
// are interleaved by state, row-major [row][R] in FP64, so the R values a lane needs for one
// factor vector are contiguous.  Accumulation is FP64.  R <= 8 per pass (R accumulators per
// factor element stay in registers; the CTA-shared row partials of k_rows_multi take 8 x 64
// x R doubles); larger batches are applied in chunks of 8, 4, 2, 1.
//   k_hgather_multi : xm[i][r] = src[g_r(perm[i])]
//   k_far_z_multi   : the unit / warp plan of k_far_z with R columns
//   k_rows_multi    : the segment plan of k_rows with R columns, scattered to dst[g_r(...)]
// g_r(b) = gidx[goff[r] + b] with an index array (ensembles: slices of the boundary vertex
// list), else goff[r] + b.
#include <algorithm>

#include "hmat.cuh"

namespace spx {

namespace {

constexpr int MZ_WARPS = 8;
constexpr int MROWS_WARPS = 8;
constexpr int MSEG = 64;  // rows per segment (the packing's segment bound)

template <class TF> struct W16;
// factor vectors kept in flight per lane: the E x R FP64 accumulators and UF 16-byte vectors
// share the 128 registers a thread has at two CTAs of 256 threads per SM
template <int E, int R> struct InFlight { static constexpr int UF = E * R >= 64 ? 1 : (E * R >= 32 ? 2 : 4); };
template <> struct W16<double> { using T = double2; static constexpr int E = 2; };
template <> struct W16<float> { using T = float4; static constexpr int E = 4; };
template <> struct W16<__nv_bfloat16> { using T = uint4; static constexpr int E = 8; };

__device__ __forceinline__ void elems(const double2& v, double o[2]) { o[0] = v.x; o[1] = v.y; }
__device__ __forceinline__ void elems(const float4& v, double o[4]) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
__device__ __forceinline__ void elems(const uint4& v, double o[8]) {
  const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    o[2 * q] = static_cast<double>(__uint_as_float(w[q] << 16));
    o[2 * q + 1] = static_cast<double>(__uint_as_float(w[q] & 0xffff0000u));
  }
}

__device__ __forceinline__ int lg32(int n) {
  int l = 0;
  while ((1 << l) < n && l < 5) ++l;
  return l;
}

__device__ __forceinline__ void pf_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

struct Offs {
  int64_t v[8];
};

template <class TS, int R>
__global__ void k_hgather_multi(int64_t Nb, const TS* __restrict__ src, const int32_t* __restrict__ gidx, Offs goff,
                                const int32_t* __restrict__ perm, double* __restrict__ xm) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= Nb) return;
  const int32_t b = perm[i];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t o = gidx ? static_cast<int64_t>(gidx[goff.v[r] + b]) : goff.v[r] + b;
    xm[i * R + r] = static_cast<double>(src[o]);
  }
}

// two CTAs per SM (128 registers a thread) unless the accumulators alone take 128 registers
template <class TF, int R>
__global__ void __launch_bounds__(MZ_WARPS * 32, W16<TF>::E * R >= 64 ? 1 : 2)
    k_far_z_multi(const FarUnit* __restrict__ units, const int32_t* __restrict__ warp_first, int nwarps,
                  const TF* __restrict__ F, const double* __restrict__ xm, double* __restrict__ z,
                  double* __restrict__ zpart, const FarGroup* __restrict__ groups, unsigned int* __restrict__ gcnt) {
  constexpr int E = W16<TF>::E;
  using VT = typename W16<TF>::T;
  const int wg = static_cast<int>((blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5);
  if (wg >= nwarps) return;  // uniform per warp
  const int lane = threadIdx.x & 31;
  const int u1 = warp_first[wg + 1];
  int u = warp_first[wg];
  if (u < u1 && lane == 0) pf_l2(F + units[u].voff, static_cast<uint32_t>(units[u].nc) * units[u].ldk * sizeof(TF));
  double acc[E][R];
#pragma unroll
  for (int t = 0; t < E; ++t)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[t][r] = 0.0;
  for (; u < u1; ++u) {
    const FarUnit U = units[u];
    if (lane == 0 && u + 1 < u1) {
      const FarUnit Nx = units[u + 1];
      pf_l2(F + Nx.voff, static_cast<uint32_t>(Nx.nc) * Nx.ldk * sizeof(TF));
    }
    const int nvq = U.ldk / E;
    const int lg = lg32(nvq);
    const int G = 1 << lg, P = 32 >> lg;
    const int vl = lane & (G - 1), ph = lane >> lg;
    if (vl < nvq) {
      const VT* tile = reinterpret_cast<const VT*>(F + U.voff) + vl;
      const double* x = xm + static_cast<int64_t>(U.xc) * R;
      int c = ph;
      constexpr int UF = InFlight<E, R>::UF;
      for (; c + (UF - 1) * P < U.nc; c += UF * P) {  // UF factor vectors in flight
        VT w[UF];
#pragma unroll
        for (int u = 0; u < UF; ++u) w[u] = tile[static_cast<int64_t>(c + u * P) * nvq];
#pragma unroll
        for (int u = 0; u < UF; ++u) {
          double e[E];
          elems(w[u], e);
          const double* xr = x + static_cast<int64_t>(c + u * P) * R;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const double a = xr[r];
#pragma unroll
            for (int t = 0; t < E; ++t) acc[t][r] += e[t] * a;
          }
        }
      }
      for (; c < U.nc; c += P) {
        double e[E];
        elems(tile[static_cast<int64_t>(c) * nvq], e);
        const double* xr = x + static_cast<int64_t>(c) * R;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const double a = xr[r];
#pragma unroll
          for (int t = 0; t < E; ++t) acc[t][r] += e[t] * a;
        }
      }
    }
    const int fl = U.flags & 3;
    if (fl == 0) continue;
#pragma unroll
    for (int t = 0; t < E; ++t)
#pragma unroll
      for (int r = 0; r < R; ++r)
        for (int o = G; o < 32; o <<= 1) acc[t][r] += __shfl_xor_sync(0xffffffffu, acc[t][r], o);
    double* out = fl == 1 ? z : zpart;
    if (ph == 0 && vl < nvq) {
#pragma unroll
      for (int t = 0; t < E; ++t) {
        const int q = vl * E + t;
        if (q < U.k)
#pragma unroll
          for (int r = 0; r < R; ++r) out[(static_cast<int64_t>(U.zout) + q) * R + r] = acc[t][r];
      }
    }
#pragma unroll
    for (int t = 0; t < E; ++t)
#pragma unroll
      for (int r = 0; r < R; ++r) acc[t][r] = 0.0;
    if (fl == 2) {  // block shared between warps: the last contributor sums the partials in order
      __threadfence();
      __syncwarp();
      const FarGroup Gp = groups[U.grp];
      unsigned last = 0;
      if (lane == 0) last = atomicAdd(gcnt + U.grp, 1u) == static_cast<unsigned>(Gp.ncontrib) - 1u ? 1u : 0u;
      last = __shfl_sync(0xffffffffu, last, 0);
      if (last) {
        __threadfence();
        for (int qr = lane; qr < Gp.k * R; qr += 32) {
          const int q = qr / R, r = qr - q * R;
          double sum = 0.0;
          for (int cc = 0; cc < Gp.ncontrib; ++cc)
            sum += __ldcg(zpart + (static_cast<int64_t>(Gp.pbase) + cc * U.ldk + q) * R + r);
          z[(static_cast<int64_t>(Gp.zdst) + q) * R + r] = sum;
        }
        if (lane == 0) atomicExch(gcnt + U.grp, 0u);
      }
    }
  }
}

// one warp's share of a segment's items: part[row][r] += tile rows x v[(src + q)][r]
template <class T, int R>
__device__ __forceinline__ void rows_items_multi(const RowItem* __restrict__ items, int64_t first, int64_t end,
                                                 const T* __restrict__ base, const double* __restrict__ vs, int nr,
                                                 double* __restrict__ part, int lane) {
  constexpr int E = W16<T>::E;
  using VT = typename W16<T>::T;
  const int nvec = (nr + E - 1) / E;
  const int lg = lg32(nvec);
  const int G = 1 << lg, P = 32 >> lg;
  const int vl = lane & (G - 1), ph = lane >> lg;
  double acc[E][R];
#pragma unroll
  for (int t = 0; t < E; ++t)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[t][r] = 0.0;
  for (int64_t it = first; it < end; it += MROWS_WARPS) {
    const RowItem I = items[it];
    if (lane == 0 && it + MROWS_WARPS < end) {
      const RowItem Nx = items[it + MROWS_WARPS];
      pf_l2(base + Nx.off, static_cast<uint32_t>(Nx.len) * static_cast<uint32_t>(nvec) * 16u);
    }
    if (vl >= nvec) continue;
    const VT* tile = reinterpret_cast<const VT*>(base + I.off) + vl;
    const double* v = vs + static_cast<int64_t>(I.src) * R;
    int q = ph;
    constexpr int UF = InFlight<E, R>::UF;
    for (; q + (UF - 1) * P < I.len; q += UF * P) {  // UF tile vectors in flight
      VT w[UF];
#pragma unroll
      for (int u = 0; u < UF; ++u) w[u] = tile[static_cast<int64_t>(q + u * P) * nvec];
#pragma unroll
      for (int u = 0; u < UF; ++u) {
        double e[E];
        elems(w[u], e);
        const double* vr = v + static_cast<int64_t>(q + u * P) * R;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const double a = vr[r];
#pragma unroll
          for (int t = 0; t < E; ++t) acc[t][r] += e[t] * a;
        }
      }
    }
    for (; q < I.len; q += P) {
      double e[E];
      elems(tile[static_cast<int64_t>(q) * nvec], e);
      const double* vr = v + static_cast<int64_t>(q) * R;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double a = vr[r];
#pragma unroll
        for (int t = 0; t < E; ++t) acc[t][r] += e[t] * a;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < E; ++t)
#pragma unroll
    for (int r = 0; r < R; ++r)
      for (int o = G; o < 32; o <<= 1) acc[t][r] += __shfl_xor_sync(0xffffffffu, acc[t][r], o);
  if (ph == 0 && vl < nvec) {
#pragma unroll
    for (int t = 0; t < E; ++t) {
      const int row = vl * E + t;
      if (row < nr)
#pragma unroll
        for (int r = 0; r < R; ++r) part[row * R + r] += acc[t][r];
    }
  }
  __syncwarp();
}

template <class TF, class TN, class TD, int R>
__global__ void __launch_bounds__(MROWS_WARPS * 32) k_rows_multi(
    const int32_t* __restrict__ seg_start, const int64_t* __restrict__ item_ptr,
    const int64_t* __restrict__ near_begin, const RowItem* __restrict__ items, const TF* __restrict__ F,
    const TN* __restrict__ Nt, const double* __restrict__ z, const double* __restrict__ xm,
    const double* __restrict__ diag, const int32_t* __restrict__ perm, const int32_t* __restrict__ gidx, Offs goff,
    TD* __restrict__ dst, const TD* __restrict__ add, TD* __restrict__ yb, Offs yoff,
    const double* __restrict__ yinit, int near_only) {
  __shared__ double part[MROWS_WARPS][MSEG * R];
  const int sgm = blockIdx.x;
  const int r0 = seg_start[sgm], nr = seg_start[sgm + 1] - r0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = lane; q < MSEG * R; q += 32) part[warp][q] = 0.0;
  __syncwarp();
  const int64_t i0 = item_ptr[sgm], im = near_begin[sgm], i1 = item_ptr[sgm + 1];
  if (!near_only) rows_items_multi<TF, R>(items, i0 + warp, im, F, z, nr, part[warp], lane);
  rows_items_multi<TN, R>(items, im + warp, i1, Nt, xm, nr, part[warp], lane);
  __syncthreads();
  for (int q = threadIdx.x; q < nr * R; q += blockDim.x) {
    const int row = q / R, r = q - row * R;
    const int64_t i = r0 + row;
    double y = diag[i] * xm[i * R + r];
    if (yinit) y += yinit[i * R + r];  // the far field from the tensor-core path
#pragma unroll
    for (int w = 0; w < MROWS_WARPS; ++w) y += part[w][row * R + r];
    const int32_t b = perm[i];
    const int64_t o = gidx ? static_cast<int64_t>(gidx[goff.v[r] + b]) : goff.v[r] + b;
    const TD yv = static_cast<TD>(y);
    dst[o] = add ? static_cast<TD>(add[o] + yv) : yv;
    if (yb) yb[yoff.v[r] + b] = yv;
  }
}

// Near field of 8 states for the tensor-core path (whose far part arrives in yinit): one CTA
// of 64 threads per row segment (<= 64 rows; leaf near blocks, staged 64 columns at a time).
// Each near tile (nc x ld elements: column q of the block is ld consecutive entries) and its
// nc x 8 states go to shared memory by cp.async (16-byte copies), double-buffered so that the
// next item's copies are in flight while the current one is summed.  Thread t sums rows
// 2 (t / 2), 2 (t / 2) + 1 for states 4 (t % 2) .. + 3 (eight FP64 accumulators, one float2 and
// two double2 shared-memory loads per column), then adds the diagonal and the far part and
// scatters like k_rows_multi.
constexpr int NEAR_THREADS = 64;
constexpr int NEAR_COLS = 64;                      // columns staged per round
template <class TN>
struct NearStage {
  static constexpr int TILE = NEAR_COLS * MSEG;    // elements of a staged tile
  static constexpr int XOFF = TILE * sizeof(TN);   // byte offset of the staged states
  static constexpr int BYTES = XOFF + NEAR_COLS * 8 * sizeof(double);
};

__device__ __forceinline__ void cp16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <class TN>
__device__ __forceinline__ void near_pair(const TN* t, double& a0, double& a1);
template <>
__device__ __forceinline__ void near_pair<float>(const float* t, double& a0, double& a1) {
  const float2 v = *reinterpret_cast<const float2*>(t);
  a0 = v.x;
  a1 = v.y;
}
template <>
__device__ __forceinline__ void near_pair<double>(const double* t, double& a0, double& a1) {
  const double2 v = *reinterpret_cast<const double2*>(t);
  a0 = v.x;
  a1 = v.y;
}

template <class TN, class TD>
__global__ void __launch_bounds__(NEAR_THREADS) k_near_multi(
    const int32_t* __restrict__ seg_start, const int64_t* __restrict__ item_ptr,
    const int64_t* __restrict__ near_begin, const RowItem* __restrict__ items, const TN* __restrict__ Nt,
    const double* __restrict__ xm, const double* __restrict__ diag, const int32_t* __restrict__ perm,
    const int32_t* __restrict__ gidx, Offs goff, TD* __restrict__ dst, const TD* __restrict__ add,
    TD* __restrict__ yb, Offs yoff, const double* __restrict__ yinit) {
  constexpr int R = 8;
  constexpr int E = W16<TN>::E;
  using S = NearStage<TN>;
  extern __shared__ __align__(16) char near_smem[];
  const int sgm = blockIdx.x;
  const int r0 = seg_start[sgm], nr = seg_start[sgm + 1] - r0;
  const int ld = (nr + E - 1) / E * E;
  const int tid = threadIdx.x, rp = 2 * (tid >> 1), sq = 4 * (tid & 1);
  const int64_t ib = near_begin[sgm], ie = item_ptr[sgm + 1];
  // issue the copies of (item it, column chunk ch) into buffer buf; returns its column count
  auto issue = [&](int64_t it, int ch, int buf) {
    const RowItem I = items[it];
    const int c0 = ch * NEAR_COLS, nc = min(NEAR_COLS, I.len - c0);
    char* b = near_smem + buf * S::BYTES;
    const int nv = nc * ld * static_cast<int>(sizeof(TN)) / 16;
    const char* src = reinterpret_cast<const char*>(Nt + I.off + static_cast<int64_t>(c0) * ld);
    for (int v = tid; v < nv; v += NEAR_THREADS) cp16(b + 16 * v, src + 16 * static_cast<int64_t>(v));
    const char* xs = reinterpret_cast<const char*>(xm + (static_cast<int64_t>(I.src) + c0) * R);
    for (int v = tid; v < nc * 4; v += NEAR_THREADS) cp16(b + S::XOFF + 16 * v, xs + 16 * static_cast<int64_t>(v));
    cp_commit();
    return nc;
  };
  double acc[2][4];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int s = 0; s < 4; ++s) acc[h][s] = 0.0;
  int64_t it = ib;
  int ch = 0, buf = 0, ncur = 0;
  if (it < ie) ncur = issue(it, 0, 0);
  while (it < ie) {
    // the next unit: the next column chunk of this item, or the next item
    int64_t itn = it;
    int chn = ch + 1;
    if (chn * NEAR_COLS >= items[it].len) {
      ++itn;
      chn = 0;
    }
    cp_wait_all();     // this unit's copies have landed (the only group in flight)
    __syncthreads();   // ... for every thread; and the other buffer is no longer read
    int nnext = 0;
    if (itn < ie) nnext = issue(itn, chn, buf ^ 1);
    const char* b = near_smem + buf * S::BYTES;
    const TN* tl = reinterpret_cast<const TN*>(b);
    const double2* xs = reinterpret_cast<const double2*>(b + S::XOFF);
    if (rp < nr) {
#pragma unroll 4
      for (int q = 0; q < ncur; ++q) {
        double a0, a1;
        near_pair<TN>(tl + q * ld + rp, a0, a1);
        const double2 x01 = xs[q * 4 + sq / 2], x23 = xs[q * 4 + sq / 2 + 1];
        acc[0][0] += a0 * x01.x; acc[0][1] += a0 * x01.y; acc[0][2] += a0 * x23.x; acc[0][3] += a0 * x23.y;
        acc[1][0] += a1 * x01.x; acc[1][1] += a1 * x01.y; acc[1][2] += a1 * x23.x; acc[1][3] += a1 * x23.y;
      }
    }
    buf ^= 1;
    it = itn;
    ch = chn;
    ncur = nnext;
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int row = rp + h;
    if (row >= nr) continue;
    const int64_t i = r0 + row;
    const int32_t b = perm[i];
    const double dg = diag[i];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int r = sq + s;
      const double y = dg * xm[i * R + r] + yinit[i * R + r] + acc[h][s];
      const int64_t o = gidx ? static_cast<int64_t>(gidx[goff.v[r] + b]) : goff.v[r] + b;
      const TD yv = static_cast<TD>(y);
      dst[o] = add ? static_cast<TD>(add[o] + yv) : yv;
      if (yb) yb[yoff.v[r] + b] = yv;
    }
  }
}

template <class TF, class TN, class TS, int R>
void launch_multi(HMatrix& H, const TS* src, const int32_t* gidx, const int64_t* goff, TS* dst, const TS* add,
                  TS* yb, const int64_t* yoff, cudaStream_t s) {
  const int64_t Nb = H.Nb;
  Offs g{}, y{};
  for (int r = 0; r < R; ++r) {
    g.v[r] = goff[r];
    y.v[r] = yoff ? yoff[r] : 0;
  }
  if (H.xmulti.n < static_cast<size_t>(Nb * R)) H.xmulti.alloc(Nb * R);
  if (H.zmulti.n < static_cast<size_t>(std::max<int64_t>(H.zlen, 1) * R)) H.zmulti.alloc(std::max<int64_t>(H.zlen, 1) * R);
  if (H.zpmulti.n < static_cast<size_t>(std::max<int64_t>(H.zpart_len, 1) * R))
    H.zpmulti.alloc(std::max<int64_t>(H.zpart_len, 1) * R);
  k_hgather_multi<TS, R><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, src, gidx, g, H.perm.p, H.xmulti.p);
  SPX_LAUNCH_CHECK();
  if (R == 8 && H.tc) {  // far field on the tensor cores, then near field + diagonal + scatter
    const double* yfar = tc_far_apply(H, H.xmulti.p, s);
    constexpr int smem = 2 * NearStage<TN>::BYTES;
    static_assert(smem <= 160 * 1024, "near-field staging");
    SPX_CUDA(cudaFuncSetAttribute(k_near_multi<TN, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_near_multi<TN, TS><<<static_cast<unsigned>(H.nseg), NEAR_THREADS, smem, s>>>(
        H.seg_start.p, H.item_ptr.p, H.near_begin.p, H.items.p, reinterpret_cast<const TN*>(H.near_f.p),
        H.xmulti.p, H.diag_perm.p, H.perm.p, gidx, g, dst, add, yb, y, yfar);
    SPX_LAUNCH_CHECK();
    return;
  }
  if (H.nunits > 0) {
    const unsigned ctas = static_cast<unsigned>((H.nwarps_z + MZ_WARPS - 1) / MZ_WARPS);
    k_far_z_multi<TF, R><<<ctas, MZ_WARPS * 32, 0, s>>>(H.units.p, H.warp_first.p, static_cast<int>(H.nwarps_z),
                                                         reinterpret_cast<const TF*>(H.far_f.p), H.xmulti.p,
                                                         H.zmulti.p, H.zpmulti.p, H.groups.p, H.gcnt.p);
    SPX_LAUNCH_CHECK();
  }
  k_rows_multi<TF, TN, TS, R><<<static_cast<unsigned>(H.nseg), MROWS_WARPS * 32, 0, s>>>(
      H.seg_start.p, H.item_ptr.p, H.near_begin.p, H.items.p, reinterpret_cast<const TF*>(H.far_f.p),
      reinterpret_cast<const TN*>(H.near_f.p), H.zmulti.p, H.xmulti.p, H.diag_perm.p, H.perm.p, gidx, g, dst, add,
      yb, y, nullptr, 0);
  SPX_LAUNCH_CHECK();
}

template <class TF, class TN, class TS>
void apply_chunks(HMatrix& H, const TS* src, const int32_t* gidx, const int64_t* goff, TS* dst, const TS* add,
                  TS* yb, const int64_t* yoff, int R, cudaStream_t s) {
  int r0 = 0;
  while (r0 < R) {
    const int left = R - r0;
    const int c = left >= 8 ? 8 : left >= 4 ? 4 : left >= 2 ? 2 : 1;
    const int64_t* g = goff + r0;
    const int64_t* y = yoff ? yoff + r0 : nullptr;
    switch (c) {
      case 8: launch_multi<TF, TN, TS, 8>(H, src, gidx, g, dst, add, yb, y, s); break;
      case 4: launch_multi<TF, TN, TS, 4>(H, src, gidx, g, dst, add, yb, y, s); break;
      case 2: launch_multi<TF, TN, TS, 2>(H, src, gidx, g, dst, add, yb, y, s); break;
      default: launch_multi<TF, TN, TS, 1>(H, src, gidx, g, dst, add, yb, y, s); break;
    }
    r0 += c;
  }
}

}  // namespace

template <class T>
void HMatrix::apply_multi(const T* src, const int32_t* gidx, const int64_t* goff, T* dst, const T* add, T* yb,
                          const int64_t* yoff, int R, cudaStream_t s) {
  SPX_CHECK(packed, "H-matrix is not packed");
  SPX_CHECK(R >= 1, "at least one right-hand side");
  switch (prec) {
    case Prec::F64: apply_chunks<double, double, T>(*this, src, gidx, goff, dst, add, yb, yoff, R, s); break;
    case Prec::F32: apply_chunks<float, float, T>(*this, src, gidx, goff, dst, add, yb, yoff, R, s); break;
    case Prec::MIXED: apply_chunks<__nv_bfloat16, float, T>(*this, src, gidx, goff, dst, add, yb, yoff, R, s); break;
    case Prec::SPLIT: {  // batches of 8 on the tensor cores when enabled, the rest one at a time
      SPX_CHECK(yb == nullptr || yoff != nullptr, "state outputs need offsets");
      int r = 0;
      if (tc)
        for (; r + 8 <= R; r += 8)
          launch_multi<float, float, T, 8>(*this, src, gidx, goff + r, dst, add, yb, yoff ? yoff + r : nullptr, s);
      for (; r < R; ++r) {
        T* y = yb ? yb + yoff[r] : nullptr;
        if (gidx) apply_gather<T>(src, gidx + goff[r], dst, add, y, s);
        else apply_gather<T>(src + goff[r], nullptr, dst + goff[r], add ? add + goff[r] : nullptr, y, s);
      }
      break;
    }
  }
}
template void HMatrix::apply_multi<double>(const double*, const int32_t*, const int64_t*, double*, const double*,
                                           double*, const int64_t*, int, cudaStream_t);
template void HMatrix::apply_multi<float>(const float*, const int32_t*, const int64_t*, float*, const float*, float*,
                                          const int64_t*, int, cudaStream_t);

}  // namespace spx
