// Far-field products of the multi-state H-matrix apply on the 5th-generation tensor cores.
//
// For R = 8 states of one boundary, the far field of Y = H X is two block-sparse GEMMs:
//   phase 1 (column clusters): for every column cluster tau, the V factors of all far blocks
//     with columns tau, stacked (M = sum of their ranks), times X~[tau] (K = |tau|, N = 8):
//     the z vectors of those blocks;
//   phase 2 (row clusters): for every row cluster sigma, [U_b1 U_b2 ...] (M = |sigma|, K = sum of
//     the blocks' ranks) times the stacked z (N = 8): their share of Y[sigma].
// Both run through one kernel, k_tc_gemm, over a list of tiles of 128 rows: A (the factor
// rows of the tile) is packed once in the canonical K-major no-swizzle shared-memory layout of
// tcgen05 (8 x 16-byte core matrices; per K-step of 8 elements 4 KB), so each stage of 4
// K-steps is one 16 KB cp.async.bulk copy; B (X~ or z for the tile's K range) is gathered by
// CUDA cores.  The products use kind::tf32 with a three-term split (A_hi B_hi + A_hi B_lo +
// A_lo B_hi, hi = the TF32 truncation, lo = the FP32 remainder): about 22 bits of A and B,
// close to the FP32 factors' own precision.  Accumulation is FP32 in tensor memory over at most
// 2048 K elements per tile; the tiles' FP32 partials are summed in FP64 (k_tc_reduce) into z
// (phase 1, per z entry over its column chunks) and into the far part of Y (phase 2, per row
// over the row clusters that contain it).  The near field, the diagonal and the scatter stay
// on k_rows_multi (hmat_multi.cu), which adds this far part.
//
// Warp roles of k_tc_gemm (384 threads, one CTA per SM, persistent over a tile list):
//   warp 0   : cp.async.bulk of A stages into a 4-stage ring (mbarrier transaction counts);
//   warp 1   : one thread issues tcgen05.mma (3 per K-step) and tcgen05.commit;
//   warp 2   : allocates / frees 32 tensor-memory columns (two 128 x 16 FP32 accumulators, of
//              which the first 8 columns are the states; B's rows 8-15 are zero);
//   warps 4-7: epilogue, tcgen05.ld of the accumulator (lanes 32 (w % 4) .. + 31) to partials;
//   warps 8-11: split A into hi / lo in place, gather and split B, fence.proxy.async.
// Every mbarrier wait is bounded; on a timeout the kernel records SPX_ERR_TIMEOUT, the roles
// stop, the MMA issuer waits (bounded) for its last commit, and tensor memory is freed.
//
// No TMA tensor maps and no cluster multicast: A copies are plain 1-D bulk copies from this
// GPU's own memory.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "hmat.cuh"

namespace spx {

struct TcTile {
  int64_t a_off;   // bytes: packed A of nsteps K-steps
  int32_t nsteps;  // K-steps of 8
  int32_t b_row0;  // first row of the B source vector for K index 0
  int32_t b_rows;  // valid K rows (B is zero past them)
  int32_t slot;    // output partial: rows slot * 128 .. + 127
};

struct TcPack {
  int64_t a_off;
  int64_t tab;     // phase 1: rowbase index of row 0; phase 2: colbase index of k = 0
  int64_t roff;    // phase 1: column offset added to rowbase; phase 2: row offset in the cluster
  int32_t nsteps, kvalid, rvalid, mode;
};

struct TcPlan {
  int64_t zlen = 0, nslots1 = 0, nslots2 = 0, a_bytes = 0;
  int kstep_max = 0;
  DevBuf<char> A1, A2;                 // packed A of the two phases
  DevBuf<TcTile> t1, t2;
  int32_t nt1 = 0, nt2 = 0;
  DevBuf<int64_t> rp1, rp2;            // CSR: z entry / perm row -> partial rows
  DevBuf<int32_t> ix1, ix2;
  DevBuf<float> part1, part2;          // [slots * 128][8]
  DevBuf<double> z, yfar;              // [zlen][8], [Nb][8]
  DevBuf<int> err;
};

namespace tc {

constexpr int R = 8;
constexpr int TM = 128;
constexpr int STEP_BYTES = TM * 8 * 4;  // 4096: 128 rows x 8 TF32
constexpr int STAGE_STEPS = 4;
constexpr int NSTAGE = 4;
constexpr int STAGE_BYTES = STAGE_STEPS * STEP_BYTES;
constexpr int NB = 16;                  // MMA N: M = 128 takes N in multiples of 16, so the
                                        // 8 states are padded with 8 zero rows of B
constexpr int BSTEP_BYTES = NB * 8 * 4;  // 512: 16 rows x 8 TF32
constexpr int KSTEP_MAX_DEFAULT = 256;  // K-steps per tile (2048 elements); the autotuner also tries 64
constexpr int THREADS = 384;
// + a 32 KB guard after the buffers, so that no descriptor-addressed read can leave the
// allocation even past the last stage
constexpr int SMEM_BYTES = 2 * NSTAGE * STAGE_BYTES + 2 * NSTAGE * STAGE_STEPS * BSTEP_BYTES + 1024 + 256 + 32768;
constexpr long long WAIT_LIMIT = 1ll << 22;  // polls of try_wait before a wait gives up

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}
// bounded wait until the phase of parity `par` has completed
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t par) {
  for (long long it = 0; it < WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(par)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   su32(dst)),
               "l"(src), "r"(bytes), "r"(su32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle; lbo / sbo in bytes
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;  // descriptor version of sm_100
  return d;                             // base offset 0, no swizzle
}
// instruction descriptor: D F32, A and B TF32, both K-major, N = 16, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((static_cast<uint32_t>(NB) >> 3) << 17) |
                           ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(
          d),
      "l"(a), "l"(b), "r"(IDESC), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_trunc(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// B (16 rows x 8 K; rows 8-15 stay zero) of one K-step, K-major core-matrix layout: K chunk
// c = k / 4 at c * 256 bytes, row group n / 8 at 128, row n % 8 at 16, element k % 4 at 4
__device__ __forceinline__ int boff(int n, int k) { return (k >> 2) * 256 + (n >> 3) * 128 + (n & 7) * 16 + (k & 3) * 4; }

__global__ void __launch_bounds__(THREADS, 1)
    k_tc_gemm(const TcTile* __restrict__ tiles, int ntiles, const char* __restrict__ A,
              const double* __restrict__ bsrc, float* __restrict__ part, int* __restrict__ err) {
  extern __shared__ __align__(1024) char smem[];
  char* sA = smem;                                         // [NSTAGE][STAGE_BYTES]
  char* sAlo = sA + NSTAGE * STAGE_BYTES;                  // [NSTAGE][STAGE_BYTES]
  char* sBhi = sAlo + NSTAGE * STAGE_BYTES;                // [NSTAGE][STAGE_STEPS][256]
  char* sBlo = sBhi + NSTAGE * STAGE_STEPS * BSTEP_BYTES;  // [NSTAGE][STAGE_STEPS][256]
  uint64_t* bars = reinterpret_cast<uint64_t*>(sBlo + NSTAGE * STAGE_STEPS * BSTEP_BYTES);
  uint64_t* full = bars;              // [NSTAGE] A copied
  uint64_t* ready = bars + NSTAGE;    // [NSTAGE] A split, B staged
  uint64_t* empty = bars + 2 * NSTAGE;  // [NSTAGE] MMAs done with the stage
  uint64_t* accf = bars + 3 * NSTAGE;   // [2] accumulator complete
  uint64_t* acce = bars + 3 * NSTAGE + 2;  // [2] accumulator read
  uint64_t* fin = bars + 3 * NSTAGE + 4;   // last MMAs done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 3 * NSTAGE + 6);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&ready[s], 128);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 128);
    }
    mbar_init(fin, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  for (int e = tid; e < 2 * NSTAGE * STAGE_STEPS * BSTEP_BYTES / 16; e += THREADS)
    reinterpret_cast<float4*>(sBhi)[e] = make_float4(0.f, 0.f, 0.f, 0.f);  // B hi and lo (contiguous)
  fence_proxy_async();
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)), "r"(32)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tbase = *tslot;

  auto fail = [&]() {
    *abort_flag = 1;
    atomicExch(err, ERR_TIMEOUT);
  };

  if (warp == 0) {
    if (lane == 0) {  // producer
      int item = 0;
      for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x) {
        const TcTile T = tiles[t];
        for (int s0 = 0; s0 < T.nsteps; s0 += STAGE_STEPS, ++item) {
          const int st = item % NSTAGE, rnd = item / NSTAGE;
          if (!mbar_wait(&empty[st], (rnd & 1) ^ 1)) { fail(); break; }
          const int ns = min(STAGE_STEPS, T.nsteps - s0);
          const uint32_t bytes = static_cast<uint32_t>(ns * STEP_BYTES);
          mbar_expect_tx(&full[st], bytes);
          bulk_g2s(sA + st * STAGE_BYTES, A + T.a_off + static_cast<int64_t>(s0) * STEP_BYTES, bytes, &full[st]);
        }
      }
      // leave no copy in flight: the last stages' copies have landed (bounded)
      for (int q = max(0, item - NSTAGE); q < item; ++q) mbar_wait(&full[q % NSTAGE], (q / NSTAGE) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      int item = 0, tc = 0;
      bool issued = false;
      for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x, ++tc) {
        const TcTile T = tiles[t];
        const int buf = tc & 1, use = tc >> 1;
        if (!mbar_wait(&acce[buf], (use & 1) ^ 1)) { fail(); break; }
        tc_after();
        const uint32_t d = tbase + static_cast<uint32_t>(buf * NB);
        uint32_t acc = 0;
        bool ok = true;
        for (int s0 = 0; s0 < T.nsteps; s0 += STAGE_STEPS, ++item) {
          const int st = item % NSTAGE, rnd = item / NSTAGE;
          if (!mbar_wait(&ready[st], rnd & 1)) { fail(); ok = false; break; }
          tc_after();
          const int ns = min(STAGE_STEPS, T.nsteps - s0);
          for (int k = 0; k < ns; ++k) {
            const uint32_t a = su32(sA + st * STAGE_BYTES + k * STEP_BYTES);
            const uint32_t al = su32(sAlo + st * STAGE_BYTES + k * STEP_BYTES);
            const uint32_t bh = su32(sBhi + (st * STAGE_STEPS + k) * BSTEP_BYTES);
            const uint32_t bl = su32(sBlo + (st * STAGE_STEPS + k) * BSTEP_BYTES);
            const uint64_t da = sdesc(a, 2048, 128), dal = sdesc(al, 2048, 128);
            const uint64_t dbh = sdesc(bh, 256, 128), dbl = sdesc(bl, 256, 128);
            mma_tf32(d, da, dbh, acc);
            acc = 1;
            mma_tf32(d, da, dbl, 1);
            mma_tf32(d, dal, dbh, 1);
          }
          mma_commit(&empty[st]);
          issued = true;
        }
        if (!ok) break;
        mma_commit(&accf[buf]);
      }
      if (issued) {  // every MMA of this CTA has completed before tensor memory is freed
        mma_commit(fin);
        mbar_wait(fin, 0);
      }
    }
  } else if (warp >= 4 && warp < 8) {  // epilogue: TMEM lanes 32 (warp % 4) .. + 31
    const int sp = warp & 3;
    int tc = 0;
    for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x, ++tc) {
      const TcTile T = tiles[t];
      const int buf = tc & 1, use = tc >> 1;
      if (!mbar_wait(&accf[buf], use & 1)) { fail(); break; }
      tc_after();
      uint32_t v[8];
      tmem_ld8(tbase + (static_cast<uint32_t>(32 * sp) << 16) + static_cast<uint32_t>(buf * NB), v);
      tc_before();
      mbar_arrive(&acce[buf]);
      const int row = 32 * sp + lane;
      float4* o = reinterpret_cast<float4*>(part + (static_cast<int64_t>(T.slot) * TM + row) * R);
      o[0] = make_float4(__uint_as_float(v[0]), __uint_as_float(v[1]), __uint_as_float(v[2]), __uint_as_float(v[3]));
      o[1] = make_float4(__uint_as_float(v[4]), __uint_as_float(v[5]), __uint_as_float(v[6]), __uint_as_float(v[7]));
    }
  } else if (warp >= 8) {  // converter: A split in place, B gathered and split
    const int ct = tid - 256;
    int item = 0;
    for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x) {
      const TcTile T = tiles[t];
      bool ok = true;
      for (int s0 = 0; s0 < T.nsteps; s0 += STAGE_STEPS, ++item) {
        const int st = item % NSTAGE, rnd = item / NSTAGE;
        const int ns = min(STAGE_STEPS, T.nsteps - s0);
        // the stage's copy has landed, so its previous MMAs are done and B / A_lo are free
        if (!mbar_wait(&full[st], rnd & 1)) { fail(); ok = false; break; }
        for (int e = ct; e < ns * 64; e += 128) {
          const int k8 = e >> 6, idx = e & 63, n = idx >> 3, j = idx & 7;
          const int kk = (s0 + k8) * 8 + j;
          const double x = kk < T.b_rows ? bsrc[(static_cast<int64_t>(T.b_row0) + kk) * R + n] : 0.0;
          const float hi = tf32_trunc(static_cast<float>(x));
          const float lo = static_cast<float>(x - static_cast<double>(hi));
          const int o = (st * STAGE_STEPS + k8) * BSTEP_BYTES + boff(n, j);
          *reinterpret_cast<float*>(sBhi + o) = hi;
          *reinterpret_cast<float*>(sBlo + o) = lo;
        }
        float4* a4 = reinterpret_cast<float4*>(sA + st * STAGE_BYTES);
        float4* l4 = reinterpret_cast<float4*>(sAlo + st * STAGE_BYTES);
        for (int e = ct; e < ns * (STEP_BYTES / 16); e += 128) {
          const float4 v = a4[e];
          const float4 h = make_float4(tf32_trunc(v.x), tf32_trunc(v.y), tf32_trunc(v.z), tf32_trunc(v.w));
          a4[e] = h;
          l4[e] = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
        }
        fence_proxy_async();
        mbar_arrive(&ready[st]);
      }
      if (!ok) break;
    }
  }
  tc_before();
  __syncthreads();
  tc_after();
  if (warp == 2) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(32) : "memory");
}

// out[i][n] = sum over p in [rp[i], rp[i+1]) of part[ix[p]][n]  (FP64, fixed order)
__global__ void k_tc_reduce(int64_t nrows, const int64_t* __restrict__ rp, const int32_t* __restrict__ ix,
                            const float* __restrict__ part, double* __restrict__ out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i = t >> 3;
  const int n = static_cast<int>(t & 7);
  if (i >= nrows) return;
  double s = 0.0;
  for (int64_t p = rp[i]; p < rp[i + 1]; ++p) s += static_cast<double>(part[static_cast<int64_t>(ix[p]) * R + n]);
  out[i * R + n] = s;
}

// packed A of one (tile, K-step): 128 rows x 8 TF32 in the core-matrix layout
// (row r, k): (k / 4) * 2048 + (r / 8) * 128 + (r % 8) * 16 + (k % 4) * 4 bytes
__global__ void k_tc_pack(const TcPack* __restrict__ jobs, int njobs, const double* __restrict__ pool,
                          const int64_t* __restrict__ rowbase, const int64_t* __restrict__ colbase,
                          char* __restrict__ A) {
  const TcPack J = jobs[blockIdx.y];
  for (int s = blockIdx.x; s < J.nsteps; s += gridDim.x) {
    float* dst = reinterpret_cast<float*>(A + J.a_off + static_cast<int64_t>(s) * STEP_BYTES);
    for (int e = threadIdx.x; e < TM * 8; e += blockDim.x) {
      const int r = e >> 3, j = e & 7;
      const int k = s * 8 + j;
      double v = 0.0;
      if (r < J.rvalid && k < J.kvalid) {
        if (J.mode == 1) {
          const int64_t b = rowbase[J.tab + r];
          if (b >= 0) v = pool[b + J.roff + k];
        } else {
          const int64_t b = colbase[J.tab + k];
          if (b >= 0) v = pool[b + J.roff + r];
        }
      }
      dst[((j >> 2) * 2048 + (r >> 3) * 128 + (r & 7) * 16 + (j & 3) * 4) >> 2] = static_cast<float>(v);
    }
  }
}

}  // namespace tc

// ------------------------------------------------------------------ host: plan and apply
namespace {

struct Csr {
  std::vector<int64_t> rp;
  std::vector<int32_t> ix;
};

Csr make_csr(int64_t nrows, const std::vector<std::pair<int64_t, int32_t>>& pairs) {
  Csr c;
  c.rp.assign(nrows + 1, 0);
  for (auto& p : pairs) c.rp[p.first + 1]++;
  for (int64_t i = 0; i < nrows; ++i) c.rp[i + 1] += c.rp[i];
  c.ix.resize(pairs.size());
  std::vector<int64_t> cur(c.rp.begin(), c.rp.end() - 1);
  for (auto& p : pairs) c.ix[cur[p.first]++] = p.second;
  return c;
}

}  // namespace

void tc_build(HMatrix& H, cudaStream_t s, int kstep_max) {
  using namespace tc;
  // K-steps of 8 per tile (FP32 accumulation in tensor memory runs over at most 8 x this many
  // products; the tiles' partials are summed in FP64).  SPX_TC_KSTEP sets it for tuning.
  int KSTEP_MAX = kstep_max > 0 ? kstep_max : KSTEP_MAX_DEFAULT;
  if (kstep_max <= 0)
    if (const char* e = std::getenv("SPX_TC_KSTEP")) KSTEP_MAX = std::max(1, std::atoi(e));
  SPX_CHECK(H.far_pool64.n > 0 || H.stats.n_far == 0, "the tensor-core apply needs the FP64 factors");
  auto P = std::make_shared<TcPlan>();
  std::vector<int> far;
  for (size_t i = 0; i < H.blocks.size(); ++i)
    if (H.blocks[i].type == 1 && H.blocks[i].rank > 0) far.push_back(static_cast<int>(i));
  // z layout of the tensor-core path: blocks grouped by row cluster, ranks padded to 8
  std::vector<std::pair<int64_t, int64_t>> rkeys;
  std::vector<std::vector<int>> rgroups;
  {
    std::vector<std::pair<std::pair<int64_t, int64_t>, int>> tmp;
    for (int b : far) tmp.push_back({{H.blocks[b].rs, H.blocks[b].re}, b});
    std::stable_sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (auto& t : tmp) {
      if (rkeys.empty() || rkeys.back() != t.first) {
        rkeys.push_back(t.first);
        rgroups.emplace_back();
      }
      rgroups.back().push_back(t.second);
    }
  }
  std::vector<int64_t> zoff(H.blocks.size(), -1);
  int64_t zlen = 0;
  for (auto& g : rgroups)
    for (int b : g) {
      zoff[b] = zlen;
      zlen += (H.blocks[b].rank + 7) / 8 * 8;
    }
  P->zlen = zlen;
  std::vector<TcTile> t1, t2;
  std::vector<TcPack> p1, p2;
  std::vector<int64_t> rowbase, colbase;
  std::vector<std::pair<int64_t, int32_t>> m1, m2;
  int64_t a1 = 0, a2 = 0;
  int32_t slot1 = 0, slot2 = 0;
  // phase 1: column clusters
  {
    std::vector<std::pair<std::pair<int64_t, int64_t>, int>> tmp;
    for (int b : far) tmp.push_back({{H.blocks[b].cs, H.blocks[b].ce}, b});
    std::stable_sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    size_t u = 0;
    while (u < tmp.size()) {
      size_t e = u;
      while (e < tmp.size() && tmp[e].first == tmp[u].first) ++e;
      const int64_t cs = tmp[u].first.first, K = tmp[u].first.second - cs;
      std::vector<std::pair<int64_t, int64_t>> rows;  // (pool base of V row q, z entry)
      for (size_t v = u; v < e; ++v) {
        const HBlock& B = H.blocks[tmp[v].second];
        const int64_t n = B.ce - B.cs;
        for (int q = 0; q < B.rank; ++q) rows.push_back({B.off_v + q * n, zoff[tmp[v].second] + q});
      }
      const int64_t ksteps = (K + 7) / 8;
      for (int64_t m0 = 0; m0 < static_cast<int64_t>(rows.size()); m0 += TM) {
        const int64_t tab = static_cast<int64_t>(rowbase.size());
        const int rv = static_cast<int>(std::min<int64_t>(TM, rows.size() - m0));
        for (int r = 0; r < TM; ++r) rowbase.push_back(r < rv ? rows[m0 + r].first : -1);
        for (int64_t k0 = 0; k0 < ksteps; k0 += KSTEP_MAX) {
          const int ns = static_cast<int>(std::min<int64_t>(KSTEP_MAX, ksteps - k0));
          const int kv = static_cast<int>(std::min<int64_t>(8 * ns, K - 8 * k0));
          t1.push_back(TcTile{a1, ns, static_cast<int32_t>(cs + 8 * k0), kv, slot1});
          p1.push_back(TcPack{a1, tab, 8 * k0, ns, kv, rv, 1});
          for (int r = 0; r < rv; ++r) m1.push_back({rows[m0 + r].second, slot1 * TM + r});
          a1 += static_cast<int64_t>(ns) * STEP_BYTES;
          ++slot1;
        }
      }
      u = e;
    }
  }
  // phase 2: row clusters
  for (size_t g = 0; g < rgroups.size(); ++g) {
    const int64_t rs = rkeys[g].first, rows = rkeys[g].second - rs;
    const int64_t kb = static_cast<int64_t>(colbase.size());
    int64_t K = 0;
    for (int b : rgroups[g]) {
      const HBlock& B = H.blocks[b];
      const int64_t m = B.re - B.rs;
      const int k8 = (B.rank + 7) / 8 * 8;
      for (int q = 0; q < k8; ++q) colbase.push_back(q < B.rank ? B.off_u + q * m : -1);
      K += k8;
    }
    const int64_t z0 = zoff[rgroups[g][0]];
    const int64_t ksteps = K / 8;
    for (int64_t m0 = 0; m0 < rows; m0 += TM) {
      const int rv = static_cast<int>(std::min<int64_t>(TM, rows - m0));
      for (int64_t k0 = 0; k0 < ksteps; k0 += KSTEP_MAX) {
        const int ns = static_cast<int>(std::min<int64_t>(KSTEP_MAX, ksteps - k0));
        const int kv = 8 * ns;
        t2.push_back(TcTile{a2, ns, static_cast<int32_t>(z0 + 8 * k0), kv, slot2});
        p2.push_back(TcPack{a2, kb + 8 * k0, m0, ns, kv, rv, 2});
        for (int r = 0; r < rv; ++r) m2.push_back({rs + m0 + r, slot2 * TM + r});
        a2 += static_cast<int64_t>(ns) * STEP_BYTES;
        ++slot2;
      }
    }
  }
  SPX_CHECK(zlen < (int64_t(1) << 31) && slot1 < (1 << 24) && slot2 < (1 << 24), "tensor-core plan too large");
  // larger tiles first, dealt round-robin to the CTAs
  auto sort_tiles = [](std::vector<TcTile>& t) {
    std::stable_sort(t.begin(), t.end(), [](const TcTile& a, const TcTile& b) { return a.nsteps > b.nsteps; });
  };
  sort_tiles(t1);
  sort_tiles(t2);
  P->nt1 = static_cast<int32_t>(t1.size());
  P->nt2 = static_cast<int32_t>(t2.size());
  P->nslots1 = slot1;
  P->nslots2 = slot2;
  P->a_bytes = a1 + a2;
  P->kstep_max = KSTEP_MAX;
  P->A1.alloc(std::max<int64_t>(a1, 16));
  P->A2.alloc(std::max<int64_t>(a2, 16));
  P->t1.upload(t1, s);
  P->t2.upload(t2, s);
  {
    DevBuf<int64_t> drb, dcb;
    drb.upload(rowbase.empty() ? std::vector<int64_t>{-1} : rowbase, s);
    dcb.upload(colbase.empty() ? std::vector<int64_t>{-1} : colbase, s);
    auto run = [&](const std::vector<TcPack>& jobs, char* dst) {
      for (size_t j0 = 0; j0 < jobs.size(); j0 += 65535) {
        const size_t c = std::min<size_t>(65535, jobs.size() - j0);
        DevBuf<TcPack> dj;
        dj.upload(jobs.data() + j0, c, s);
        k_tc_pack<<<dim3(32, static_cast<unsigned>(c)), 256, 0, s>>>(dj.p, static_cast<int>(c), H.far_pool64.p,
                                                                     drb.p, dcb.p, dst);
        SPX_LAUNCH_CHECK();
        SPX_CUDA(cudaStreamSynchronize(s));
      }
    };
    run(p1, P->A1.p);
    run(p2, P->A2.p);
  }
  Csr c1 = make_csr(zlen, m1), c2 = make_csr(H.Nb, m2);
  P->rp1.upload(c1.rp, s);
  P->ix1.upload(c1.ix.empty() ? std::vector<int32_t>{0} : c1.ix, s);
  P->rp2.upload(c2.rp, s);
  P->ix2.upload(c2.ix.empty() ? std::vector<int32_t>{0} : c2.ix, s);
  P->part1.alloc(std::max<int64_t>(slot1, 1) * TM * R);
  P->part2.alloc(std::max<int64_t>(slot2, 1) * TM * R);
  P->z.alloc(std::max<int64_t>(zlen, 1) * R);
  P->yfar.alloc(H.Nb * R);
  P->err.alloc(1);
  P->err.zero(s);
  SPX_CUDA(cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
  SPX_CUDA(cudaStreamSynchronize(s));
  H.tc = P;
}

// far part of Y (perm order, FP64 [Nb][8]) from the gathered X~ ([Nb][8]); returns yfar
const double* tc_far_apply(HMatrix& H, const double* xm, cudaStream_t s) {
  using namespace tc;
  TcPlan& P = *H.tc;
  const int grid = num_sms(H.device);
  if (P.nt1 > 0) {
    k_tc_gemm<<<grid, THREADS, SMEM_BYTES, s>>>(P.t1.p, P.nt1, P.A1.p, xm, P.part1.p, P.err.p);
    SPX_LAUNCH_CHECK();
  }
  if (P.zlen > 0) {
    k_tc_reduce<<<grid_for(P.zlen * R, 256), 256, 0, s>>>(P.zlen, P.rp1.p, P.ix1.p, P.part1.p, P.z.p);
    SPX_LAUNCH_CHECK();
  }
  if (P.nt2 > 0) {
    k_tc_gemm<<<grid, THREADS, SMEM_BYTES, s>>>(P.t2.p, P.nt2, P.A2.p, P.z.p, P.part2.p, P.err.p);
    SPX_LAUNCH_CHECK();
  }
  k_tc_reduce<<<grid_for(H.Nb * R, 256), 256, 0, s>>>(H.Nb, P.rp2.p, P.ix2.p, P.part2.p, P.yfar.p);
  SPX_LAUNCH_CHECK();
  return P.yfar.p;
}

int tc_error(HMatrix& H, cudaStream_t s) {
  if (!H.tc) return 0;
  int e = 0;
  SPX_CUDA(cudaMemcpyAsync(&e, H.tc->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  return e;
}

int64_t tc_bytes(const HMatrix& H) {
  if (!H.tc) return 0;
  const TcPlan& P = *H.tc;
  return static_cast<int64_t>(P.A1.bytes() + P.A2.bytes() + P.part1.bytes() + P.part2.bytes() + P.z.bytes() +
                              P.yfar.bytes() + P.rp1.bytes() + P.rp2.bytes() + P.ix1.bytes() + P.ix2.bytes());
}

}  // namespace spx
