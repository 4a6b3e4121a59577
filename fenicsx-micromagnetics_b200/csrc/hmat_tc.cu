// Far-field products of the multi-state H-matrix apply on the 5th-generation tensor cores,
// with exact integer products (the Ozaki scheme on tcgen05 kind::i8).
//
// For R = 8 states of one boundary, the far field of Y = H X is two block-sparse GEMMs:
//   phase 1 (column clusters): for every column cluster tau, the V factors of all far blocks
//     with columns tau, stacked (M = sum of their ranks), times X~[tau] (K = |tau|, N = 8):
//     the z vectors of those blocks;
//   phase 2 (row clusters): for every row cluster sigma, [U_b1 U_b2 ...] (M = |sigma|, K = sum of
//     the blocks' ranks) times the stacked z (N = 8): their share of Y[sigma].
// Both run through one kernel, k_tc_gemm, over a list of tiles of 128 rows and at most 2048 K
// elements.
//
// Arithmetic.  The thin film's double-layer potential is a small difference of large surface
// contributions, so the far field needs FP64-class products: TF32 operands with FP32 tile sums
// are 100x too coarse for a 1e-5 demag error.  Instead every operand is a fixed-point integer
// cut into balanced base-256 digits (int8 in [-128, 127]):
//   A element  a = 2^(e_r - 31) sum_{t<4} d_t 256^(3 - t),  e_r from the largest |a| of the tile
//              row (|a| < 2^(e_r - 1)); a is the FP32 factor, exact whenever |a| >= 2^(e_r - 8);
//   B element  b = 2^(f_n - 47) sum_{u<6} c_u 256^(5 - u),  f_n from the largest |b| of state n
//              over the B rows of the cluster (or row group).
// sum_k a_k b_k = 2^(e_r + f_n - 78) sum_{t,u} 256^(8 - t - u) D_tu with D_tu = sum_k d_tk c_uk an
// exact int32 sum (|d c| <= 2^14, K <= 8192 per tile: |D| <= 2^27).  No digit pair is dropped.
// The six digits of every B element sit side by side in the MMA's N dimension (column
// 8 u + n), so ONE MMA of N = 48 per A digit computes all 24 digit pairs of a K step: four
// MMAs (M = 128, N = 48, K = 32) per stage into four int32 accumulators D_t in tensor memory.
// The A digits are cut once, when the plan is built, into the MMA's shared-memory layout: a
// stage is 16 KB in HBM (4 digits x 128 rows x 32 K), the same 4 bytes per factor element as
// the FP32 packing, and goes to shared memory by one bulk copy with no conversion.  Only the
// B rows (X~ or z, FP64) of a stage (8 states x 32 K) are cut at run time.  The epilogue forms
// the FP64 value of each tile row; tile partials are summed in FP64 (k_tc_reduce) into z
// (phase 1) and into the far part of Y (phase 2).  The near field, the diagonal and the scatter
// stay on k_rows_multi (hmat_multi.cu), which adds this far part.
//
// Data path of k_tc_gemm (384 threads, one CTA per SM, persistent over a tile list): an
// 8-stage ring; a stage is the A digits (16 KB) and the stage's B rows (FP64, up to 2 KB), both
// brought by cp.async.bulk onto one mbarrier (transaction counts), and the B digit tile.  Every
// role loads the next tile's descriptor (and exponents) while it works on the current one.
//   warp 0     : cp.async.bulk of the A digits and the B rows;
//   warp 1     : MMA issuer (4 MMAs per stage, tcgen05.commit);
//   warp 2     : allocates / frees 512 tensor-memory columns (two buffers of 4 x 48 int32);
//   warps 4-7  : epilogue (TMEM lanes 32 (w % 4) .. + 31) to FP64 partials;
//   warps 8-11 : cut the B rows of each stage (from shared memory) into digits (canonical
//                K-major layout).
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
  int64_t a_off;   // bytes: A digits of nsteps stages
  int32_t nsteps;  // stages of 32 K elements
  int32_t b_row0;  // first row of the B source for K index 0
  int32_t b_rows;  // valid K rows (B is zero past them)
  int32_t slot;    // output partial: rows slot * 128 .. + 127
  int32_t bsc;     // row of the B exponent table (column cluster or row group)
  int32_t direct;  // 1: the tile covers its rows' whole K range; the epilogue writes the
                   // result rows straight to `zout` (rows mapped by zmap), not to partials
};

struct TcPack {
  int64_t a_off;
  int64_t tab;     // phase 1: rowbase index of row 0; phase 2: colbase index of k = 0
  int64_t roff;    // phase 1: column offset added to rowbase; phase 2: row offset in the cluster
  int32_t nsteps, kvalid, rvalid, mode;
  int32_t slot, pad;
};

struct TcPlan {
  int64_t zlen = 0, nslots1 = 0, nslots2 = 0, a_bytes = 0;
  int kstep_max = 0;
  DevBuf<char> A1, A2;                 // A digits of the two phases, stage by stage
  DevBuf<int32_t> ea1, ea2;            // A row exponents per slot [slots][128]
  DevBuf<TcTile> t1, t2;
  int32_t nt1 = 0, nt2 = 0;
  DevBuf<int64_t> rp1, rp2;            // CSR: z entry / perm row -> partial rows
  DevBuf<int32_t> ix1, ix2;
  DevBuf<int64_t> zrows1;              // z entries summed from partials (tiles split in K)
  int64_t nz1 = 0;
  DevBuf<int32_t> zmap1;               // phase 1: slot row -> z entry (-1: padding) [slots][128]
  DevBuf<int64_t> br1, br2;            // B row ranges per exponent row [n][2]
  int32_t nb1 = 0, nb2 = 0;
  DevBuf<int32_t> eb1, eb2;            // B exponents [n][8]
  DevBuf<double> part1, part2;         // [slots * 128][8]
  DevBuf<double> z, yfar;              // [zlen][8], [Nb][8]
  DevBuf<int> err;
};

namespace tc {

constexpr int R = 8;
constexpr int TM = 128;
constexpr int KS = 32;                        // K elements per stage (one kind::i8 MMA)
constexpr int NDA = 4;                        // base-256 digits of an A element (31-bit fixed point)
constexpr int NDB = 6;                        // base-256 digits of a B element (47-bit fixed point)
constexpr int FIXA = 8 * NDA - 1;             // fixed-point bits below 2^e
constexpr int FIXB = 8 * NDB - 1;
constexpr int NSTAGE = 8;
constexpr int AD_BYTES = TM * KS;             // one digit plane of an A stage: 4 KB
constexpr int AST_BYTES = NDA * AD_BYTES;     // an A stage: 16 KB (4 bytes per element)
constexpr int NB = NDB * R;                   // MMA N = 48: column 8 u + n = digit u of state n
constexpr int BST_BYTES = NB * KS;            // the B digits of a stage: 1.5 KB
constexpr int BX_BYTES = KS * R * 8;          // the B rows of a stage as copied (FP64): 2 KB
constexpr int ACOLS = NDA * NB;               // TMEM columns of one accumulator buffer (4 x 48)
constexpr int TCOLS = 512;                    // allocated TMEM columns (2 buffers of 192)
constexpr int KSTEP_MAX_DEFAULT = 64;         // stages per tile (2048 K elements)
constexpr int THREADS = 384;
constexpr int CONV_THREADS = 128;             // warps 8-11
// + a 32 KB guard after the buffers, so that no descriptor-addressed read can leave the
// allocation even past the last stage
constexpr int SMEM_BYTES = NSTAGE * (AST_BYTES + BST_BYTES + BX_BYTES) + 1024 + 32768;
constexpr long long WAIT_LIMIT = 1ll << 22;  // polls of try_wait before a wait gives up
static_assert(NDB == 6, "digits6 cuts the B rows");
static_assert((TM / 8) * 128 * (KS / 16) == AD_BYTES && (NB / 8) * 128 * (KS / 16) == BST_BYTES, "digit tile layouts");
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
// instruction descriptor: D S32, A and B signed int8, both K-major, N = 32, M = 128
constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((static_cast<uint32_t>(NB) >> 3) << 17) |
                           ((128u >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(
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
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ND balanced base-256 digits (most significant first) of the (8 ND - 1)-bit fixed-point
// value llrint(v 2^(8 ND - 1 - e)), |v| < 2^(e - 1): sum_t d[t] 256^(ND - 1 - t) equals that
// integer exactly.
template <int ND>
__device__ __forceinline__ void digits(double v, int e, int8_t (&d)[ND]) {
  long long m = llrint(ldexp(v, 8 * ND - 1 - e));  // |m| <= 2^(8 ND - 2)
#pragma unroll
  for (int t = ND - 1; t >= 0; --t) {
    const int lo = static_cast<int>(m & 255);
    const int s = lo >= 128 ? lo - 256 : lo;  // balanced digit in [-128, 127]
    d[t] = static_cast<int8_t>(s);
    m = (m - s) >> 8;
  }
}

// 2^k as a double, -1022 <= k <= 1023 (exponent bits)
__device__ __forceinline__ double pow2i(int k) { return __longlong_as_double(static_cast<long long>(k + 1023) << 52); }

// digits<6>(v, e, d) for the B rows of every stage, in 32-bit integer steps: the 47-bit value
// m = hi 2^24 + lo (lo in [0, 2^24)) gives three balanced digits of lo, whose carry (0 or 1)
// goes into hi, and three of hi.  The digits are those of digits<6>.
__device__ __forceinline__ void digits6(double v, int e, int8_t (&d)[6]) {
  const int k = FIXB - e;
  const double sv = (k >= -1022 && k <= 1023) ? v * pow2i(k) : ldexp(v, k);
  const long long m = __double2ll_rn(sv);  // |m| <= 2^46
  int lo = static_cast<int>(m & 0xFFFFFF);
  int hi = static_cast<int>(m >> 24);      // |hi| <= 2^22
#pragma unroll
  for (int t = 5; t >= 3; --t) {
    const int q = static_cast<int>(static_cast<int8_t>(lo & 255));
    d[t] = static_cast<int8_t>(q);
    lo = (lo - q) >> 8;
  }
  hi += lo;
#pragma unroll
  for (int t = 2; t >= 1; --t) {
    const int q = static_cast<int>(static_cast<int8_t>(hi & 255));
    d[t] = static_cast<int8_t>(q);
    hi = (hi - q) >> 8;
  }
  d[0] = static_cast<int8_t>(hi);
}

// byte offset of element (row, k) of a K-major no-swizzle int8 tile of 32 K columns:
// 16-byte core-matrix rows, row groups of 8 at 128 bytes, the two K halves `half` bytes apart
__device__ __forceinline__ int i8off(int row, int k, int half) {
  return (k >> 4) * half + (row >> 3) * 128 + (row & 7) * 16 + (k & 15);
}

__global__ void __launch_bounds__(THREADS, 1)
    k_tc_gemm(const TcTile* __restrict__ tiles, int ntiles, const char* __restrict__ A,
              const int32_t* __restrict__ ea, const int32_t* __restrict__ eb, const double* __restrict__ bsrc,
              double* __restrict__ part, double* __restrict__ zout, const int32_t* __restrict__ zmap,
              int* __restrict__ err) {
  extern __shared__ __align__(1024) char smem[];
  char* sA = smem;                                   // [NSTAGE][NDA][AD_BYTES] A digits (as in HBM)
  char* sB = sA + NSTAGE * AST_BYTES;                // [NSTAGE][BST_BYTES]    B digits, N = 48 rows
  char* sX = sB + NSTAGE * BST_BYTES;                // [NSTAGE][BX_BYTES]     B rows as copied (FP64 [32][8])
  uint64_t* bars = reinterpret_cast<uint64_t*>(sX + NSTAGE * BX_BYTES);
  uint64_t* full = bars;                 // [NSTAGE] A copied
  uint64_t* ready = bars + NSTAGE;       // [NSTAGE] B digits written
  uint64_t* empty = bars + 2 * NSTAGE;   // [NSTAGE] MMAs done with the stage
  uint64_t* accf = bars + 3 * NSTAGE;    // [2] accumulator complete
  uint64_t* acce = bars + 3 * NSTAGE + 2;  // [2] accumulator read
  uint64_t* fin = bars + 3 * NSTAGE + 4;   // last MMAs done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 3 * NSTAGE + 6);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&ready[s], CONV_THREADS);
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
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)),
                 "r"(TCOLS)
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
    if (lane == 0) {  // producer: A digits and the stage's B rows (FP64) on one mbarrier
      int item = 0;
      int t = blockIdx.x;
      TcTile T;
      if (t < ntiles) T = tiles[t];
      for (; t < ntiles && !*abort_flag; t += gridDim.x) {
        TcTile Tn;
        if (t + static_cast<int>(gridDim.x) < ntiles) Tn = tiles[t + gridDim.x];  // next tile in flight
        for (int s0 = 0; s0 < T.nsteps; ++s0, ++item) {
          const int st = item % NSTAGE, rnd = item / NSTAGE;
          const int nb = min(KS, T.b_rows - s0 * KS);  // valid B rows of the stage
          if (!mbar_wait(&empty[st], (rnd & 1) ^ 1)) { fail(); break; }
          mbar_expect_tx(&full[st], AST_BYTES + (nb > 0 ? nb * R * 8 : 0));
          bulk_g2s(sA + st * AST_BYTES, A + T.a_off + static_cast<int64_t>(s0) * AST_BYTES, AST_BYTES, &full[st]);
          if (nb > 0)
            bulk_g2s(sX + st * BX_BYTES, bsrc + (static_cast<int64_t>(T.b_row0) + s0 * KS) * R, nb * R * 8,
                     &full[st]);
        }
        T = Tn;
      }
      // leave no copy in flight: the last stages' copies have landed (bounded)
      for (int q = max(0, item - NSTAGE); q < item; ++q) mbar_wait(&full[q % NSTAGE], (q / NSTAGE) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      int item = 0, tc = 0;
      bool issued = false;
      int t = blockIdx.x;
      int ns = t < ntiles ? tiles[t].nsteps : 0;
      for (; t < ntiles && !*abort_flag; t += gridDim.x, ++tc) {
        const int nsn = t + static_cast<int>(gridDim.x) < ntiles ? tiles[t + gridDim.x].nsteps : 0;
        const int buf = tc & 1, use = tc >> 1;
        if (!mbar_wait(&acce[buf], (use & 1) ^ 1)) { fail(); break; }
        tc_after();
        const uint32_t d0 = tbase + static_cast<uint32_t>(buf * ACOLS);
        bool ok = true;
        for (int s0 = 0; s0 < ns; ++s0, ++item) {
          const int st = item % NSTAGE, rnd = item / NSTAGE;
          if (!mbar_wait(&full[st], rnd & 1) || !mbar_wait(&ready[st], rnd & 1)) { fail(); ok = false; break; }
          tc_after();
          const uint64_t db = sdesc(su32(sB + st * BST_BYTES), (NB / 8) * 128, 128);
#pragma unroll
          for (int ta = 0; ta < NDA; ++ta) {
            const uint64_t da = sdesc(su32(sA + st * AST_BYTES + ta * AD_BYTES), (TM / 8) * 128, 128);
            mma_i8(d0 + static_cast<uint32_t>(ta * NB), da, db, s0 > 0 ? 1u : 0u);
          }
          mma_commit(&empty[st]);
          issued = true;
        }
        if (!ok) break;
        mma_commit(&accf[buf]);
        ns = nsn;
      }
      if (issued) {  // every MMA of this CTA has completed before tensor memory is freed
        mma_commit(fin);
        mbar_wait(fin, 0);
      }
    }
  } else if (warp >= 4 && warp < 8) {  // epilogue: TMEM lanes 32 (warp % 4) .. + 31
    const int sp = warp & 3;
    const int row = 32 * sp + lane;
    // 256^(8 - g) for the digit-pair weight g = t + u (exact powers of two)
    const double wgt[NDA + NDB - 1] = {0x1p64, 0x1p56, 0x1p48, 0x1p40, 0x1p32, 0x1p24, 0x1p16, 0x1p8, 1.0};
    int tc = 0;
    for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x, ++tc) {
      // the tile's exponents are loaded while its accumulators are being computed
      const TcTile T = tiles[t];
      const int er = ea[static_cast<int64_t>(T.slot) * TM + row];
      int en[R];
#pragma unroll
      for (int n = 0; n < R; ++n) en[n] = eb[static_cast<int64_t>(T.bsc) * R + n];
      const int buf = tc & 1, use = tc >> 1;
      if (!mbar_wait(&accf[buf], use & 1)) { fail(); break; }
      tc_after();
      const uint32_t ta0 = tbase + (static_cast<uint32_t>(32 * sp) << 16) + static_cast<uint32_t>(buf * ACOLS);
      double y[R];
#pragma unroll
      for (int n = 0; n < R; ++n) y[n] = 0.0;
#pragma unroll
      for (int ta = 0; ta < NDA; ++ta) {
        uint32_t v[NDB][8];  // v[u][n] = D_{ta,u}[row][n]
#pragma unroll
        for (int u = 0; u < NDB; ++u) tmem_ld8(ta0 + static_cast<uint32_t>(ta * NB + u * 8), v[u]);
        tmem_wait_ld();
#pragma unroll
        for (int n = 0; n < R; ++n)
#pragma unroll
          for (int u = 0; u < NDB; ++u) y[n] += static_cast<double>(static_cast<int32_t>(v[u][n])) * wgt[ta + u];
      }
      tc_before();
      mbar_arrive(&acce[buf]);
      double* o = part + (static_cast<int64_t>(T.slot) * TM + row) * R;
      if (T.direct) {  // the only partial of this row: straight to its z entry (padding rows dropped)
        const int32_t zi = zmap[static_cast<int64_t>(T.slot) * TM + row];
        o = zi >= 0 ? zout + static_cast<int64_t>(zi) * R : nullptr;
      }
      if (o) {
#pragma unroll
        for (int n = 0; n < R; ++n) o[n] = ldexp(y[n], er + en[n] - FIXA - FIXB);
      }
    }
  } else if (warp >= 8) {  // B digits: thread -> (state n, two k); rows 8 u + n of the N = 48 tile
    const int ct = tid - (THREADS - CONV_THREADS);
    const int n = ct >> 4, k0 = (ct & 15) * 2;
    int item = 0;
    int t = blockIdx.x;
    TcTile T;
    int e = 0;
    if (t < ntiles) {
      T = tiles[t];
      e = eb[static_cast<int64_t>(T.bsc) * R + n];
    }
    for (; t < ntiles && !*abort_flag; t += gridDim.x) {
      TcTile Tn;
      int en = 0;
      if (t + static_cast<int>(gridDim.x) < ntiles) {  // next tile and its exponent in flight
        Tn = tiles[t + gridDim.x];
        en = eb[static_cast<int64_t>(Tn.bsc) * R + n];
      }
      bool ok = true;
      for (int s0 = 0; s0 < T.nsteps; ++s0, ++item) {
        const int st = item % NSTAGE, rnd = item / NSTAGE;
        // the stage's copies have landed, so its previous MMAs are done and the digits are free
        if (!mbar_wait(&full[st], rnd & 1)) { fail(); ok = false; break; }
        const double* xs = reinterpret_cast<const double*>(sX + st * BX_BYTES);
        char* bs = sB + st * BST_BYTES;
        const int nb = T.b_rows - s0 * KS;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int k = k0 + j;
          const double x = k < nb ? xs[k * R + n] : 0.0;
          int8_t c[NDB];
          digits6(x, e, c);
#pragma unroll
          for (int u = 0; u < NDB; ++u) bs[i8off(8 * u + n, k, (NB / 8) * 128)] = static_cast<char>(c[u]);
        }
        fence_proxy_async();
        mbar_arrive(&ready[st]);
      }
      if (!ok) break;
      T = Tn;
      e = en;
    }
  }
  tc_before();
  __syncthreads();
  tc_after();
  if (warp == 2) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TCOLS) : "memory");
}

// out[i][n] = sum over p in [rp[i], rp[i+1]) of part[ix[p]][n]  (FP64, fixed order)
__global__ void k_tc_reduce(int64_t nrows, const int64_t* __restrict__ rows, const int64_t* __restrict__ rp,
                            const int32_t* __restrict__ ix,
                            const double* __restrict__ part, double* __restrict__ out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i = t >> 3;
  const int n = static_cast<int>(t & 7);
  if (i >= nrows) return;
  double s = 0.0;
  for (int64_t p = rp[i]; p < rp[i + 1]; ++p) s += part[static_cast<int64_t>(ix[p]) * R + n];
  out[(rows ? rows[i] : i) * R + n] = s;
}

// exponent e with max |v| < 2^(e - 1) (one bit of headroom for the rounding of the 42-bit
// value), 0 for zero
__device__ __forceinline__ int headroom_exp(double mx) { return mx > 0.0 ? ilogb(mx) + 2 : 0; }

// B exponents: for every range [rng[2j], rng[2j+1]) of rows of src ([rows][8] FP64) and every
// state n, out[j][n] = the exponent of the range's largest |value| (one CTA per range)
__global__ void k_tc_bexp(int nr, const int64_t* __restrict__ rng, const double* __restrict__ src,
                          int32_t* __restrict__ out) {
  __shared__ double sh[8][32];
  const int j = blockIdx.x;
  if (j >= nr) return;
  const int n = threadIdx.x & 7, w = threadIdx.x >> 3;  // 256 threads: 32 row lanes x 8 states
  double mx = 0.0;
  for (int64_t i = rng[2 * j] + w; i < rng[2 * j + 1]; i += 32) mx = fmax(mx, fabs(src[i * R + n]));
  sh[n][w] = mx;
  __syncthreads();
  if (threadIdx.x < 8) {
    double m = 0.0;
    for (int q = 0; q < 32; ++q) m = fmax(m, sh[threadIdx.x][q]);
    out[static_cast<int64_t>(j) * R + threadIdx.x] = headroom_exp(m);
  }
}

// The FP32 value of element (row r, K index k) of pack job J (0 past the valid rows / K).
__device__ __forceinline__ float tc_value(const TcPack& J, int r, int k, const double* __restrict__ pool,
                                          const int64_t* __restrict__ rowbase, const int64_t* __restrict__ colbase) {
  double v = 0.0;
  if (r < J.rvalid && k < J.kvalid) {
    if (J.mode == 1) {
      const int64_t b = rowbase[J.tab + r];
      if (b >= 0) v = pool[b + J.roff + k];
    } else {
      const int64_t c = colbase[J.tab + k];
      if (c >= 0) v = pool[c + J.roff + r];
    }
  }
  return static_cast<float>(v);
}

// Row maxima of the pack jobs: one CTA per (job, stage) of the flat stage list js, a thread per
// row; amax[slot][r] holds the bits of the largest |FP32 value| (non-negative floats order like
// their bit patterns), zeroed before.
__global__ void k_tc_rowmax(const TcPack* __restrict__ jobs, const int2* __restrict__ js,
                            const double* __restrict__ pool, const int64_t* __restrict__ rowbase,
                            const int64_t* __restrict__ colbase, unsigned int* __restrict__ amax) {
  const int2 q = js[blockIdx.x];
  const TcPack J = jobs[q.x];
  const int r = threadIdx.x;  // 128 threads
  float mx = 0.0f;
#pragma unroll 4
  for (int j = 0; j < KS; ++j) mx = fmaxf(mx, fabsf(tc_value(J, r, q.y * KS + j, pool, rowbase, colbase)));
  if (mx > 0.0f) atomicMax(amax + static_cast<int64_t>(J.slot) * TM + r, __float_as_uint(mx));
}

// A digits of one stage of a pack job: digit planes t = 0..3, each the rows 0..127 x K elements
// 32 s .. 32 s + 31 in the K-major no-swizzle layout of the MMA; ea[slot][r] = the exponent of row
// r's largest |value| over the tile.  The values are the FP32 factors (the FP32 packing's
// rounding).  One CTA per (job, stage), a thread per row.
__global__ void k_tc_pack(const TcPack* __restrict__ jobs, const int2* __restrict__ js,
                          const double* __restrict__ pool, const int64_t* __restrict__ rowbase,
                          const int64_t* __restrict__ colbase, const unsigned int* __restrict__ amax,
                          char* __restrict__ A, int32_t* __restrict__ ea) {
  const int2 q = js[blockIdx.x];
  const TcPack J = jobs[q.x];
  const int r = threadIdx.x;  // 128 threads
  const int e = headroom_exp(static_cast<double>(__uint_as_float(amax[static_cast<int64_t>(J.slot) * TM + r])));
  char* st = A + J.a_off + static_cast<int64_t>(q.y) * AST_BYTES;
  for (int k = 0; k < KS; k += 4) {  // four K elements -> one 32-bit word per digit plane
    uint32_t w[NDA] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int8_t d[NDA];
      digits<NDA>(static_cast<double>(tc_value(J, r, q.y * KS + k + j, pool, rowbase, colbase)), e, d);
#pragma unroll
      for (int t = 0; t < NDA; ++t) w[t] |= static_cast<uint32_t>(static_cast<uint8_t>(d[t])) << (8 * j);
    }
    char* o = st + i8off(r, k, (TM / 8) * 128);
#pragma unroll
    for (int t = 0; t < NDA; ++t) *reinterpret_cast<uint32_t*>(o + t * AD_BYTES) = w[t];
  }
  if (q.y == 0) ea[static_cast<int64_t>(J.slot) * TM + r] = e;
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
  // stages of 32 K elements per tile (the int32 group sums stay exact far beyond the largest
  // tile); SPX_TC_KSTEP sets it for tuning
  int KSTEP_MAX = kstep_max > 0 ? kstep_max : KSTEP_MAX_DEFAULT;
  if (kstep_max <= 0)
    if (const char* e = std::getenv("SPX_TC_KSTEP")) KSTEP_MAX = std::max(1, std::atoi(e));
  KSTEP_MAX = std::min(KSTEP_MAX, 256);
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
  std::vector<int64_t> rowbase, colbase, br1, br2;
  std::vector<std::pair<int64_t, int32_t>> m1, m2;
  std::vector<int32_t> zmap1;
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
      const int32_t bsc = static_cast<int32_t>(br1.size() / 2);
      br1.push_back(cs);
      br1.push_back(cs + K);
      std::vector<std::pair<int64_t, int64_t>> rows;  // (pool base of V row q, z entry)
      for (size_t v = u; v < e; ++v) {
        const HBlock& B = H.blocks[tmp[v].second];
        const int64_t n = B.ce - B.cs;
        for (int q = 0; q < B.rank; ++q) rows.push_back({B.off_v + q * n, zoff[tmp[v].second] + q});
      }
      const int64_t ksteps = (K + KS - 1) / KS;
      for (int64_t m0 = 0; m0 < static_cast<int64_t>(rows.size()); m0 += TM) {
        const int64_t tab = static_cast<int64_t>(rowbase.size());
        const int rv = static_cast<int>(std::min<int64_t>(TM, rows.size() - m0));
        for (int r = 0; r < TM; ++r) rowbase.push_back(r < rv ? rows[m0 + r].first : -1);
        for (int64_t k0 = 0; k0 < ksteps; k0 += KSTEP_MAX) {
          const int ns = static_cast<int>(std::min<int64_t>(KSTEP_MAX, ksteps - k0));
          const int kv = static_cast<int>(std::min<int64_t>(KS * ns, K - KS * k0));
          const int direct = ksteps <= KSTEP_MAX ? 1 : 0;
          t1.push_back(TcTile{a1, ns, static_cast<int32_t>(cs + KS * k0), kv, slot1, bsc, direct});
          p1.push_back(TcPack{a1, tab, KS * k0, ns, kv, rv, 1, slot1, 0});
          for (int r = 0; r < TM; ++r) zmap1.push_back(direct && r < rv ? static_cast<int32_t>(rows[m0 + r].second) : -1);
          if (!direct)
            for (int r = 0; r < rv; ++r) m1.push_back({rows[m0 + r].second, slot1 * TM + r});
          a1 += static_cast<int64_t>(ns) * AST_BYTES;
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
    const int32_t bsc = static_cast<int32_t>(br2.size() / 2);
    br2.push_back(z0);
    br2.push_back(z0 + K);
    const int64_t ksteps = (K + KS - 1) / KS;
    for (int64_t m0 = 0; m0 < rows; m0 += TM) {
      const int rv = static_cast<int>(std::min<int64_t>(TM, rows - m0));
      for (int64_t k0 = 0; k0 < ksteps; k0 += KSTEP_MAX) {
        const int ns = static_cast<int>(std::min<int64_t>(KSTEP_MAX, ksteps - k0));
        const int kv = static_cast<int>(std::min<int64_t>(KS * ns, K - KS * k0));
        t2.push_back(TcTile{a2, ns, static_cast<int32_t>(z0 + KS * k0), kv, slot2, bsc, 0});
        p2.push_back(TcPack{a2, kb + KS * k0, m0, ns, kv, rv, 2, slot2, 0});
        for (int r = 0; r < rv; ++r) m2.push_back({rs + m0 + r, slot2 * TM + r});
        a2 += static_cast<int64_t>(ns) * AST_BYTES;
        ++slot2;
      }
    }
  }
  SPX_CHECK(zlen < (int64_t(1) << 31) && slot1 < (1 << 24) && slot2 < (1 << 24) &&
                H.Nb + 2 * KS * KSTEP_MAX < (int64_t(1) << 31),
            "tensor-core plan too large");
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
  P->ea1.alloc(std::max<int64_t>(slot1, 1) * TM);
  P->ea2.alloc(std::max<int64_t>(slot2, 1) * TM);
  P->t1.upload(t1, s);
  P->t2.upload(t2, s);
  {
    DevBuf<int64_t> drb, dcb;
    drb.upload(rowbase.empty() ? std::vector<int64_t>{-1} : rowbase, s);
    dcb.upload(colbase.empty() ? std::vector<int64_t>{-1} : colbase, s);
    auto run = [&](const std::vector<TcPack>& jobs, char* dst, int32_t* ea, int64_t nslots) {
      if (jobs.empty()) return;
      std::vector<int2> js;
      for (size_t j = 0; j < jobs.size(); ++j)
        for (int st = 0; st < jobs[j].nsteps; ++st) js.push_back(make_int2(static_cast<int>(j), st));
      DevBuf<TcPack> dj;
      dj.upload(jobs, s);
      DevBuf<int2> djs;
      djs.upload(js, s);
      DevBuf<unsigned int> amax;
      amax.alloc(nslots * TM);
      amax.zero(s);
      const unsigned g = static_cast<unsigned>(js.size());
      k_tc_rowmax<<<g, TM, 0, s>>>(dj.p, djs.p, H.far_pool64.p, drb.p, dcb.p, amax.p);
      SPX_LAUNCH_CHECK();
      k_tc_pack<<<g, TM, 0, s>>>(dj.p, djs.p, H.far_pool64.p, drb.p, dcb.p, amax.p, dst, ea);
      SPX_LAUNCH_CHECK();
      SPX_CUDA(cudaStreamSynchronize(s));
    };
    run(p1, P->A1.p, P->ea1.p, slot1);
    run(p2, P->A2.p, P->ea2.p, slot2);
  }
  // phase 1: partial sums only for the z entries of tiles split in K (compacted row list)
  std::sort(m1.begin(), m1.end());
  std::vector<int64_t> zr1;
  std::vector<std::pair<int64_t, int32_t>> m1c;
  for (auto& pr : m1) {
    if (zr1.empty() || zr1.back() != pr.first) zr1.push_back(pr.first);
    m1c.push_back({static_cast<int64_t>(zr1.size()) - 1, pr.second});
  }
  Csr c1 = make_csr(static_cast<int64_t>(zr1.size()), m1c), c2 = make_csr(H.Nb, m2);
  P->nz1 = static_cast<int64_t>(zr1.size());
  P->zrows1.upload(zr1.empty() ? std::vector<int64_t>{0} : zr1, s);
  P->zmap1.upload(zmap1.empty() ? std::vector<int32_t>{-1} : zmap1, s);
  P->rp1.upload(c1.rp, s);
  P->ix1.upload(c1.ix.empty() ? std::vector<int32_t>{0} : c1.ix, s);
  P->rp2.upload(c2.rp, s);
  P->ix2.upload(c2.ix.empty() ? std::vector<int32_t>{0} : c2.ix, s);
  P->nb1 = static_cast<int32_t>(br1.size() / 2);
  P->nb2 = static_cast<int32_t>(br2.size() / 2);
  P->br1.upload(br1.empty() ? std::vector<int64_t>{0, 0} : br1, s);
  P->br2.upload(br2.empty() ? std::vector<int64_t>{0, 0} : br2, s);
  P->eb1.alloc(std::max<int64_t>(P->nb1, 1) * R);
  P->eb2.alloc(std::max<int64_t>(P->nb2, 1) * R);
  P->part1.alloc(std::max<int64_t>(slot1, 1) * TM * R);
  P->part2.alloc(std::max<int64_t>(slot2, 1) * TM * R);
  P->z.alloc(std::max<int64_t>(zlen, 1) * R);
  P->z.zero(s);  // rank-padding entries stay zero (no tile writes them)
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
    k_tc_bexp<<<P.nb1, 256, 0, s>>>(P.nb1, P.br1.p, xm, P.eb1.p);
    SPX_LAUNCH_CHECK();
    k_tc_gemm<<<grid, THREADS, SMEM_BYTES, s>>>(P.t1.p, P.nt1, P.A1.p, P.ea1.p, P.eb1.p, xm, P.part1.p, P.z.p,
                                               P.zmap1.p, P.err.p);
    SPX_LAUNCH_CHECK();
  }
  if (P.nz1 > 0) {
    k_tc_reduce<<<grid_for(P.nz1 * R, 256), 256, 0, s>>>(P.nz1, P.zrows1.p, P.rp1.p, P.ix1.p, P.part1.p, P.z.p);
    SPX_LAUNCH_CHECK();
  }
  if (P.nt2 > 0) {
    k_tc_bexp<<<P.nb2, 256, 0, s>>>(P.nb2, P.br2.p, P.z.p, P.eb2.p);
    SPX_LAUNCH_CHECK();
    k_tc_gemm<<<grid, THREADS, SMEM_BYTES, s>>>(P.t2.p, P.nt2, P.A2.p, P.ea2.p, P.eb2.p, P.z.p, P.part2.p, nullptr,
                                               nullptr, P.err.p);
    SPX_LAUNCH_CHECK();
  }
  k_tc_reduce<<<grid_for(H.Nb * R, 256), 256, 0, s>>>(H.Nb, nullptr, P.rp2.p, P.ix2.p, P.part2.p, P.yfar.p);
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
  return static_cast<int64_t>(P.A1.bytes() + P.A2.bytes() + P.ea1.bytes() + P.ea2.bytes() + P.part1.bytes() +
                              P.part2.bytes() + P.z.bytes() + P.yfar.bytes() + P.rp1.bytes() + P.rp2.bytes() +
                              P.ix1.bytes() + P.ix2.bytes() + P.br1.bytes() + P.br2.bytes() + P.eb1.bytes() +
                              P.eb2.bytes() + P.zrows1.bytes() + P.zmap1.bytes());
}

}  // namespace spx
