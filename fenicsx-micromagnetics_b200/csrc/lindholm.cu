// Lindholm double-layer weights and block fill (FP64, sm_100a).
//
// Device restatement of the analytic kernel of gpu/fields/Lindholm_kernel.py:30-125
// (solid angle via atan2, edge logs via log1p with the 1e-300 floor, opposite-edge
// convention) and of the block fill of lindholm_hmatrix_gpu/entry_provider.py:41-117.
//
// Fill design.  A CTA owns a tile of TR=128 block rows x TC=32 block columns.  Its
// first 32 threads build the list of triangles incident to the tile's columns (each
// triangle kept once, by its lowest in-tile column, in a fixed order so results are
// deterministic), then every thread (one per row) walks that list, evaluates the three
// weights once per (row, triangle) and adds them to its private row of a shared-memory
// accumulator.  Triangles incident to the row vertex are skipped (incident_policy
// "skip", gpu/fields/Demag_Lindholm.py:87-96).  The tile is written back row-major with
// consecutive threads on consecutive columns.  No atomics.
#include <cmath>

#include "spx_internal.cuh"

namespace spx {

// packed triangle record (36 doubles):
// p0[3] p1[3] p2[3] n[3] area s[3] eta[3][3] gamma[3][3] pad[2]
constexpr int TRI_REC = 36;

__device__ __forceinline__ void lindholm_weights_dev(const double x0, const double x1, const double x2,
                                                     const double* __restrict__ T, double& w0,
                                                     double& w1, double& w2) {
  const double tiny = 1e-300;
  const double r00 = __ldg(T + 0) - x0, r01 = __ldg(T + 1) - x1, r02 = __ldg(T + 2) - x2;
  const double r10 = __ldg(T + 3) - x0, r11 = __ldg(T + 4) - x1, r12 = __ldg(T + 5) - x2;
  const double r20 = __ldg(T + 6) - x0, r21 = __ldg(T + 7) - x1, r22 = __ldg(T + 8) - x2;
  const double n0 = sqrt(r00 * r00 + r01 * r01 + r02 * r02) + tiny;
  const double n1 = sqrt(r10 * r10 + r11 * r11 + r12 * r12) + tiny;
  const double n2 = sqrt(r20 * r20 + r21 * r21 + r22 * r22) + tiny;
  const double h = __ldg(T + 9) * r00 + __ldg(T + 10) * r01 + __ldg(T + 11) * r02;
  const double* eta = T + 16;
  const double e0 = __ldg(eta + 0) * r00 + __ldg(eta + 1) * r01 + __ldg(eta + 2) * r02;
  const double e1 = __ldg(eta + 3) * r10 + __ldg(eta + 4) * r11 + __ldg(eta + 5) * r12;
  const double e2 = __ldg(eta + 6) * r20 + __ldg(eta + 7) * r21 + __ldg(eta + 8) * r22;
  const double s0 = __ldg(T + 13), s1 = __ldg(T + 14), s2 = __ldg(T + 15);
  double d;
  d = n0 + n1 - s0; d = d < tiny ? tiny : d; const double P0 = log1p((2.0 * s0) / d);
  d = n1 + n2 - s1; d = d < tiny ? tiny : d; const double P1 = log1p((2.0 * s1) / d);
  d = n2 + n0 - s2; d = d < tiny ? tiny : d; const double P2 = log1p((2.0 * s2) / d);
  const double det = r00 * (r11 * r22 - r12 * r21) - r01 * (r10 * r22 - r12 * r20) +
                     r02 * (r10 * r21 - r11 * r20);
  const double d01 = r00 * r10 + r01 * r11 + r02 * r12;
  const double d12 = r10 * r20 + r11 * r21 + r12 * r22;
  const double d20 = r20 * r00 + r21 * r01 + r22 * r02;
  const double omega = 2.0 * atan2(det, n0 * n1 * n2 + d01 * n2 + d12 * n0 + d20 * n1);
  const double* g = T + 25;
  const double gP0 = __ldg(g + 0) * P0 + __ldg(g + 1) * P1 + __ldg(g + 2) * P2;
  const double gP1 = __ldg(g + 3) * P0 + __ldg(g + 4) * P1 + __ldg(g + 5) * P2;
  const double gP2 = __ldg(g + 6) * P0 + __ldg(g + 7) * P1 + __ldg(g + 8) * P2;
  const double c = 1.0 / (8.0 * 3.141592653589793 * (__ldg(T + 12) + tiny));
  w0 = s1 * c * (e1 * omega - h * gP0);
  w1 = s2 * c * (e2 * omega - h * gP1);
  w2 = s0 * c * (e0 * omega - h * gP2);
}

__global__ void k_lindholm_pairs(int64_t P, const double* __restrict__ x0, const int32_t* __restrict__ tri,
                                 const double* __restrict__ T, int64_t Nt, double* __restrict__ w) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= P) return;
  if (tri[k] < 0 || tri[k] >= Nt) {  // invalid triangle id: NaN weights, no access
    w[3 * k] = w[3 * k + 1] = w[3 * k + 2] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  double a, b, c;
  lindholm_weights_dev(x0[3 * k], x0[3 * k + 1], x0[3 * k + 2], T + (int64_t)tri[k] * TRI_REC, a, b, c);
  w[3 * k] = a;
  w[3 * k + 1] = b;
  w[3 * k + 2] = c;
}

struct FillDesc {
  int64_t out_off;   // offset of the block in the output pool (row-major m x n)
  int64_t rows_off;  // offset into rows pool
  int64_t cols_off;  // offset into cols pool
  int32_t m, n;
};

constexpr int FILL_TR = 128;
constexpr int FILL_TC = 32;

// tile_start[b] = first task of block b (prefix sum of ceil(m/TR)*ceil(n/TC)); nb blocks
__global__ void __launch_bounds__(FILL_TR) k_fill_tiles(
    const FillDesc* __restrict__ blocks, const int64_t* __restrict__ tile_start, int nb,
    const int32_t* __restrict__ rows_pool, const int32_t* __restrict__ cols_pool,
    const double* __restrict__ Xb, const int32_t* __restrict__ tri_lid,
    const double* __restrict__ T, const int32_t* __restrict__ inc_ptr,
    const int32_t* __restrict__ inc_tri, int maxinc, int64_t Nb, double* __restrict__ out) {
  extern __shared__ double smem[];
  double* acc = smem;                                                       // [TR][TC+1]
  int32_t* scol = reinterpret_cast<int32_t*>(acc + FILL_TR * (FILL_TC + 1));  // [TC]
  int32_t* scnt = scol + FILL_TC;                                            // [TC]
  int32_t* stri = scnt + FILL_TC;                                            // [TC*maxinc]
  int32_t* sslot = stri + FILL_TC * maxinc;                                  // [TC*maxinc] packed slots

  const int64_t task = blockIdx.x;
  // find block: largest b with tile_start[b] <= task
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_start[mid] <= task) lo = mid; else hi = mid - 1;
  }
  const FillDesc bd = blocks[lo];
  const int64_t local = task - tile_start[lo];
  const int ntc = (bd.n + FILL_TC - 1) / FILL_TC;
  const int rt = static_cast<int>(local / ntc), ct = static_cast<int>(local % ntc);
  const int row0 = rt * FILL_TR, col0 = ct * FILL_TC;
  const int tc = min(FILL_TC, bd.n - col0);
  const int tid = threadIdx.x;

  if (tid < FILL_TC) {
    int32_t cv = (tid < tc) ? cols_pool[bd.cols_off + col0 + tid] : -1;
    scol[tid] = (cv >= 0 && cv < Nb) ? cv : -1;  // out-of-range column ids contribute nothing
  }
  for (int i = tid; i < FILL_TR * (FILL_TC + 1); i += blockDim.x) acc[i] = 0.0;
  __syncthreads();
  if (tid < FILL_TC) {
    int cnt = 0;
    if (tid < tc && scol[tid] >= 0) {
      const int32_t node = scol[tid];
      for (int32_t q = inc_ptr[node]; q < inc_ptr[node + 1]; ++q) {
        const int32_t t = inc_tri[q];
        int slot[3];
        int first = FILL_TC;
        for (int v = 0; v < 3; ++v) {
          const int32_t gv = tri_lid[3 * (int64_t)t + v];
          slot[v] = -1;
          for (int c = 0; c < tc; ++c)
            if (scol[c] == gv) { slot[v] = c; break; }
          if (slot[v] >= 0 && slot[v] < first) first = slot[v];
        }
        if (first == tid && cnt < maxinc) {
          stri[tid * maxinc + cnt] = t;
          sslot[tid * maxinc + cnt] = (slot[0] + 1) | ((slot[1] + 1) << 8) | ((slot[2] + 1) << 16);
          ++cnt;
        }
      }
    }
    scnt[tid] = cnt;
  }
  __syncthreads();

  const int r = row0 + tid;
  const int32_t gi = (r < bd.m) ? rows_pool[bd.rows_off + r] : -1;
  if (gi >= 0 && gi < Nb) {  // out-of-range row ids leave their row at zero
    const double x0 = Xb[3 * (int64_t)gi], x1 = Xb[3 * (int64_t)gi + 1], x2 = Xb[3 * (int64_t)gi + 2];
    double* my = acc + tid * (FILL_TC + 1);
    for (int c = 0; c < tc; ++c) {
      const int cnt = scnt[c];
      for (int k = 0; k < cnt; ++k) {
        const int32_t t = stri[c * maxinc + k];
        const int32_t a = __ldg(tri_lid + 3 * (int64_t)t), b = __ldg(tri_lid + 3 * (int64_t)t + 1),
                      cc = __ldg(tri_lid + 3 * (int64_t)t + 2);
        if (gi == a || gi == b || gi == cc) continue;
        double w0, w1, w2;
        lindholm_weights_dev(x0, x1, x2, T + (int64_t)t * TRI_REC, w0, w1, w2);
        const int sl = sslot[c * maxinc + k];
        const int s0 = (sl & 0xff) - 1, s1 = ((sl >> 8) & 0xff) - 1, s2 = ((sl >> 16) & 0xff) - 1;
        if (s0 >= 0) my[s0] += w0;
        if (s1 >= 0) my[s1] += w1;
        if (s2 >= 0) my[s2] += w2;
      }
    }
  }
  __syncthreads();
  const int tr = min(FILL_TR, bd.m - row0);
  for (int idx = tid; idx < tr * FILL_TC; idx += blockDim.x) {
    const int rr = idx / FILL_TC, cc = idx % FILL_TC;
    if (cc < tc) out[bd.out_off + (int64_t)(row0 + rr) * bd.n + col0 + cc] = acc[rr * (FILL_TC + 1) + cc];
  }
}

__global__ void k_add_diag(int64_t Nb, const double* __restrict__ omega_sum, double* __restrict__ B) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < Nb) B[i * Nb + i] += omega_sum[i] * (1.0 / (4.0 * 3.141592653589793)) - 1.0;
}

size_t fill_smem_bytes(int maxinc) {
  return sizeof(double) * FILL_TR * (FILL_TC + 1) + sizeof(int32_t) * (2 * FILL_TC + 2 * FILL_TC * maxinc);
}

// Host launcher: fill nb blocks described by host descriptors (device pools given).
void launch_fill(const FillDesc* d_blocks, const int64_t* d_tile_start, int nb, int64_t ntiles,
                 const int32_t* rows_pool, const int32_t* cols_pool, const double* Xb,
                 const int32_t* tri_lid, const double* T, const int32_t* inc_ptr,
                 const int32_t* inc_tri, int maxinc, int64_t Nb, double* out, cudaStream_t s) {
  if (ntiles <= 0) return;
  const size_t smem = fill_smem_bytes(maxinc);
  static bool attr_set = false;
  if (!attr_set) {
    SPX_CUDA(cudaFuncSetAttribute(k_fill_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    attr_set = true;
  }
  SPX_CHECK(smem <= 160 * 1024, "too many incident triangles per boundary vertex for the fill kernel");
  SPX_CHECK(ntiles < (1ll << 31), "fill launch too large; split the batch");
  {
    k_fill_tiles<<<static_cast<unsigned>(ntiles), FILL_TR, smem, s>>>(
        d_blocks, d_tile_start, nb, rows_pool, cols_pool, Xb, tri_lid, T, inc_ptr, inc_tri, maxinc, Nb, out);
    SPX_LAUNCH_CHECK();
  }
}

void launch_lindholm_pairs(int64_t P, const double* x0, const int32_t* tri, const double* T, int64_t Nt, double* w,
                           cudaStream_t s) {
  if (P <= 0) return;
  k_lindholm_pairs<<<grid_for(P, 128), 128, 0, s>>>(P, x0, tri, T, Nt, w);
  SPX_LAUNCH_CHECK();
}

void launch_add_diag(int64_t Nb, const double* omega_sum, double* B, cudaStream_t s) {
  if (Nb <= 0) return;
  k_add_diag<<<grid_for(Nb, 256), 256, 0, s>>>(Nb, omega_sum, B);
  SPX_LAUNCH_CHECK();
}

// pack the boundary triangles into 36-double records
void pack_triangles(const HostBoundary& bd, std::vector<double>& rec) {
  rec.assign(static_cast<size_t>(bd.Nt) * TRI_REC, 0.0);
  for (int64_t t = 0; t < bd.Nt; ++t) {
    double* R = rec.data() + t * TRI_REC;
    for (int k = 0; k < 9; ++k) R[k] = bd.tri_pts[9 * t + k];
    for (int k = 0; k < 3; ++k) R[9 + k] = bd.ntri[3 * t + k];
    R[12] = bd.area[t];
    for (int k = 0; k < 3; ++k) R[13 + k] = bd.s_edge[3 * t + k];
    for (int k = 0; k < 9; ++k) R[16 + k] = bd.eta[9 * t + k];
    for (int k = 0; k < 9; ++k) R[25 + k] = bd.gamma[9 * t + k];
  }
}

}  // namespace spx
