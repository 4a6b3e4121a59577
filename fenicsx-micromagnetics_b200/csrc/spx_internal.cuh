// Internal declarations shared by the libspx translation units.
//
// Layout conventions (device):
//   * nodal vectors are AoS: node-major, 3 components (x,y,z) per node, the
//     layout of the reference's PETSc CUDA Vec with block size 3
//     (gpu/solvers/llg_module_GPU.py:25-39);
//   * sparse FEM operators share ONE scalar node-node pattern stored as
//     SELL-32 (32-row slices, column-major inside a slice, rows padded with
//     zero entries that point at the row itself) so one thread per row reads
//     coalesced column indices and values;  value planes: 1 (stiffness),
//     3 (Div, G: one plane per component) or 9 (DMI 3x3 blocks).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace spx {

enum Status : int {
  OK = 0,
  ERR_INVALID = 1,
  ERR_CUDA = 2,
  ERR_OOM = 3,
  ERR_NOT_CONVERGED = 4,
  ERR_TIMEOUT = 5,
  ERR_INTERNAL = 6,
  ERR_NO_DEVICE = 7,
};

struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define SPX_CUDA(x)                                                                      \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) {                                                             \
      throw ::spx::Error(e_ == cudaErrorMemoryAllocation ? ::spx::ERR_OOM : ::spx::ERR_CUDA, \
                         std::string(#x) + ": " + cudaGetErrorString(e_));               \
    }                                                                                    \
  } while (0)

#define SPX_CHECK(cond, msg)                                     \
  do {                                                           \
    if (!(cond)) throw ::spx::Error(::spx::ERR_INVALID, (msg));   \
  } while (0)

#define SPX_LAUNCH_CHECK() SPX_CUDA(cudaGetLastError())

// ---------------------------------------------------------------- buffers
// Allocation-failure injection for tests of the out-of-memory paths (spx_debug_fail_alloc):
// the next g_fail_alloc_count device allocations of at least g_fail_alloc_min_bytes bytes
// fail with ERR_OOM before cudaMalloc is called.  Host-side only; no device fault.
extern std::atomic<int64_t> g_fail_alloc_min_bytes;
extern std::atomic<int32_t> g_fail_alloc_count;
inline void injected_alloc_failure(size_t bytes) {
  if (g_fail_alloc_count.load(std::memory_order_relaxed) <= 0) return;
  if (static_cast<int64_t>(bytes) < g_fail_alloc_min_bytes.load(std::memory_order_relaxed)) return;
  if (g_fail_alloc_count.fetch_sub(1) > 0)
    throw Error(ERR_OOM, "cudaMalloc: out of memory (injected by spx_debug_fail_alloc, " + std::to_string(bytes) +
                             " bytes)");
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) {
      injected_alloc_failure(count * sizeof(T));
      SPX_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T)));
    }
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void upload(const T* h, size_t count, cudaStream_t s = 0) {
    if (count != n) alloc(count);
    if (count) SPX_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& v, cudaStream_t s = 0) { upload(v.data(), v.size(), s); }
  void download(T* h, size_t count, cudaStream_t s = 0) const {
    if (count) SPX_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  void zero(cudaStream_t s = 0) {
    if (n) SPX_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------- host geometry
// Boundary data of build_boundary_data_serial (gpu/fields/Demag_Lindholm.py:177-285)
// in the canonical facet order (facets sorted by ascending vertex triple).
struct HostBoundary {
  int64_t N = 0, Nb = 0, Nt = 0;
  std::vector<int32_t> bverts;   // [Nb] global vertex of each boundary row
  std::vector<int32_t> tris;     // [Nt*3] global vertex ids (oriented)
  std::vector<int32_t> tri_lid;  // [Nt*3] boundary-local ids
  std::vector<double> Xb;        // [Nb*3]
  std::vector<double> tri_pts;   // [Nt*9]
  std::vector<double> ntri;      // [Nt*3]
  std::vector<double> area;      // [Nt]
  std::vector<double> s_edge;    // [Nt*3]
  std::vector<double> eta;       // [Nt*9]
  std::vector<double> gamma;     // [Nt*9]
  std::vector<double> omega_sum; // [Nb]
};

void build_boundary(const double* X, int64_t N, const int32_t* tets, int64_t E, HostBoundary& out);

// Scalar node-node CSR pattern of a P1 mesh (sorted columns, diagonal included)
// and the assembled P1 operators on it.
struct HostFem {
  int64_t N = 0, E = 0;
  std::vector<int64_t> rowptr;  // [N+1]
  std::vector<int32_t> col;     // [nnz]
  std::vector<double> A;        // [nnz]   stiffness  int grad u . grad v
  std::vector<double> Div;      // [3*nnz] Div[i,(j,c)]/Ms = sum vol/4 d_c lambda_i
  std::vector<double> G;        // [3*nnz] G[(i,c), j] = -sum vol/4 d_c lambda_j
  std::vector<double> vol;      // [N]     lumped nodal volume
};

void assemble_fem(const double* X, int64_t N, const int32_t* tets, int64_t E, HostFem& out);

// Interfacial-DMI operator restating gpu/fields/DMI_Interfacial_GPU.py:140-172 as
// 3x3 blocks on the scalar pattern (unscaled; callers apply the row prefactor).
void assemble_dmi_interfacial(const double* X, const int32_t* tets, int64_t E, const HostFem& fem,
                              const HostBoundary& bd, const double* n_nodes,
                              std::vector<double>& blocks9);

// Bulk-DMI operator restating gpu/fields/DMI_Bulk_GPU.py:52-66 as 3x3 blocks (unscaled).
void assemble_dmi_bulk(const double* X, const int32_t* tets, int64_t E, const HostFem& fem, const HostBoundary& bd,
                       std::vector<double>& blocks9);
// Both DMI operators with their row prefactors (interfacial -2 D_int / (mu0 Ms) / 1e-9 / V_i,
// DMI_Interfacial_GPU.py:160-165; bulk 2 D_bulk / (mu0 Ms) * 1e9 / V_i, DMI_Bulk_GPU.py:63-66),
// summed; a term with a zero constant is left out.
void dmi_blocks_scaled(const double* X, const int32_t* tets, int64_t E, const HostFem& fem, const HostBoundary& bd,
                       double Ms, double D_int, const double* n_int, double D_bulk, std::vector<double>& blocks9);

// Zhang-Li operator int (J . grad u) v dx on the node pattern (unscaled), J nodal [3N].
void assemble_zhang_li(const double* X, const int32_t* tets, int64_t E, const HostFem& fem, const double* J,
                       std::vector<double>& K);

// Cluster tree of gpu/fields/lindholm_hmatrix_gpu/tree.py:41-96 (bit-exact permutation).
struct TreeNode {
  int32_t start, stop;
  double bmin[3], bmax[3];
  int32_t left = -1, right = -1;
  bool leaf() const { return left < 0 && right < 0; }
  int32_t size() const { return stop - start; }
  double diameter() const;
};
struct ClusterTree {
  std::vector<int32_t> perm;
  std::vector<TreeNode> nodes;  // nodes[0] is the root
};
void build_cluster_tree(const double* pts, int64_t n, int leaf_size, ClusterTree& out);
bool admissible(const TreeNode& a, const TreeNode& b, double eta);

// ---------------------------------------------------------------- SELL-32
constexpr int SELL_C = 32;
struct HostSell {
  int64_t nrows = 0;
  int64_t nslices = 0;
  std::vector<int64_t> slice_ptr;  // [nslices+1] offsets into col/values (multiples of 32)
  std::vector<int32_t> col;        // [slice_ptr.back()]
  std::vector<int64_t> map;        // [nnz of source CSR] position of each CSR entry in SELL
};
// rows: subset of CSR rows (in order); col_map: column index remap (-1 = drop entry)
void build_sell(const std::vector<int64_t>& rowptr, const std::vector<int32_t>& col,
                const std::vector<int32_t>& rows, const std::vector<int32_t>* col_map,
                HostSell& out);
// values_out[plane][sell] from CSR values [plane-major stride nnz or interleaved]
template <class T>
void sell_values(const HostSell& s, const double* csr_vals, int planes, bool interleaved,
                 int64_t nnz, double scale, std::vector<T>& out) {
  const int64_t L = s.slice_ptr.back();
  out.assign(static_cast<size_t>(L) * planes, T(0));
  for (int64_t k = 0; k < static_cast<int64_t>(s.map.size()); ++k) {
    const int64_t pos = s.map[k];
    if (pos < 0) continue;
    for (int p = 0; p < planes; ++p) {
      const double v = interleaved ? csr_vals[k * planes + p] : csr_vals[p * nnz + k];
      out[static_cast<size_t>(p) * L + pos] = static_cast<T>(v * scale);
    }
  }
}

template <class T>
struct DevSell {
  int64_t nrows = 0, nslices = 0, len = 0;
  DevBuf<int64_t> slice_ptr;
  DevBuf<int32_t> col;
  void upload(const HostSell& h, cudaStream_t s = 0) {
    nrows = h.nrows;
    nslices = h.nslices;
    len = h.slice_ptr.back();
    slice_ptr.upload(h.slice_ptr, s);
    col.upload(h.col, s);
  }
};

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; result valid in every thread. smem needs >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* smem) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  double t = (threadIdx.x < nw) ? smem[threadIdx.x] : 0.0;
  if (wid == 0) t = warp_sum(t);
  if (threadIdx.x == 0) smem[0] = t;
  __syncthreads();
  const double r = smem[0];
  __syncthreads();
  return r;
}

// Grid-wide barrier for cooperative (co-resident) launches.  Every wait is bounded:
// after `limit` polls the waiting block raises *err and returns false; callers then
// leave the kernel.  count/gen live in device memory zeroed before the launch.
__device__ __forceinline__ bool grid_barrier(unsigned int* count, unsigned int* gen,
                                             unsigned int nblocks, int* err,
                                             long long limit = (1ll << 26)) {
  // One monotonic arrival counter (zeroed before the launch): after the CTA's own barrier,
  // thread 0 adds 1 with release semantics at GPU scope (covering every write the CTA made
  // before bar.sync) and polls with acquire loads until the counter reaches the next multiple
  // of nblocks; the closing bar.sync hands the acquired view to the CTA.  The error word is
  // read every 1024 polls only (a CTA that gave up never arrives, so the others stop by it or
  // by their own poll limit).  `gen` is not used.
  (void)gen;
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(count) : "memory");
    const unsigned int target = (old / nblocks + 1u) * nblocks;
    int ok = 1;
    for (long long it = 1;; ++it) {
      unsigned int v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
      if (static_cast<int>(v - target) >= 0) break;
      if ((it & 1023) == 0 && *reinterpret_cast<volatile int*>(err) != 0) {
        ok = 0;
        break;
      }
      if (it > limit) {
        atomicCAS(err, 0, ERR_TIMEOUT);
        ok = 0;
        break;
      }
      if (it > 4096) __nanosleep(32);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ------------------------------------------------------------------ CTA reductions
// sum of up to 4 values over the CTA; result valid in every thread (sh >= 4*32+4 doubles)
__device__ __forceinline__ void cta_sum4(double v[4], double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = warp_sum(v[q]);
  __syncthreads();
  if (lane == 0)
    for (int q = 0; q < 4; ++q) sh[4 * wid + q] = v[q];
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double t = (lane < nw) ? sh[4 * lane + q] : 0.0;
      t = warp_sum(t);
      if (lane == 0) sh[128 + q] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = sh[128 + q];
  __syncthreads();
}

// write this CTA's partials of slot s
__device__ __forceinline__ void cta_partial(double* part, int s, double a, double b, double c, double d,
                                            double* sh) {
  double v[4] = {a, b, c, d};
  cta_sum4(v, sh);
  if (threadIdx.x < 4) part[(static_cast<int64_t>(s) * gridDim.x + blockIdx.x) * 4 + threadIdx.x] = v[threadIdx.x];
}

// total of slot s over all CTAs, same order in every CTA (call after a grid barrier)
__device__ __forceinline__ void cta_total(const double* part, int s, double out[4], double* sh) {
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int c = threadIdx.x; c < static_cast<int>(gridDim.x); c += blockDim.x) {
    const double* p = part + (static_cast<int64_t>(s) * gridDim.x + c) * 4;
    v[0] += p[0];
    v[1] += p[1];
    v[2] += p[2];
    v[3] += p[3];
  }
  cta_sum4(v, sh);
  for (int q = 0; q < 4; ++q) out[q] = v[q];
}


// precision helpers
template <class T> __device__ __forceinline__ float to_f(T v) { return static_cast<float>(v); }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

inline int num_sms(int dev = -1) {
  if (dev < 0) SPX_CUDA(cudaGetDevice(&dev));
  int v = 0;
  SPX_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
  return v;
}

inline unsigned grid_for(int64_t n, int threads, int64_t cap = 1ll << 30) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return static_cast<unsigned>(b);
}

}  // namespace spx
