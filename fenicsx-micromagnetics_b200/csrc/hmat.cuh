// H-matrix handle: construction (batched GPU fill + full-pivot ACA) and apply.
#pragma once

#include <memory>

#include "spx_internal.cuh"

namespace spx {

struct FillDesc;
void launch_fill(const FillDesc* d_blocks, const int64_t* d_tile_start, int nb, int64_t ntiles,
                 const int32_t* rows_pool, const int32_t* cols_pool, const double* Xb,
                 const int32_t* tri_lid, const double* T, const int32_t* inc_ptr,
                 const int32_t* inc_tri, int maxinc, int64_t Nb, double* out, cudaStream_t s);
void launch_lindholm_pairs(int64_t P, const double* x0, const int32_t* tri, const double* T, int64_t Nt, double* w,
                           cudaStream_t s);
void launch_add_diag(int64_t Nb, const double* omega_sum, double* B, cudaStream_t s);
void pack_triangles(const HostBoundary& bd, std::vector<double>& rec);

// Boundary geometry resident on one device.
struct BoundaryDev {
  int device = 0;
  HostBoundary host;
  DevBuf<double> Xb, T, omega_sum;
  DevBuf<int32_t> tri_lid, inc_ptr, inc_tri, bverts;
  int maxinc = 0;
  void create(const double* X, int64_t N, const int32_t* tets, int64_t E);
  // fill B[rows, cols] (no diagonal jump) for one block into out (row-major m x n)
  void fill_block(const int32_t* rows_dev, int64_t m, const int32_t* cols_dev, int64_t n, double* out,
                  cudaStream_t s) const;
  void dense_B(double* B, cudaStream_t s) const;
};

// packing of the H-matrix apply data: F64 / F32 factors and tiles; MIXED = BF16 factors with
// FP32 tiles; SPLIT = recompressed factors with FP32 leading and FP16 trailing columns, FP32
// tiles (pipelines use F64, F32 and MIXED only)
enum class Prec : int { F64 = 0, F32 = 1, MIXED = 2, SPLIT = 3 };

struct HBuildConfig {
  double epsilon = 1e-5;
  double eta = 2.0;
  int leaf_size = 64;
  int max_rank = -1;  // <0: None
  int64_t max_temporary_block_bytes = 256ll * 1024 * 1024;
  double low_rank_storage_factor = 0.95;
  int64_t batch_bytes = 6ll * 1024 * 1024 * 1024;  // device workspace per fill/ACA batch
  bool recompress = false;  // SVD recompression of the far factors after the build
};

struct HStats {
  int64_t dense_blocks = 0, low_rank_blocks = 0, rejected_low_rank_blocks = 0;
  int64_t forced_subdivisions_memory = 0, compression_tolerance_subdivisions = 0;
  int64_t max_observed_rank = 0, sum_observed_rank = 0, block_entry_evaluations = 0;
  int64_t near_entries = 0, far_entries = 0, n_far = 0, n_near = 0, aca_steps = 0, waves = 0;
  double build_seconds = 0.0;
};

struct HBlock {
  int32_t rs, re, cs, ce;
  int32_t type;  // 1 far, 0 near
  int32_t rank;
  int64_t off_u, off_v;  // far: offsets (FP64 pool) of U^T (k x m) and V (k x n); near: off_u = tile offset
  double relres;
};

// Apply-side records (see hmat.cu).  FarUnit: columns [xc, xc + nc) of far block V^T rows
// (nc rows of ldk elements at element voff: row c holds V[0..k-1, c]); flags & 3 at the last
// unit of the block in a warp: 1 write z[zout + q], 2 write partial slot zout + q of group
// grp.  FarGroup: a block whose units several warps share: partials at pbase + c * ldk + q
// for contributor c < ncontrib, result z[zdst + q], q < k.  RowItem: a tile of len rows at
// element off, row q scaled by z[src + q] (far) or x~[src + q] (near).
struct FarUnit {
  int64_t voff;
  int32_t ldk, nc, xc, k, zout, grp, flags, pad;
};
struct FarGroup {
  int32_t pbase, ncontrib, zdst, k;
};
struct RowItem {
  int64_t off;
  int32_t len, src;
};

struct TcPlan;  // hmat_tc.cu

struct RecompressStats {
  int64_t entries_before = 0, entries_after = 0, rewritten = 0;
  double truncation_error_max = 0.0;  // largest truncation error of a block, relative to its norm
};

struct HMatrix {
  int device = 0;
  int64_t Nb = 0;
  HBuildConfig cfg;
  HStats stats;
  ClusterTree tree;
  std::vector<HBlock> blocks;     // partition, in creation order
  DevBuf<double> far_pool64;      // U^T / V factors, FP64
  DevBuf<double> near_pool64;     // near tiles, FP64 row-major
  DevBuf<double> diag_perm;       // diag_jump[perm]
  DevBuf<int32_t> perm;
  // apply-side packed data (built by pack())
  Prec prec = Prec::F64;
  bool packed = false;
  DevBuf<char> far_f, near_f;     // factor / tile storage in the packed precision
  DevBuf<FarUnit> units;          // k_far_z work units
  DevBuf<int32_t> warp_first;     // [nwarps_z + 1] unit range of each k_far_z warp
  DevBuf<FarGroup> groups;        // far blocks shared by several k_far_z warps
  DevBuf<unsigned int> gcnt;      // per group: contributors arrived (reset by the last one)
  DevBuf<int32_t> seg_start;      // [nseg + 1] row segments (perm space)
  DevBuf<int64_t> item_ptr;       // [nseg + 1] items of each segment: far ones, then near ones
  DevBuf<int64_t> near_begin;     // [nseg] first near item of each segment
  DevBuf<RowItem> items;
  DevBuf<char> far_h;             // SPLIT: FP16 trailing columns (V^T rows and U tiles)
  DevBuf<FarUnit> units_h;        // SPLIT: k_far_z units of the FP16 columns
  DevBuf<int32_t> warp_first_h;
  DevBuf<int64_t> half_begin;     // SPLIT: [nseg] first FP16 far item of each segment
  DevBuf<double> zscale;          // SPLIT: [zlen] sigma of each FP16 column (1 elsewhere)
  int64_t nunits_h = 0, nwarps_z_h = 0;
  DevBuf<char> z, zpart;          // far z vectors and partial sums (accumulation type)
  DevBuf<char> xperm;             // x in perm order (vector type)
  int64_t nseg = 0, zlen = 0, zpart_len = 0, n_far = 0, n_near = 0, nunits = 0, nwarps_z = 0;
  int64_t bytes_far = 0, bytes_near = 0;
  std::unique_ptr<HMatrix> tr;    // H^T (same tree; built on first use by transposed())
  DevBuf<double> xmulti, zmulti, zpmulti;  // state-interleaved work vectors of apply_multi
  // far-field GEMMs of apply_multi on the tensor cores for batches of 8 (hmat_tc.cu); null: off
  std::shared_ptr<TcPlan> tc;

  // SVD recompression of the far factors (hrecompress.cu); columns ordered by decreasing
  // singular value, sigma[block] holds them for rewritten blocks (empty otherwise)
  bool recompressed = false;
  std::vector<std::vector<double>> sigma;
  RecompressStats recompress(cudaStream_t s);
  void build(const BoundaryDev& bd, const HBuildConfig& c, cudaStream_t s);
  void pack(Prec p, cudaStream_t s);
  // y = H x in the original boundary ordering, FP64 vectors
  void apply_f64(const double* x, double* y, cudaStream_t s);
  // apply with gather/scatter fused: x_b = src[gidx[i]] (i in boundary order), result written
  // as dst[gidx[i]] = y_i (+ add[gidx[i]] if add != nullptr).  T is the vector type.
  template <class T>
  void apply_gather(const T* src, const int32_t* gidx, T* dst, const T* add, T* yb, cudaStream_t s);
  // R right-hand sides at once (hmat_multi.cu): for state r, x_r(b) = src[g_r(b)] and
  // dst[g_r(b)] = y_r(b) (+ add[g_r(b)]), g_r(b) = gidx[goff[r] + b] with an index array, else
  // goff[r] + b; yb[yoff[r] + b] = y_r(b) when yb is given.  goff / yoff: host arrays of R.
  template <class T>
  void apply_multi(const T* src, const int32_t* gidx, const int64_t* goff, T* dst, const T* add, T* yb,
                   const int64_t* yoff, int R, cudaStream_t s);
  int64_t device_bytes() const;
  // H^T packed in the same precision: far blocks keep their factors with the roles of U^T and
  // V exchanged, near tiles are transposed (hio.cu).  Built once, kept in `tr`.
  HMatrix& transposed(cudaStream_t s);
};

// The reference's cache representation (hio.cu): near field as CSR in permutation space
// (zeros dropped), far blocks as meta (rs, re, cs, ce, k), relres, U (m x k), V (k x n).
void hmat_near_csr(const HMatrix& H, std::vector<int32_t>& indptr, std::vector<int32_t>& indices,
                   std::vector<double>& data);
void hmat_far_sizes(const HMatrix& H, int64_t& nfar, int64_t& u_entries, int64_t& v_entries);
void hmat_export_far(const HMatrix& H, int64_t* meta5, double* relres, double* U, double* V);
void hmat_import(HMatrix& H, const BoundaryDev& bd, const HBuildConfig& c, Prec p, int64_t nfar, const int64_t* meta5,
                 const double* relres, const double* U, const double* V, const int32_t* indptr,
                 const int32_t* indices, const double* data, const int32_t* perm_in, const double* diag_jump,
                 cudaStream_t s);

// Block-diagonal concatenation of packed H-matrices (same packing precision) for one apply
// over all of them (hio.cu); apply-side data only.
void hmat_merge(const std::vector<const HMatrix*>& parts, HMatrix& M, cudaStream_t s);

// tensor-core far field of the multi-state apply (hmat_tc.cu): tc_build packs the factors
// (needs the FP64 pools), tc_far_apply returns the far part of Y (perm order, [Nb][8] FP64)
// for the gathered X~ ([Nb][8]); tc_error reads the kernels' timeout flag
void tc_build(HMatrix& H, cudaStream_t s, int kstep_max = 0);
const double* tc_far_apply(HMatrix& H, const double* xm, cudaStream_t s);
int tc_error(HMatrix& H, cudaStream_t s);
int64_t tc_bytes(const HMatrix& H);

// y = H x (original boundary ordering, FP64) using the library's static device scratch
// instead of allocated buffers (see spx_hmat_apply_noalloc in include/spx.h).
void hmat_apply_noalloc(HMatrix& H, const double* x, double* y, cudaStream_t s);
extern std::atomic<int64_t> g_noalloc_cap;  // test cap on its accepted scratch (0: none)

}  // namespace spx
