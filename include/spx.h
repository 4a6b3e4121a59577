/* libspx: B200 (sm_100a) FEM/BEM demagnetising field and LLG right-hand side.
 *
 * Drop-in C ABI for the hot path of the SpinFEMx GPU backend
 * (NanoPilot1/FEniCSx-Micromagnetics, package src/spinfemx).  Every entry point
 * is extern "C", takes plain pointers and sizes, returns an int status (SPX_OK
 * on success) and never throws or exits; the message of the last failure on the
 * calling thread is returned by spx_last_error().
 *
 * Conventions
 *   - mesh coordinates X [N][3] in nm (the unit the reference's operators assume,
 *     gpu/fields/Exchange_GPU.py:62), tets [E][4] int32 vertex ids;
 *   - nodal vectors are AoS FP64 device pointers [N][3], the layout of the
 *     reference's PETSc CUDA Vec with block size 3 (gpu/solvers/llg_module_GPU.py:25-39);
 *   - "device" pointers are CUDA device memory of the current device; calls are
 *     ordered on the given stream (NULL = legacy default stream);
 *   - handles are not thread-safe; one handle per thread or external locking.
 */
#ifndef SPX_H
#define SPX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SPX_API __attribute__((visibility("default")))
#else
#define SPX_API
#endif

typedef struct CUstream_st* spx_stream_t; /* same type as cudaStream_t */

#define SPX_OK 0
#define SPX_ERR_INVALID 1
#define SPX_ERR_CUDA 2
#define SPX_ERR_OOM 3
#define SPX_ERR_NOT_CONVERGED 4
#define SPX_ERR_TIMEOUT 5
#define SPX_ERR_INTERNAL 6
#define SPX_ERR_NO_DEVICE 7

/* Precision codes.  They mean different things in the two places that take them:
 *
 *   code            spx_hmat_config.precision /        spx_demag_options.precision /
 *                   spx_hmat_repack (packed storage    spx_llg_params.precision (the whole
 *                   of the H-matrix apply)             demag + LLG pipeline)
 *   SPX_PREC_F64    FP64 far factors, FP64 near tiles  FP64 vectors, operators, solvers
 *   SPX_PREC_F32    FP32 far factors, FP32 near tiles  FP32 vectors, operators, CG
 *   SPX_PREC_MIXED  BF16 far factors, FP32 near tiles  FP64 vectors with FP32 operators: FP32
 *                   (compensated sums)                 AMG cycle / CG inside FP64 refinement
 *
 * An H-matrix apply always accumulates in the type of the vectors it is given (FP64 for
 * spx_hmat_apply).  With a pipeline precision of SPX_PREC_MIXED the H-matrix packing is
 * spx_hmat_config.precision (SPX_PREC_F32 by default in the Python layer); BF16 factors
 * (packing SPX_PREC_MIXED) do not meet a 1e-5 demag tolerance on thin films. */
#define SPX_PREC_F64 0
#define SPX_PREC_F32 1
#define SPX_PREC_MIXED 2
/* H-matrix packing only (spx_hmat_config.precision, spx_hmat_repack): factors recompressed
 * (SPX_HMAT_RECOMPRESS, implied) with the leading columns of each far block in FP32 and the
 * trailing ones, whose FP16 rounding stays within a tenth of the block's epsilon budget, as
 * FP16 unit vectors scaled by their singular values; FP32 near tiles.  A transposed apply
 * packs its transpose in FP32; ensembles (merged H-matrices) do not take it. */
#define SPX_PREC_F32_F16 3

/* ------------------------------------------------------------------ library */
SPX_API const char* spx_last_error(void);
SPX_API int spx_version(void);
/* number of visible CUDA devices (0 without a GPU; never fails) */
SPX_API int spx_device_count(int32_t* n);
/* Failure-detection probe (no counterpart in the reference, which has no bounded waits): runs
 * a grid barrier on nblocks CTAs (2 .. number of SMs) that one CTA never reaches.  The others'
 * bounded waits run out after `limit` polls (1 .. 2^24) and return; *status receives the error
 * code the device recorded (SPX_ERR_TIMEOUT) and *timed_out_ctas how many CTAs gave up.  The
 * context stays usable.  Returns SPX_OK when the probe ran. */
SPX_API int spx_debug_barrier_probe(int32_t nblocks, int64_t limit, int32_t* status, int32_t* timed_out_ctas);
/* Cost of the grid barrier that separates the phases of the persistent solvers: nbarriers
 * barriers in a row on nblocks CTAs (1 .. number of SMs) of `threads` threads, timed with CUDA
 * events on a cooperative launch; *us_per_barrier = microseconds per barrier. */
SPX_API int spx_debug_barrier_time(int32_t nblocks, int32_t threads, int32_t nbarriers, double* us_per_barrier);
/* Per-phase time of the AMG-PCG kernel: spx_debug_pcg_timing(1) makes later launches record,
 * for 32 phase slots (V-cycle phases in order: pre-smoothing, residual and restriction per
 * level down, the coarse solve, prolongation and two post-smoothing sweeps per level up; 28
 * the PCG product, 29 the update, 30 the true residual), the nanoseconds from the previous
 * phase end to this one's as CTA 0 saw them (the slowest CTA's work plus the barrier).
 * spx_debug_pcg_phase_times returns the summed times and sample counts and clears them. */
SPX_API int spx_debug_pcg_timing(int32_t enable);
SPX_API int spx_debug_pcg_phase_times(double* ns32, int64_t* counts32);
/* The L2 set-aside for persisting accesses of this process's context (raised by the AMG setup
 * to hold the cycle's matrices, which it loads with an evict_last policy) and the device's
 * maximum, in bytes. */
SPX_API int spx_device_l2_persisting(int64_t* current_bytes, int64_t* max_bytes);
/* Out-of-memory injection for tests of the recovery paths (no counterpart in the reference,
 * whose builder catches CuPy's OutOfMemoryError, lindholm_hmatrix_gpu/builder.py:597-662):
 * the next `count` device allocations of the library of at least `min_bytes` bytes fail with
 * SPX_ERR_OOM on the host, before cudaMalloc is called (count 0 switches it off). */
SPX_API int spx_debug_fail_alloc(int64_t min_bytes, int32_t count);
/* Lowers the scratch size that spx_hmat_apply_noalloc accepts to `bytes` (0: back to its
 * 32 MiB), so that its refusal of a too-large H-matrix can be tested on a small one. */
SPX_API int spx_debug_noalloc_cap(int64_t bytes);

/* ------------------------------------------------------------------ host geometry
 * Boundary data of build_boundary_data_serial (gpu/fields/Demag_Lindholm.py:177-285):
 * outward boundary triangles in a canonical order (sorted ascending vertex triples),
 * Xb in ascending vertex order, omega_sum = sum over tets of |solid angle|. */
SPX_API int spx_boundary_sizes(const double* X, int64_t N, const int32_t* tets, int64_t E, int64_t* Nb, int64_t* Nt);
/* any output may be NULL; sizes Nb / Nt from spx_boundary_sizes */
SPX_API int spx_boundary_data(const double* X, int64_t N, const int32_t* tets, int64_t E, int32_t* bverts,
                      int32_t* tri_lid, double* Xb, double* ntri, double* area, double* omega_sum);
/* P1 operators of gpu/fields/Demag_Lindholm_GPU.py:188-261, 554-567 and the lumped
 * volume of llg_module_GPU.py:469-484 on the scalar node pattern (CSR, sorted columns):
 * A = int grad u.grad v ; Div[k*3+c] = int d_c(v_i) phi_j (multiply by Ms) ;
 * G[k*3+c] = -int phi_i d_c(phi_j) ; vol = int phi_i. */
SPX_API int spx_fem_sizes(const double* X, int64_t N, const int32_t* tets, int64_t E, int64_t* nnz);
SPX_API int spx_fem_assemble(const double* X, int64_t N, const int32_t* tets, int64_t E, int64_t* rowptr, int32_t* col,
                     double* A, double* Div, double* G, double* vol);
/* cluster-tree permutation of gpu/fields/lindholm_hmatrix_gpu/tree.py:41-96 (bit-exact) */
SPX_API int spx_cluster_tree(const double* pts, int64_t n, int32_t leaf_size, int32_t* perm);

/* ------------------------------------------------------------------ boundary geometry on the device */
typedef struct spx_boundary_s* spx_boundary;
SPX_API int spx_boundary_create(const double* X, int64_t N, const int32_t* tets, int64_t E, spx_boundary* out);
SPX_API int spx_boundary_destroy(spx_boundary b);
SPX_API int spx_boundary_info(spx_boundary b, int64_t* Nb, int64_t* Nt, int32_t* max_incident);
/* Lindholm weights (gpu/fields/Lindholm_kernel.py:66-125, CUDA twin
 * lindholm_hmatrix_gpu/entry_provider_gpu.py:94-203) for P targets x0 [P][3] against
 * boundary triangles tri [P]; w [P][3].  Device pointers. */
SPX_API int spx_lindholm_pairs(spx_boundary b, const double* x0, const int32_t* tri, int64_t P, double* w,
                       spx_stream_t s);
/* B[rows, cols] without the diagonal jump, row-major m x n (LindholmEntryProviderGPU.fill_block_device,
 * entry_provider_gpu.py:687-750; CPU entry_provider.py:41-117).  rows/cols: device int32 boundary ids. */
SPX_API int spx_lindholm_fill_block(spx_boundary b, const int32_t* rows, int64_t m, const int32_t* cols, int64_t n,
                            double* out, spx_stream_t s);
/* dense Nb x Nb row-major B including diag Omega/4pi - 1 (assemble_B_rows_owned,
 * gpu/fields/Demag_Lindholm.py:51-116) */
SPX_API int spx_dense_b_assemble(spx_boundary b, double* B, spx_stream_t s);
/* y = B x (cp.matmul in DemagFieldLindholmGPU._apply_B_gpu, Demag_Lindholm_GPU.py:600-605) */
SPX_API int spx_dense_b_apply(const double* B, int64_t Nb, const double* x, double* y, spx_stream_t s);

/* ------------------------------------------------------------------ H-matrix */
typedef struct spx_hmat_s* spx_hmat;
typedef struct {
  double epsilon;                    /* ACA tolerance (HMatrixBuildConfig.epsilon, builder.py:24-95) */
  double eta;                        /* admissibility */
  int32_t leaf_size;
  int32_t max_rank;                  /* <= 0: no limit */
  int64_t max_temporary_block_bytes; /* forced subdivision above this dense size */
  int32_t precision;                 /* SPX_PREC_* of the packed apply data */
  int32_t flags;                     /* SPX_HMAT_RECOMPRESS: SVD-recompress the ACA factors after the build */
  int64_t batch_bytes;               /* device workspace per fill/ACA batch (0: default) */
} spx_hmat_config;
/* flags: after the ACA build, rewrite every far block (rank <= 64) from the SVD of its core,
 * truncated to the smallest rank that keeps ||A - U V||_F <= epsilon ||A||_F given its ACA
 * residual (checked a posteriori per block; no counterpart in the reference, whose builder
 * stores the ACA factors; its truncated_svd compressor, compressors.py:102-235, is the same
 * family applied to dense blocks).  Columns come out in decreasing singular value, which the
 * SPX_PREC_F32_F16 packing needs. */
#define SPX_HMAT_RECOMPRESS 1
/* build: cluster tree, block partition, GPU fill and full-pivot ACA
 * (HMatrixBuilder.build / build_or_load_hmatrix, builder.py:186-419, 814-927) */
SPX_API int spx_hmat_build(spx_boundary b, const spx_hmat_config* cfg, spx_hmat* out);
/* stats[16]: dense_blocks, low_rank_blocks, rejected_low_rank_blocks, forced_subdivisions_memory,
 * compression_tolerance_subdivisions, max_observed_rank, sum_observed_rank, block_entry_evaluations,
 * near_entries, far_entries, n_far, n_near, aca_steps, waves, Nb, 0 */
SPX_API int spx_hmat_stats(spx_hmat h, int64_t* stats16, double* build_seconds);
SPX_API int spx_hmat_num_blocks(spx_hmat h, int64_t* n);
/* blocks [n][6]: row_start, row_stop, col_start, col_stop, is_far, rank (permuted coordinates) */
SPX_API int spx_hmat_blocks(spx_hmat h, int64_t* out6, int64_t capacity);
SPX_API int spx_hmat_perm(spx_hmat h, int32_t* perm);
/* y = H x in the original boundary ordering (HMatrixGPUPackedFused.matvec, backend_fused.py:496-512) */
SPX_API int spx_hmat_apply(spx_hmat h, const double* x, double* y, spx_stream_t s);
SPX_API int spx_hmat_repack(spx_hmat h, int32_t precision);
/* SVD recompression of the far factors (see SPX_HMAT_RECOMPRESS) of a built or imported
 * H-matrix, repacked in its current precision; out3 = (far factor entries before, after,
 * blocks rewritten), *max_rel_err = the largest truncation error of a block relative to its
 * norm.  No counterpart in the reference. */
SPX_API int spx_hmat_recompress(spx_hmat h, int64_t* out3, double* max_rel_err);
/* y = H x like spx_hmat_apply, for callers that cannot allocate device memory while they
 * run: a solver callback whose device memory is owned by another allocator (a PETSc or
 * framework memory pool that must not be bypassed), or a loop that may not stall on
 * cudaMalloc.  No counterpart in the reference.  This entry point allocates nothing: its
 * scratch lives in one fixed 32 MiB device array that every GPU loading libspx holds until
 * exit.  The scratch is FP64 whatever the packing: x in permuted order (Nb), the far-field
 * z vectors (sum of ranks) and the partial sums of far blocks split between warps (zpart),
 * (Nb + zlen + zpart_len) x 8 bytes with each part rounded up to 256 bytes, i.e. about 4.19M
 * elements for every packing; larger H-matrices are rejected with SPX_ERR_INVALID.  The
 * first call on a device looks up that array's device address with cudaGetSymbolAddress
 * and keeps it for the life of the process, so make the first call on each device before
 * any stream capture, and do not reset the device (cudaDeviceReset) afterwards.  All calls
 * share the array and overwrite it completely (nothing in it has to start at zero), so
 * calls that overlap on the GPU (other streams, other threads) race; serialise them.
 * x, y: FP64 device vectors of length Nb. */
SPX_API int spx_hmat_apply_noalloc(spx_hmat h, const double* x, double* y, spx_stream_t s);
/* Y = H X for nrhs vectors at once (no counterpart in the reference, whose fused apply takes one
 * vector): X and Y hold nrhs FP64 device vectors of length Nb one after the other (vector r at
 * X + r Nb).  Each packed factor vector read from memory serves all nrhs products (FP64
 * accumulation), so the factor traffic of an apply is shared; batches above 8 are applied in
 * chunks of at most 8.  Results equal nrhs calls of spx_hmat_apply up to rounding. */
SPX_API int spx_hmat_apply_multi(spx_hmat h, const double* X, double* Y, int32_t nrhs, spx_stream_t s);
/* Tensor cores for spx_hmat_apply_multi (no counterpart in the reference): with enable != 0,
 * batches of 8 states run their far field as two block-sparse GEMMs on tcgen05 (column
 * clusters: Z = V X; row clusters: Y += U Z) with exact integer products: the FP32 factors as
 * 31-bit fixed-point values per tile row and the FP64 states as 47-bit fixed-point values,
 * cut into base-256 int8 digits (kind::i8, exact int32 digit-pair sums per tile of at most
 * 2048 K elements, FP64 combination and FP64 sums of the tiles); the near field and diagonal
 * on the CUDA cores.  Builds the digit plan (about the FP32 factor bytes plus tile padding;
 * *plan_bytes = device bytes of the plan); enable = 0 drops it.  The plan holds the factors
 * rounded to FP32 whatever the packing (with an FP64 packing the tensor-core far field is
 * that of the FP32 packing).  Needs the H-matrix's FP64 factors (built or imported, not
 * merged); spx_hmat_recompress drops the plan.  spx_hmat_tc_status returns (and clears) the
 * timeout flag of its kernels (SPX_ERR_TIMEOUT if a bounded wait ran out, else SPX_OK). */
/* enable = 2 autotunes: one 8-state apply is timed on the CUDA-core kernels and on tensor-core
 * tiles of 512 and of 2048 K elements, and the fastest is kept (*plan_bytes = 0 when the
 * CUDA cores win). */
SPX_API int spx_hmat_tensor_cores(spx_hmat h, int32_t enable, int64_t* plan_bytes);
SPX_API int spx_hmat_tc_status(spx_hmat h, int32_t* status);
/* y = H^T x (original boundary ordering, FP64 device vectors of length Nb).  No counterpart
 * in the reference (its H-matrix backends apply H only); the adjoint of the demag operator
 * needs it.  The transposed H-matrix (same cluster tree, transposed partition, far factors
 * shared with U^T and V exchanged, near tiles transposed) is packed in the same precision on
 * the first call and kept with the handle; spx_hmat_repack drops it. */
SPX_API int spx_hmat_apply_transpose(spx_hmat h, const double* x, double* y, spx_stream_t s);
/* low-rank factors U^T (k x m) and V (k x n) of far block `index` (as listed by spx_hmat_blocks), FP64 host */
SPX_API int spx_hmat_far_factors(spx_hmat h, int64_t index, double* Ut, double* V);
SPX_API int spx_hmat_memory(spx_hmat h, int64_t* far_bytes, int64_t* near_bytes, int64_t* total_bytes);
/* frees a handle made by spx_hmat_build / spx_hmat_import; handles lent by a demag object
 * (spx_demag_hmat, spx_demag_ensemble_hmat) are refused: they go with the demag object */
SPX_API int spx_hmat_destroy(spx_hmat h);
/* The reference's cache contents (HMatrixCPUData, lindholm_hmatrix_gpu/storage.py:29-325; the
 * npz file itself is read and written by numpy in the Python layer):
 *   perm[Nb]; diag_jump[Nb] (original order); near field as CSR in permutation space with exact
 *   zeros dropped (indptr[Nb+1], indices, data); far blocks as far_meta5[nfar][5] =
 *   (row_start, row_stop, col_start, col_stop, rank), relres[nfar], U_flat (m x k row-major
 *   per block), V_flat (k x n row-major per block), blocks in the same order.
 * export_sizes computes the near CSR and must precede export (HMatrixCPUData.save, :72-149). */
SPX_API int spx_hmat_export_sizes(spx_hmat h, int64_t* nfar, int64_t* u_entries, int64_t* v_entries,
                                  int64_t* near_nnz);
SPX_API int spx_hmat_export(spx_hmat h, int32_t* perm, double* diag_jump, int64_t* far_meta5, double* relres,
                            double* U, double* V, int32_t* near_indptr, int32_t* near_indices, double* near_data);
/* HMatrixCPUData.load (:151-209) + upload: the cluster tree is rebuilt from the boundary and
 * must reproduce `perm`; the near CSR becomes dense leaf x leaf tiles; packed in
 * cfg->precision.  diag_jump may be NULL (then taken from the boundary's solid angles). */
SPX_API int spx_hmat_import(spx_boundary b, const spx_hmat_config* cfg, const int32_t* perm, const double* diag_jump,
                            int64_t nfar, const int64_t* far_meta5, const double* relres, const double* U,
                            const double* V, const int32_t* near_indptr, const int32_t* near_indices,
                            const double* near_data, spx_hmat* out);

/* ------------------------------------------------------------------ demag field */
typedef struct spx_demag_s* spx_demag;
typedef struct {
  int32_t backend;   /* 0 dense, 1 hmatrix (DemagFieldLindholmGPU boundary_backend, :319-345) */
  int32_t precision; /* SPX_PREC_* */
  double rtol_u1, rtol_u2, atol; /* ksp_rtol_u1/u2 (:216-226, :271-281), atol 1e-12 */
  int32_t maxit_u1, maxit_u2;    /* 2000 / 12000 in the reference */
  int32_t warm_start;            /* 0 zero start (reference), 1 previous solution, 2 extrapolated per RK stage,
                                    3 as 2 with stages 2-4 corrected by stage 1's prediction error */
  int32_t u1_preconditioner;     /* 0 smoothed-aggregation AMG (the reference's PC "gamg", :219-222), 1 Jacobi */
  spx_hmat_config hmat;
} spx_demag_options;
/* DemagFieldLindholmGPU.__init__ (gpu/fields/Demag_Lindholm_GPU.py:101-155) */
SPX_API int spx_demag_create(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms,
                     const spx_demag_options* opt, spx_demag* out);
/* DemagFieldLindholmGPU.compute_vec (:643-670): H = -grad(u1+u2) lumped, AoS FP64 device */
/* DemagFieldLindholmGPU with an H-matrix from build_or_load_hmatrix (Demag_Lindholm_GPU.py:
 * 377-430): opt->backend must be 1; the H-matrix is moved into the demag object (h keeps no
 * data afterwards and is still destroyed by the caller) and repacked if opt->hmat.precision
 * differs from its packing */
SPX_API int spx_demag_create_with_hmat(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms,
                                       const spx_demag_options* opt, spx_hmat h, spx_demag* out);
/* Ensemble of independent samples (batched form; no counterpart in the reference, which runs
 * one mesh per object): X / tets is the disjoint union of the samples' meshes, sample s owning
 * nodes [node_offsets[s], node_offsets[s+1]) (node_offsets[0] = 0, node_offsets[nsamples] = N)
 * and the tetrahedra that reference them.  FEM operators, both Poisson solves and
 * spx_demag_apply run once for all samples; the boundary operator is block diagonal: the
 * Lindholm operator of each sample's own boundary, dense (one batched launch for all dense
 * samples) when the sample's Nb <= dense_max_nb, else an H-matrix with opt->hmat; samples
 * of one geometry (equal up to a translation) share one H-matrix applied to all of them at
 * once, and 2, 4 or 8 samples whose stiffness matrices are identical share the u1 matrix and
 * AMG hierarchy.  opt->backend is ignored.  spx_demag_apply_transpose is not available for
 * ensembles. */
/* out6 = (samples, dense samples, dense block entries, boundary rows of the merged H-matrix of
 * the other samples, its far-factor bytes, its near-tile bytes); zeros for a non-ensemble */
SPX_API int spx_demag_ensemble_info(spx_demag d, int64_t* out6);
/* H-matrix shared by the samples of geometry group `group` of an ensemble (lent like
 * spx_demag_hmat, valid while d lives; groups are numbered in order of their first sample) */
SPX_API int spx_demag_ensemble_hmat(spx_demag d, int32_t group, spx_hmat* h);
SPX_API int spx_demag_create_ensemble(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms,
                                      const spx_demag_options* opt, int64_t nsamples, const int64_t* node_offsets,
                                      int64_t dense_max_nb, spx_demag* out);
SPX_API int spx_demag_apply(spx_demag d, const double* m, double* H, spx_stream_t s);
/* out = D^T w for the linear demag map D: m -> H of spx_demag_apply (AoS FP64 device,
 * length 3N).  No counterpart in the reference.  Evaluated as
 * Div^T Pi A^+ Pi (psi + E^T B^T (psi_B - A_BI A_II^-1 psi_I)) with psi = (G/V)^T w: the
 * same two CG solves as the forward map (symmetric systems) and B^T (transposed dense GEMV
 * or spx_hmat_apply_transpose's operator); the transposed value planes are built on the
 * first call. */
SPX_API int spx_demag_apply_transpose(spx_demag d, const double* w, double* out, spx_stream_t s);
/* potentials of the last apply (FP64 device, N each) */
SPX_API int spx_demag_potentials(spx_demag d, double* u1, double* u2, spx_stream_t s);
/* Energy_lumped_gpu (:706-724): E = -1/2 mu0 Ms sum V_i m.H / 1e27  (J) */
SPX_API int spx_demag_energy(spx_demag d, const double* m, const double* H, double* E, spx_stream_t s);
/* last_its_u1 / last_its_u2 and the relative residuals of the last apply */
SPX_API int spx_demag_stats(spx_demag d, int64_t* its_u1, int64_t* its_u2, double* res_u1, double* res_u2);
SPX_API int spx_demag_info(spx_demag d, int64_t* N, int64_t* Nb, int64_t* NI, int64_t* device_bytes);
/* H-matrix of an hmatrix-backend demag (borrowed, valid while d lives; every spx_hmat call
 * accepts it, spx_hmat_destroy and spx_demag_create_with_hmat refuse it) */
SPX_API int spx_demag_hmat(spx_demag d, spx_hmat* h);
SPX_API int spx_demag_destroy(spx_demag d);

/* ------------------------------------------------------------------ LLG */
typedef struct spx_llg_s* spx_llg;
typedef struct {
  double Ms, gamma, alpha, do_precess; /* LLG_GPU(mesh, Ms, gamma, alpha, do_precess), llg_module_GPU.py:1549 */
  double Aex;                          /* add_exchange */
  double Ku;                           /* add_anisotropy (uniform) */
  const double* Ku_nodes;              /* [N] per-node Ku, or NULL */
  const double* n_ani;                 /* [N][3] easy axes, or NULL */
  double D_int;                        /* add_dmi_interfacial */
  const double* n_int;                 /* [N][3] interface normal, or NULL */
  const double* H0_nodes;              /* [N][3] static field (A/m), or NULL */
  double H0_uniform[3];                /* set_uniform_field */
  int32_t use_demag;
  int32_t precision;                   /* used when d == NULL; otherwise the demag's precision */
  /* Zhang-Li spin-transfer torque (LLG_STT_GPU.add_current, llg_stt_module_GPU.py:1409-1414;
   * EffectiveFieldSTTGPU, :523-590): current density J (A/m^2), polarisation P, non-adiabaticity
   * beta, nodal current direction [N][3] (NULL: no STT) */
  double stt_J, stt_P, stt_beta;
  const double* stt_dir;
  /* spin-orbit torque (EffectiveFieldSOTGPU.set_sot, llg_SOT_module_GPU.py:812-862): damping-like
   * and field-like fields (A/m), nodal polarisation [N][3] (normalised per node; NULL: no SOT) */
  double sot_Hdl, sot_Hfl;
  const double* sot_p;
  /* bulk DMI (LLG_GPU.add_dmi_bulk, DMIBULK in gpu/fields/DMI_Bulk_GPU.py:43-77): D (J/m^2) of
   * H = 2D/(mu0 Ms) M_lump^-1 K m, K = -curl + boundary term; 0 = none */
  double D_bulk;
} spx_llg_params;
/* EffectiveField.__init__ (llg_module_GPU.py:388-724); d may be NULL (no demag) */
SPX_API int spx_llg_create(spx_demag d, const double* X, int64_t N, const int32_t* tets, int64_t E,
                   const spx_llg_params* p, spx_llg* out);
SPX_API int spx_llg_heff(spx_llg l, const double* m, double* H, spx_stream_t s);   /* compute_H_eff_vec  :972-1006 */
SPX_API int spx_llg_hjac(spx_llg l, const double* m, double* H, spx_stream_t s);   /* compute_H_jac_vec  :1232-1257 */
SPX_API int spx_llg_rhs(spx_llg l, const double* m, double* rhs, spx_stream_t s);  /* llg_rhs_vec        :1261-1285 */
SPX_API int spx_llg_update_jac_state(spx_llg l, const double* m, spx_stream_t s); /* update_jac_state  :1287-1290 */
SPX_API int spx_llg_jv(spx_llg l, const double* v, double* out, spx_stream_t s);   /* jac_vec_times_vec  :1293-1323 */
/* JvContext.update_pc_full_fast_gpu (:1449-1507) and apply (:1519-1543) */
SPX_API int spx_llg_pc_build(spx_llg l, double shift, int32_t include_stab, int32_t use_abs_kappa, spx_stream_t s);
SPX_API int spx_llg_pc_apply(spx_llg l, const double* x, double* y, spx_stream_t s);
/* integrator state (FP64 device AoS) and fixed-step classic RK4 (4 RHS evaluations per step);
 * the reference steps with PETSc TS rk/5dp or BDF (llg_module_GPU.py:1724-1787, 2052-2181) */
SPX_API int spx_llg_set_state(spx_llg l, const double* m, spx_stream_t s);
SPX_API int spx_llg_get_state(spx_llg l, double* m, spx_stream_t s);
SPX_API int spx_llg_step(spx_llg l, double dt, int64_t nsteps, spx_stream_t s);
/* end-to-end call with HOST buffers: copy m_in to the device, run nsteps, copy the
 * result back (pinned host memory gives full PCIe/C2C bandwidth) */
SPX_API int spx_llg_run_host(spx_llg l, const double* m_in, double* m_out, double dt, int64_t nsteps);
/* Time-dependent applied field (EffectiveField H_time_func, llg_module_GPU.py:909-956; added
 * to H_eff at the current time, :998-1000).  The callback lives on the host side; these
 * calls take its values.
 *   spx_llg_set_time_field:  the field at the current time, used by spx_llg_heff / _hjac /
 *                            _rhs / _update_jac_state until changed: h_uniform3 host [3] or
 *                            NULL (zero) plus h_nodes device [N][3] or NULL; both add up.
 *   spx_llg_step_time_field: one classic RK4 step of size dt whose stage s (times t, t+dt/2,
 *                            t+dt/2, t+dt) adds h_uniform4x3[3s..3s+2] (host, or NULL) and
 *                            h_nodes4 + 3N s (device [4][N][3], or NULL). */
SPX_API int spx_llg_set_time_field(spx_llg l, const double* h_uniform3, const double* h_nodes, spx_stream_t s);
SPX_API int spx_llg_step_time_field(spx_llg l, double dt, const double* h_uniform4x3, const double* h_nodes4,
                                    spx_stream_t s);
/* Embedded explicit Runge-Kutta attempt (the reference's PETSc TS rk/5dp, llg_module_GPU.py:
 * 1724-1787; the step-size adaptor is the caller's, as PETSc's TSAdapt is outside the RHS).
 * scheme 0 = Dormand-Prince 5(4).  From the state, computes the 5th-order candidate of one
 * step of size dt (not committed) and *err_norm = sqrt(mean_i (e_i / tol_i)^2) over the 3N
 * entries, e the difference to the embedded 4th-order solution, tol_i = atol + rtol
 * max(|y5_i|, |y4_i|) (PETSc's weighted 2-norm).  Stage i (time t + c_i dt, c = 0, 1/5,
 * 3/10, 4/5, 8/9, 1, 1) adds h_uniform7x3[3i..] (host) and h_nodes7 + 3N i (device) when
 * given.  reuse_fsal != 0 takes stage 1 from the last accepted attempt's stage 7 (first same
 * as last) when that is still valid.  Reads one scalar back (synchronises the stream).
 * spx_llg_rk_accept makes the candidate the state. */
SPX_API int spx_llg_rk_attempt(spx_llg l, int32_t scheme, double dt, double rtol, double atol,
                               const double* h_uniform7x3, const double* h_nodes7, int32_t reuse_fsal,
                               double* err_norm, spx_stream_t s);
SPX_API int spx_llg_rk_accept(spx_llg l, spx_stream_t s);
/* Implicit BDF(2) attempt: the stage solves of the reference's implicit driver
 * (LLG_GPU._ensure_solver / relax, llg_module_GPU.py:2052-2381: PETSc TS bdf, SNES newtonls
 * with the bt line search of order 2, KSP gmres left-preconditioned by JvContext's 3x3 block
 * inverse, operator shift I - J, residual ydot - f).  The step-size adaptor is the caller's.
 *   spx_bdf_default_opts: the reference's options (ts rtol/atol 1e-6, snes rtol 1e-2, atol
 *       1e-4, stol 1e-8, divtol 1e4, max 8 its; ksp rtol 1e-4, atol 1e-50, dtol 1e5, max 200
 *       its, restart 30; line search alpha 1e-4, min lambda 1e-12, max step 1e8, max 40 its;
 *       use_pc 1 = the block preconditioner, 0 = none).
 *   spx_llg_bdf_attempt: from the state at time t, one step of size dt (not committed).  With
 *       no history (after create, set_state, any other stepping call or bdf_reset) a
 *       backward-Euler half step to t + dt/2 comes first.  h_uniform2x3 (host [2][3]) and
 *       h_nodes2 (device [2][N][3]) are the time-dependent field at t + dt/2 and t + dt, or
 *       NULL.  Fills *r: snes_reason (> 0 converged: 2 |F| < atol, 3 |F| <= rtol |F_0|,
 *       4 small step; < 0 the attempt failed), wlte (weighted RMS local error estimate,
 *       tol_i = atol + rtol max(|y_i|, |m_i|)), order (of the estimate, for the adaptor's
 *       exponent -1/order), restarted, and the Newton / GMRES iterations and RHS evaluations.
 *   spx_llg_bdf_accept: makes a converged attempt the state and shifts the history. */
typedef struct {
  double rtol, atol;
  double snes_rtol, snes_atol, snes_stol, snes_divtol;
  double ksp_rtol, ksp_atol, ksp_dtol;
  double ls_alpha, ls_minlambda, ls_maxstep;
  int32_t snes_max_it, ksp_max_it, ksp_restart, ls_max_it;
  int32_t use_pc, reserved;
} spx_bdf_opts;
typedef struct {
  double wlte;
  int32_t snes_reason, order, restarted, newton_its, linear_its, fevals;
} spx_bdf_result;
SPX_API int spx_bdf_default_opts(spx_bdf_opts* o);
SPX_API int spx_llg_bdf_attempt(spx_llg l, double t, double dt, const spx_bdf_opts* o, const double* h_uniform2x3,
                                const double* h_nodes2, spx_bdf_result* r, spx_stream_t s);
SPX_API int spx_llg_bdf_accept(spx_llg l, spx_stream_t s);
SPX_API int spx_llg_bdf_reset(spx_llg l);
/* max over nodes of |a_i - b_i| for FP64 device AoS vectors [N][3] (StopByMaxDmdtFDGPU's
 * max |du|, llg_module_GPU.py:355-359) */
SPX_API int spx_vec_node_diff_max(const double* a, const double* b, int64_t N, double* out, spx_stream_t s);
/* EffectiveField.set_uniform_field (llg_module_GPU.py:897-904): replace the static field by a uniform one */
SPX_API int spx_llg_set_uniform_field(spx_llg l, double hx, double hy, double hz);
/* Adjoint and tangent products (no counterpart in the reference, which has no gradients).
 * Vectors are FP64 device AoS of length 3N.  gKu (length N) and gH0 (length 3) are FP64
 * device accumulators: the call ADDS dL/dKu_i (J/m^3, per node) and dL/dH0 (A/m, uniform
 * applied field) to them; either may be NULL.  gKu needs an anisotropy axis given at
 * creation.
 *   spx_llg_set_anisotropy_map: replace the nodal Ku map (host, N values, J/m^3).
 *   spx_llg_rhs_vjp:  mbar = J(m)^T w, J the Jacobian of llg_rhs_vec (demag included).
 *   spx_llg_step_vjp: lam_out = (d m_{n+1}/d m_n)^T lam_in for one classic RK4 step of
 *                     size dt from m_n (the four stages are recomputed); lam_out may be
 *                     lam_in.
 *   spx_llg_step_jvp: one RK4 step of the state and of its tangent: m_out = step(m_n),
 *                     dm_out = d step . (dm, dKu, dH0); dKu: device N or NULL, dH0: host 3
 *                     or NULL. */
/* Spin torques.  With spx_llg_params.stt_dir set, spx_llg_rhs / spx_llg_step include the Zhang-Li
 * torque (llg_rhs_STT_vec, llg_stt_module_GPU.py:1054-1085), spx_llg_jv the STT Jacobian
 * (jac_vec_times_STT_vec, :1123-1163) and spx_llg_pc_build the STT block preconditioner
 * (JvContextSTT, :1248-1296); with sot_p set, the SOT forms (llg_rhs_SOT_vec,
 * llg_SOT_module_GPU.py:1069-1096; jac_vec_times_SOT_vec, :1114-1150; JvContextSOT, :1218-1251,
 * use_abs_kappa standing for use_abs_diag).
 *   spx_llg_zhang_li: out = (J . grad) m / V_i (ZhangLiGPU.compute_vec, :431-435).
 *   spx_llg_set_sot:  EffectiveFieldSOTGPU.set_sot (:855-862); polarization host [N][3] or NULL
 *                     (keep the current one), normalised per node. */
SPX_API int spx_llg_zhang_li(spx_llg l, const double* m, double* out, spx_stream_t s);
SPX_API int spx_llg_set_sot(spx_llg l, double H_dl, double H_fl, const double* polarization);
/* LaBonte / Barzilai-Borwein energy minimiser, device part (LaBonteBBMinimizerGPU,
 * Minimizer_GPU.py:171-845; the step-length and acceptance logic is host code, see
 * spinfemx_b200/minimizer.py).  FP64 device AoS vectors; out5 (host) = (E [J, lumped, as
 * compute_Energy_minimize_gpu, llg_module_GPU.py:1079-1229], max_i |d_i|, s.y, s.s, y.y).
 *   spx_llg_min_eval:  (m normalised in place when normalize != 0) d = H_eff(m) - (m.H_eff) m;
 *                      out5[2..4] = 0.
 *   spx_llg_min_trial: m_trial = Cayley step of m_old along d_old with step alpha
 *                      (_CAYLEY_KERNEL, :46-74), d_trial = projected field at m_trial,
 *                      s = m_trial - m_old, y = d_old - d_trial. */
SPX_API int spx_llg_min_eval(spx_llg l, double* m, double* d, int32_t normalize, double* out5, spx_stream_t s);
SPX_API int spx_llg_min_trial(spx_llg l, const double* m_old, const double* d_old, double alpha, double* m_trial,
                              double* d_trial, double* out5, spx_stream_t s);
/* CUDA graphs for spx_llg_step (no counterpart in the reference): with enable != 0, each RK4
 * step is replayed from captured graphs (five captures, one per phase of the per-stage Krylov
 * extrapolation history) after five ordinary steps; the graphs are recaptured when dt, the
 * applied field, the Ku map or the solver tolerances change or when any other call used the
 * demag solvers.  Results are those of ordinary steps.  spx_llg_graph_stats reports the steps
 * replayed from graphs and whether graphs are active; if capture failed, stepping continues
 * without graphs and spx_last_error holds the reason. */
SPX_API int spx_llg_set_graph(spx_llg l, int32_t enable);
SPX_API int spx_llg_graph_stats(spx_llg l, int64_t* replays, int32_t* active);
SPX_API int spx_llg_set_anisotropy_map(spx_llg l, const double* Ku_nodes);
SPX_API int spx_llg_rhs_vjp(spx_llg l, const double* m, const double* w, double* mbar, double* gKu, double* gH0,
                            spx_stream_t s);
SPX_API int spx_llg_step_vjp(spx_llg l, const double* m_n, double dt, const double* lam_in, double* lam_out,
                             double* gKu, double* gH0, spx_stream_t s);
SPX_API int spx_llg_step_jvp(spx_llg l, const double* m_n, const double* dm, const double* dKu, const double* dH0,
                             double dt, double* m_out, double* dm_out, spx_stream_t s);
/* CUDA-event timing of the pipeline by kernel group, recorded on the launching stream
 * between begin and end.  ms[8] / kernel launches[8] / group executions[8] per group: 0 Div SpMV, 1 u1 solve,
 * 2 boundary operator (gather + far + rows, or dense GEMV), 3 u2 right-hand side,
 * 4 u2 solve, 5 potential assembly, 6 fused field/RHS/RK stage, 7 unused.
 * counters[4]: CG inner iterations, refinement steps, solves (since create), 0. */
SPX_API int spx_demag_profile_begin(spx_demag d);
SPX_API int spx_demag_profile_end(spx_demag d, double* ms8, int64_t* launches8, int64_t* groups8);
SPX_API int spx_demag_counters(spx_demag d, int64_t* u1_counters4, int64_t* u2_counters4);
/* sums over all solves since create of the relative residual ||b - A x0||/||b|| at the
 * starting guess ([0]) and at return ([1]), for the u1 and u2 solves (no counterpart in
 * the reference: its KSP solves, Demag_Lindholm_GPU.py:577 and :640, report nothing) */
SPX_API int spx_demag_residuals(spx_demag d, double* u1_res2, double* u2_res2);
/* levels of the u1 AMG hierarchy (0 when u1 uses the Jacobi solver): per level rows,
 * nonzeros of A, P and R = P^T (the last level is the dense coarsest one; the reference's
 * PETSc GAMG hierarchy, Demag_Lindholm_GPU.py:219-222, is not exposed) */
SPX_API int spx_demag_amg_levels(spx_demag d, int64_t* levels4, int32_t max_levels, int32_t* nlev);
/* change the Krylov tolerances / iteration limits after create (the reference fixes them
 * with KSP.setTolerances, Demag_Lindholm_GPU.py:219 and :274) */
SPX_API int spx_demag_set_tolerances(spx_demag d, double rtol_u1, double rtol_u2, double atol, int32_t maxit_u1,
                                     int32_t maxit_u2);
/* steps, RHS evaluations, LLG kernel launches */
SPX_API int spx_llg_stats(spx_llg l, int64_t* steps, int64_t* rhs_evals, int64_t* launches);
SPX_API int spx_llg_destroy(spx_llg l);

#ifdef __cplusplus
}
#endif
#endif /* SPX_H */
