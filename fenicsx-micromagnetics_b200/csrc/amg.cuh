// Smoothed-aggregation algebraic multigrid for the scalar P1 Poisson systems.
//
// The reference preconditions its u1 Krylov solve with PETSc GAMG
// (gpu/fields/Demag_Lindholm_GPU.py:215-222: KSP "cg", PC "gamg").  This is a restatement
// of the same method family, set up on the host once per mesh and cycled on the device:
//   * strength of connection |a_ij| > theta sqrt(a_ii a_jj), three-pass greedy aggregation
//     (root + strong neighbours; attach leftovers to a neighbouring aggregate; group the
//     rest), in vertex order;
//   * tentative prolongator from the near-null vector w (piecewise w / ||w_aggregate||),
//     smoothed once: P = (I - omega D^-1 A) P0, omega = 4 / (3 lambda_max(D^-1 A));
//   * Galerkin coarse operators A_c = P^T A P, down to at most `coarse_max` unknowns, whose
//     dense inverse (with a rank-one term w w^T when the system is singular; Gauss-Jordan in
//     FP64 on the device at set-up) is applied exactly as a GEMV;
//   * V(2,2) cycle with Chebyshev-Jacobi smoothing on [0.1, 1.1] x lambda_max(D^-1 A)
//     (PETSc's default eigenvalue transform for GAMG level smoothers).
// The cycle runs in FP32 inside an FP64 preconditioned CG (k_pcg_amg in amg.cu).  The
// hierarchy is built for the Jacobi-scaled matrix D^-1/2 A D^-1/2; its finest level is cycled
// on the unscaled A (P_0 and R_0 absorb D^-1/2), so that the PCG and the cycle read one copy
// of the level-0 matrix.
#pragma once

#include <cuda_fp16.h>

#include "spx_internal.cuh"

namespace spx {

struct CsrHost {
  int64_t n = 0, ncols = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> ci;
  std::vector<double> v;
};

struct AmgOptions {
  double theta = 0.0;         // strength threshold (0: every nonzero off-diagonal is strong)
  int64_t coarse_max = 2500;  // dense coarsest level (inverted once, applied as a GEMV)
  int max_levels = 10;
  int power_iters = 20;
};

struct AmgHostLevel {
  CsrHost A, P, R;         // P: n x n_next, R = P^T
  std::vector<double> dinv;
  double lmax = 0.0;       // estimate of lambda_max(D^-1 A)
};

struct AmgHost {
  std::vector<AmgHostLevel> lv;      // lv.back() is the dense coarsest level (no P/R)
  std::vector<double> coarse_dense;  // n_c x n_c, row-major, SPD
};

// A: symmetric positive (semi)definite CSR with sorted columns; null: its near-null vector
// (A null = 0 when singular).
void amg_build(const CsrHost& A, const std::vector<double>& null, bool singular, const AmgOptions& o,
               AmgHost& out);

// Device side ---------------------------------------------------------------------------
struct AmgLevelDev {
  int64_t n, nslices;
  const int64_t* sp;       // A: SELL-32
  const int32_t* col;
  const float* val;
  const __half* val16;     // FP16 copy of val for the cycle's sweeps (null: val)
  const float* dinv;
  int64_t p_nslices;       // P: SELL-32, n rows
  const int64_t* p_sp;
  const int32_t* p_col;
  const float* p_val;
  const int64_t* r_rp;     // R = P^T: CSR, rows of the next level, `r_lanes` lanes per row
  const int32_t* r_col;
  const float* r_val;
  int r_lanes;
  float *b, *db, *x, *x2, *d, *r;  // db = D^-1 b
  float theta, delta, sigma;
};

struct AmgDevice {
  int nlev = 0;            // levels 0..nlev-2 are cycled, level nlev-1 is the dense coarsest
  int64_t n0 = 0, nc = 0, ldc = 0;  // ldc: row stride of the coarsest inverse (cinv)
  int reps = 1;
  std::vector<DevSell<float>> A, P;
  std::vector<DevBuf<int64_t>> rrp;
  std::vector<DevBuf<int32_t>> rcol;
  std::vector<DevBuf<float>> val, pval, rval, dinv, vec;
  std::vector<DevBuf<__half>> val16;  // FP16 sweep values (SPX_AMG_FP16)
  DevBuf<AmgLevelDev> lv;
  DevBuf<float> cinv;
  std::vector<int64_t> sizes, nnz, pnnz, rnnz;  // per level: rows, nonzeros of A, P, R
  // top0: when set, level 0's matrix is this SELL-32 (slice pointers, columns, FP32 values of
  // nslices0 slices) owned by the caller instead of a copy of lv[0].A
  // nrep: the cycle runs on nrep identical blocks at once (level vectors of nrep x rows)
  void upload(const AmgHost& h, cudaStream_t s, const int64_t* sp0 = nullptr, const int32_t* col0 = nullptr,
              const float* val0 = nullptr, int64_t nslices0 = 0, int nrep = 1);
  int64_t device_bytes() const;
};

}  // namespace spx
