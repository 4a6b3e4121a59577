// FEM operators on the device, the persistent CG solvers and the demag pipeline.
//
// Precision: DemagCtx<TV, TM> keeps nodal vectors (m, u1, u2, phi, b, g) in TV and the large
// matrices (Div, G/V, the CG values) in TM.
//   <double, double>  FP64 everywhere, pipelined FP64 CG
//   <float,  float>   plain FP32 (FP32 CG inside FP64 iterative refinement, FP32 vectors)
//   <double, float>   mixed: FP64 vectors, FP32 matrices, FP32 inner CG + FP64 refinement
// Operators whose rows sum to zero (G, exchange) are applied in difference form
// sum_j a_ij (v_j - v_i), and Div as sum_j D_ij (m_j - m_i) + (sum_j D_ij) m_i, so a
// rounded matrix value multiplies a small nodal difference instead of a large value.
#pragma once

#include <memory>

#include <nvtx3/nvToolsExt.h>

#include "amg.cuh"
#include "hmat.cuh"

namespace spx {

struct CgStats {
  int64_t iterations = 0;
  double rel_residual = 0.0;
  int converged = 0;
};

// Per-category CUDA-event timing of the demag/LLG pipeline (enabled on demand; events
// are recorded on the launching stream around each kernel group).  Every group is also an
// NVTX range of the same name (seen by Nsight Systems / Compute; a no-op without a tool).
enum ProfCat : int { PC_DIV = 0, PC_CG1 = 1, PC_BND = 2, PC_U2RHS = 3, PC_CG2 = 4, PC_PHI = 5, PC_STAGE = 6, PC_N = 8 };
inline const char* prof_cat_name(int c) {
  static const char* const names[PC_N] = {"div", "u1_solve", "boundary_apply", "u2_rhs", "u2_solve", "phi", "stage",
                                          "other"};
  return c >= 0 && c < PC_N ? names[c] : "other";
}
struct Profiler {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  std::vector<int> cat;
  size_t used = 0;
  int64_t launches[PC_N] = {};
  int64_t groups[PC_N] = {};
  bool nvtx_open[PC_N] = {};
  void mark(int c, cudaStream_t s) {  // call before and after a group: pairs (start, stop)
    if (c >= 0 && c < PC_N) {  // groups do not nest: a push on the start mark, a pop on the stop
      if (nvtx_open[c]) nvtxRangePop();
      else nvtxRangePushA(prof_cat_name(c));
      nvtx_open[c] = !nvtx_open[c];
    }
    if (!on) return;
    if ((used & 1) == 0) groups[c]++;
    if (used == pool.size()) {
      cudaEvent_t e;
      SPX_CUDA(cudaEventCreate(&e));
      pool.push_back(e);
      cat.push_back(c);
    }
    cat[used] = c;
    SPX_CUDA(cudaEventRecord(pool[used++], s));
  }
  void begin() {
    on = true;
    used = 0;
    for (auto& l : launches) l = 0;
    for (auto& g : groups) g = 0;
  }
  void end(double* ms, int64_t* nl, int64_t* ng) {
    for (int c = 0; c < PC_N; ++c) { ms[c] = 0.0; nl[c] = launches[c]; ng[c] = groups[c]; }
    if (used) SPX_CUDA(cudaEventSynchronize(pool[used - 1]));
    for (size_t k = 0; k + 1 < used; k += 2) {
      float t = 0.f;
      SPX_CUDA(cudaEventElapsedTime(&t, pool[k], pool[k + 1]));
      ms[cat[k]] += t;
    }
    on = false;
    used = 0;
  }
  ~Profiler() {
    for (auto e : pool) cudaEventDestroy(e);
  }
};

// Scaled SPD system  A^ = D^-1/2 A D^-1/2  on a SELL-32 pattern solved in one cooperative
// launch: TM = double -> pipelined FP64 CG (one grid barrier per iteration); TM = float ->
// FP32 single-reduction CG inside FP64 iterative refinement (FP64 values kept for the
// true residual, FP64 solution state kept between calls).
//
// Starting guesses: with `slot` >= 0 the solver keeps the last five solutions returned
// for that slot (e.g. one slot per RK stage) and starts from their quartic extrapolation
// 5 x1 - 10 x2 + 10 x3 - 5 x4 + x5 (lower orders while fewer are stored; measured on the
// 400x400x2 film: u1 6.2 iterations per solve with the quartic start, 6.4 with the cubic
// and 7.3 with the quadratic one).  The stopping
// rule does not change; only the iteration count does.  Slots 0-3: forward RK stages,
// 4-7: adjoint stages, 8-11: tangent stages (CG_SLOTS).
constexpr int CG_SLOTS = 12;
constexpr int CG_HIST = 5;  // stored solutions per slot (quartic extrapolation)

template <class TM>
struct CgSystem {
  int64_t n = 0;       // unknowns: reps blocks of n1 rows
  int64_t n1 = 0;      // rows of the stored matrix
  int reps = 1;        // identical diagonal blocks sharing the stored matrix (AMG path only)
  DevSell<TM> P;
  DevBuf<TM> vals;     // scaled values
  DevBuf<double> vals64, sdinv64, diag64, y64, bh64;  // FP64 data of the refinement solve
  DevBuf<TM> sdinv;    // 1/sqrt(d) (pipelined FP64 path)
  DevBuf<TM> diag;
  DevBuf<char> work;   // solver vectors
  DevBuf<double> part;  // per-CTA partial sums [3 slots][grid][4]
  DevBuf<double> red;   // scalars
  DevBuf<unsigned int> bar;
  DevBuf<int> err;
  DevBuf<int> iters;
  DevBuf<double> resid;
  DevBuf<unsigned long long> iters_acc;  // [0] inner iterations, [1] refinement steps, [2] solves
  DevBuf<double> res_acc;                // [0] sum of initial, [1] sum of final relative residuals
  DevBuf<double> hist[CG_SLOTS][CG_HIST];
  int hcount[CG_SLOTS] = {}, hhead[CG_SLOTS] = {};
  // the ring bookkeeping of `count` slots from `first` as a solve on each leaves it (a replayed
  // CUDA graph runs the solves' kernels without this host code)
  void advance_slots(int first, int count) {
    for (int s = first; s < first + count && s < CG_SLOTS; ++s) {
      hhead[s] = (hhead[s] + 1) % CG_HIST;
      hcount[s] = hcount[s] + 1 < CG_HIST ? hcount[s] + 1 : CG_HIST;
    }
  }
  // stage correction: slots 1..3 add slot 0's last prediction error (solution - guess)
  bool stage_correct = false, have_pred0 = false, have_delta = false;
  // kind of the last solve (0 forward, 1 adjoint, 2 tangent): a warm start from the solver
  // state (y64 or x) is taken only from a solve of the same kind, whose right-hand sides
  // have the same scale; otherwise the solve starts from zero
  int last_kind = 0;
  // singular systems made of several independent components (ensembles): node offsets of
  // the components; a projected solve removes every component's mean from the right-hand
  // side (each component's system must be consistent on its own) and from the solution
  DevBuf<int64_t> seg_off;
  int seg_maxch = 0;          // chunks of the largest component (component-mean kernels)
  DevBuf<double> seg_part;    // chunk sums [components][seg_maxch]
  void set_segments(const std::vector<int64_t>& offsets, cudaStream_t s);
  DevBuf<char> bseg;  // right-hand side with every component's mean removed (TV)
  DevBuf<double> pred0, delta;
  double inner_rtol = 1e-3;
  int max_outer = 10;
  int grid = 0, block = 0;
  // AMG-preconditioned FP64 CG (k_pcg_amg) instead of the Jacobi solvers when enabled
  std::unique_ptr<AmgDevice> amg;
  DevBuf<double> amg_work;  // r, p, q
  DevBuf<float> amg_a32;    // unscaled values on the SELL pattern (FP32)
  DevBuf<double> amg_rsum;  // row sums of the unscaled matrix
  double amg_ww = 0.0;
  bool amg_singular = false;
  int amg_grid = 0;
  // nrep > 1: the system is nrep copies of this block on the diagonal (vectors of nrep x rows)
  void setup(const HostSell& s, const std::vector<double>& vals_sell, const std::vector<double>& d, int nrep = 1);
  // build the AMG hierarchy of D^-1/2 A D^-1/2 from the CSR of A (same rows as setup)
  void enable_amg(const HostSell& hs, const std::vector<int64_t>& rowptr, const std::vector<int32_t>& col, const std::vector<double>& a,
                  const std::vector<double>& d, bool singular, cudaStream_t s);
  template <class TV>
  void launch_amg(const TV* b, TV* x, double rtol, double atol, int maxit, bool warm, bool project, cudaStream_t st,
                  bool bh_given = false);
  // kind: 0 forward, 1 adjoint, 2 tangent; -1 derives it from the slot (0-3, 4-7, 8-11)
  template <class TV>
  CgStats solve(const TV* b, TV* x, double rtol, double atol, int maxit, bool warm, bool project, int slot,
                cudaStream_t st, bool sync_stats, int kind = -1);
  void reset_history() {
    for (int s = 0; s < CG_SLOTS; ++s) hcount[s] = hhead[s] = 0;
    have_pred0 = have_delta = false;
  }
};

// Block-diagonal boundary operator of an ensemble (a disjoint union of independent sample
// meshes, ensemble.cu): each sample's Lindholm operator over its own boundary only.  Samples
// with Nb <= dense_max_nb keep a dense block (TM precision, all blocks applied by one
// batched launch); larger ones an H-matrix built on the sample's own boundary.
struct BlockBoundary {
  int64_t nsamples = 0;
  std::vector<int64_t> b0, nb;        // per sample: first boundary row (union order), count
  std::vector<int> dense;             // per sample: 1 dense block, 0 H-matrix
  int64_t ndense = 0, dense_rows = 0, dense_entries = 0, ntiles = 0, max_ld = 0;
  DevBuf<int32_t> d_tiles;            // [ntiles][2]: dense sample, first row of a 64-row tile
  DevBuf<int64_t> d_b0, d_nb, d_off;  // per dense sample: boundary offset, Nb, pool offset
  DevBuf<char> pool;                  // dense blocks, row-major per sample (TM)
  std::vector<std::unique_ptr<HMatrix>> H;  // per sample while building (null for dense samples)
  // all H-matrix samples merged into one block-diagonal H-matrix (one apply for all)
  std::unique_ptr<HMatrix> Hm;
  // samples of one geometry: one H-matrix and the members' first boundary rows
  struct Shared {
    std::unique_ptr<HMatrix> H;
    std::vector<int64_t> b0;
  };
  std::vector<Shared> shared;
  DevBuf<int32_t> hidx;               // merged boundary index -> ensemble vertex
  DevBuf<int32_t> hmap;               // merged boundary index -> ensemble boundary row
  DevBuf<char> gbh;                   // merged-order result (TV)
  int64_t device_bytes() const;
};

struct DemagOptions;
template <class TM>
void block_boundary_build(BlockBoundary& bb, const BoundaryDev& bd, const double* X, int64_t N, const int32_t* tets,
                          int64_t E, const DemagOptions& o, cudaStream_t s);
// g = B u1|bnd per sample, phi[bverts] = u1 + g; returns the number of launches
template <class TV, class TM>
int block_boundary_apply(BlockBoundary& bb, int64_t Nb, const int32_t* bverts, const TV* u1, TV* xb, TV* phi, TV* gB,
                         cudaStream_t s);

struct DemagOptions {
  int backend = 0;          // 0 dense, 1 hmatrix, 2 block-diagonal ensemble (BlockBoundary)
  Prec prec = Prec::F64;    // vector / matrix precision of the pipeline
  Prec hprec = Prec::F64;   // storage precision of the H-matrix factors
  double rtol_u1 = 1e-6, rtol_u2 = 1e-6, atol = 1e-12;
  int maxit_u1 = 2000, maxit_u2 = 12000;
  int warm_start = 0;       // 0 zero start, 1 previous solution, 2 extrapolated per RK stage,
                            // 3 as 2, stages 2-4 corrected by stage 1's prediction error
  int u1_pc = 0;            // u1 preconditioner: 0 smoothed-aggregation AMG, 1 Jacobi
  HMatrix* preset = nullptr;  // hmatrix backend: adopt this H-matrix (moved in) instead of building
  HBuildConfig hcfg;
  // ensemble backend: sample s owns nodes [sample_offsets[s], sample_offsets[s + 1])
  std::vector<int64_t> sample_offsets;
  int64_t dense_max_nb = 4096;
};

// Transposed operators of the demag map m -> H, built on first use of
// DemagCtx::apply_transpose (adjoint.cu).
template <class TV, class TM>
struct DemagAdjoint {
  bool ready = false;
  DevBuf<TM> GvT;          // 3 planes: GvT_c(j, i) = Gv_c(i, j)
  DevBuf<double> GvTsum;   // [3][N] row sums of GvT
  DevBuf<TM> DivT;         // 3 planes: DivT_c(j, i) = Div(i, (j, c)); rows sum to zero
  DevSell<double> PBI;     // boundary rows (bverts order) x interior columns of A
  DevBuf<double> ABI;
  DevBuf<double> part;     // dense B^T partial sums
  DevBuf<TV> psi, bIbar, xIbar, gbar, yb, u1bar, bbar;
};

template <class TV, class TM>
struct DemagCtx {
  int device = 0;
  int64_t N = 0, E = 0, Nb = 0, NI = 0;
  double Ms = 0.0, mu0 = 4e-7 * 3.141592653589793;
  DemagOptions opt;
  BoundaryDev bd;
  HostFem fem;
  HostSell hsell;
  DevSell<TM> P;
  DevBuf<TM> Div;        // 3 planes, Ms * int grad v . m
  DevBuf<double> Dsum;   // [3][N] row sums of Div (boundary flux terms)
  DevBuf<TM> Gv;         // 3 planes, G / vol_i
  DevBuf<double> vol;
  DevBuf<int32_t> interior, bverts;
  CgSystem<TM> cg1, cg2;
  DevSell<TM> PIB;
  DevBuf<double> AIB;    // interior rows x boundary columns, FP64
  DevBuf<double> Bdense;
  HMatrix H;
  BlockBoundary blk;
  DevBuf<TV> b, u1, phi, gB, bI, xI, xb;
  CgStats last1, last2;
  int64_t applies = 0;
  int64_t epoch = 0;   // solves issued outside a captured step (invalidates step graphs)
  Profiler prof;
  int64_t launches = 0;
  void create(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms, const DemagOptions& o,
              cudaStream_t s);
  // potential phi = u1 + u2 for magnetisation m (AoS, TV); slot: RK stage for extrapolated starts
  void potential(const TV* m, cudaStream_t s, bool sync_stats, int slot = -1);
  // host bookkeeping of one RK4 step's four stage solves (slots 0-3) for a step replayed
  // from a CUDA graph, so that later captures and ordinary steps see the rings as they are
  void replay_step_advance() {
    if (opt.warm_start >= 2) {
      cg1.advance_slots(0, 4);
      cg2.advance_slots(0, 4);
    }
  }
  // H_demag = G phi / vol (AoS)
  void field(TV* H, cudaStream_t s);
  // out (+)= D^T w for the linear map D: m -> H_demag (AoS, 3N); slot: adjoint RK stage (4-7)
  // or -1.  The two Poisson solves are the forward ones (symmetric), with their own slots.
  DemagAdjoint<TV, TM> adj;
  void apply_transpose(const TV* w, TV* out, bool accumulate, int slot, cudaStream_t s);
  int64_t device_bytes() const;
};

}  // namespace spx
