// FEM operators on the device, the persistent CG solver and the demag pipeline.
#pragma once

#include "hmat.cuh"

namespace spx {

struct CgStats {
  int64_t iterations = 0;
  double rel_residual = 0.0;
  int converged = 0;
};

// Scaled SPD system  A^ = D^-1/2 A D^-1/2  on a SELL-32 pattern, solved by a pipelined
// CG (one grid barrier per iteration) in one cooperative launch.
template <class T>
struct CgSystem {
  int64_t n = 0;
  DevSell<T> P;
  DevBuf<T> vals;    // scaled values
  DevBuf<T> sdinv;   // 1/sqrt(d)
  DevBuf<T> diag;    // d (for the unscaled residual norm)
  DevBuf<T> work;    // 7 vectors of n
  DevBuf<double> red;
  DevBuf<unsigned int> bar;
  DevBuf<int> err;
  DevBuf<int> iters;
  DevBuf<double> resid;
  DevBuf<unsigned long long> iters_acc;
  // FP32 systems: FP64 values and state for the iterative-refinement solve
  DevBuf<double> vals64, sdinv64, diag64, y64, bh64;
  double inner_rtol = 1e-3;
  int max_outer = 8;
  int grid = 0;
  void setup(const HostSell& s, const std::vector<double>& vals_sell, const std::vector<double>& d);
  // solve A x = b; x holds the initial guess if warm; project: remove the constant null space
  CgStats solve(const T* b, T* x, double rtol, double atol, int maxit, bool warm, bool project,
                cudaStream_t st, bool sync_stats = true);
};

// Per-category CUDA-event timing of the demag/LLG pipeline (enabled on demand; events
// are recorded on the launching stream around each kernel group).
enum ProfCat : int { PC_DIV = 0, PC_CG1 = 1, PC_BND = 2, PC_U2RHS = 3, PC_CG2 = 4, PC_PHI = 5, PC_STAGE = 6, PC_N = 8 };
struct Profiler {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  std::vector<int> cat;
  size_t used = 0;
  int64_t launches[PC_N] = {};
  int64_t groups[PC_N] = {};
  void mark(int c, cudaStream_t s) {  // call before and after a group: pairs (start, stop)
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

struct DemagOptions {
  int backend = 0;          // 0 dense, 1 hmatrix
  Prec prec = Prec::F64;    // vector / solver precision (F64 or F32) and H storage
  double rtol_u1 = 1e-6, rtol_u2 = 1e-6, atol = 1e-12;
  int maxit_u1 = 2000, maxit_u2 = 12000;
  int warm_start = 0;
  HBuildConfig hcfg;
};

template <class T>
struct DemagCtx {
  int device = 0;
  int64_t N = 0, E = 0, Nb = 0, NI = 0;
  double Ms = 0.0, mu0 = 4e-7 * 3.141592653589793;
  DemagOptions opt;
  BoundaryDev bd;
  HostFem fem;
  // full pattern (all nodes)
  HostSell hsell;
  DevSell<T> P;
  DevBuf<T> Div;        // 3 planes, Ms * int grad v . m
  DevBuf<T> Gv;         // 3 planes, G / vol_i  (H = Gv phi)
  DevBuf<double> vol;   // lumped nodal volume
  DevBuf<int32_t> interior, bverts;
  CgSystem<T> cg1, cg2;
  DevSell<T> PIB;       // interior rows x boundary columns
  DevBuf<T> AIB;
  DevBuf<double> Bdense;
  HMatrix H;
  // work
  DevBuf<T> b, u1, phi, gB, bI, xI, xb, yb;
  DevBuf<double> sum;
  CgStats last1, last2;
  int64_t applies = 0;
  Profiler prof;
  int64_t launches = 0;
  void create(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms, const DemagOptions& o,
              cudaStream_t s);
  // potential phi = u1 + u2 for magnetisation m (AoS, T)
  void potential(const T* m, cudaStream_t s, bool sync_stats);
  // H_demag = G phi / vol (AoS)
  void field(T* H, cudaStream_t s);
  int64_t device_bytes() const;
};

}  // namespace spx
