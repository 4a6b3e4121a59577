// LLG context: effective field, RHS, Jv, block preconditioner and RK4 stepping.
#pragma once

#include "fem.cuh"

namespace spx {

struct LLGParams {
  double Ms = 8e5, gamma = 2.211e5, alpha = 0.5, do_precess = 1.0;
  double Aex = 0.0;
  double Ku = 0.0;
  const double* Ku_nodes = nullptr;  // [N] per-node Ku (spatial Ku(x)); overrides Ku
  const double* n_ani = nullptr;     // [3N]
  double D_int = 0.0;
  const double* n_int = nullptr;     // [3N] interface normal
  const double* H0_nodes = nullptr;  // [3N] static field (A/m)
  double H0_uniform[3] = {0.0, 0.0, 0.0};
  int use_demag = 1;
};

template <class TV, class TM> struct StageArgs;

// TV: nodal vector type, TM: operator value type (see DemagCtx)
template <class TV, class TM>
struct LLGCtx {
  int device = 0;
  int64_t N = 0;
  LLGParams prm;
  DemagCtx<TV, TM>* demag = nullptr;
  HostFem own_fem;
  HostSell own_sell;
  DevSell<TM> P;
  DevBuf<TM> Kex, Kd;        // exchange (difference form) and DMI 3x3 blocks
  DevBuf<double> Ksum;       // [9][N] row sums of the DMI blocks
  DevBuf<TV> ani_n, ani_p, H0, diagK;
  double ani_p0 = 0.0, h0[3] = {0, 0, 0};
  double pref = 0, stab = 0, c1 = 0, c2 = 0;
  bool has_dmi = false, has_ani = false, use_demag = false, pc_ready = false;
  DevBuf<TV> m, ms0, ms1, acc, Mstate, Hm, pcinv;
  DevBuf<double> red;
  int64_t steps = 0, rhs_evals = 0;
  mutable int64_t launches = 0;

  void create(DemagCtx<TV, TM>* dm, const double* X, int64_t N, const int32_t* tets, int64_t E,
              const LLGParams& p, cudaStream_t s);
  StageArgs<TV, TM> args(const TV* min, TV* out, int mode, bool with_demag) const;
  void launch_stage(const StageArgs<TV, TM>& a, bool with_demag, cudaStream_t s) const;
  void heff(const TV* m, TV* H, bool with_demag, cudaStream_t s);
  void rhs(const TV* m, TV* out, cudaStream_t s);
  void step_rk4(double dt, int64_t nsteps, cudaStream_t s);
  void update_jac_state(const TV* m, cudaStream_t s);
  void jv(const TV* v, TV* out, cudaStream_t s);
  void pc_build(double shift, int include_stab, int use_abs_kappa, cudaStream_t s);
  void pc_apply(const TV* x, TV* y, cudaStream_t s);
};

template <class A, class B>
void convert(int64_t n, const A* src, B* dst, cudaStream_t s);

template <class TV, class TM>
double demag_energy(DemagCtx<TV, TM>& d, const TV* m, const TV* H, cudaStream_t s);

}  // namespace spx
