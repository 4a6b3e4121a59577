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

template <class T> struct StageArgs;

template <class T>
struct LLGCtx {
  int device = 0;
  int64_t N = 0;
  LLGParams prm;
  DemagCtx<T>* demag = nullptr;
  HostFem own_fem;
  HostSell own_sell;
  DevSell<T> P;
  DevBuf<T> Kex, Kd, ani_n, ani_p, H0, diagK;
  double ani_p0 = 0.0, h0[3] = {0, 0, 0};
  double pref = 0, stab = 0, c1 = 0, c2 = 0;
  bool has_dmi = false, has_ani = false, use_demag = false, pc_ready = false;
  DevBuf<T> m, ms0, ms1, acc, tmp, tmp2, Mstate, Hm, pcinv;
  DevBuf<double> red;
  int64_t steps = 0, rhs_evals = 0;
  mutable int64_t launches = 0;

  void create(DemagCtx<T>* dm, const double* X, int64_t N, const int32_t* tets, int64_t E, const LLGParams& p,
              cudaStream_t s);
  StageArgs<T> args(const T* min, T* out, int mode, bool with_demag) const;
  void launch_stage(const StageArgs<T>& a, bool with_demag, cudaStream_t s) const;
  void heff(const T* m, T* H, bool with_demag, cudaStream_t s);
  void rhs(const T* m, T* out, cudaStream_t s);
  void step_rk4(double dt, int64_t nsteps, cudaStream_t s);
  void update_jac_state(const T* m, cudaStream_t s);
  void jv(const T* v, T* out, cudaStream_t s);
  void pc_build(double shift, int include_stab, int use_abs_kappa, cudaStream_t s);
  void pc_apply(const T* x, T* y, cudaStream_t s);
  double mdoth(const double* w, const T* a, const T* b, cudaStream_t s);
};

template <class A, class B>
void convert(int64_t n, const A* src, B* dst, cudaStream_t s);

template <class T>
double demag_energy(DemagCtx<T>& d, const T* m, const T* H, cudaStream_t s);

}  // namespace spx
