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
  double D_bulk = 0.0;               // bulk DMI constant (J/m^2)
  const double* H0_nodes = nullptr;  // [3N] static field (A/m)
  double H0_uniform[3] = {0.0, 0.0, 0.0};
  int use_demag = 1;
  // Zhang-Li spin-transfer torque (gpu/solvers/llg_stt_module_GPU.py)
  double stt_J = 0.0, stt_P = 0.0, stt_beta = 0.0;
  const double* stt_dir = nullptr;   // [3N] current direction (null: no STT)
  // spin-orbit torque (gpu/solvers/llg_SOT_module_GPU.py)
  double sot_Hdl = 0.0, sot_Hfl = 0.0;
  const double* sot_p = nullptr;     // [3N] polarisation (null: no SOT)
};

// Arguments of the fused stage kernel k_stage (llg.cu)
template <class TV, class TM>
struct StageArgs {
  int64_t n, nslices;
  const int64_t* sp;
  const int32_t* col;
  int64_t L;
  const TM* Kex;     // [L] exchange, row-scaled
  const TM* Kd;      // [9L] DMI blocks, row-scaled (or null)
  const double* Ksum;  // [9n] DMI row sums
  const TM* Gv;      // [3L] G / vol (or null: no demag)
  const TV* phi;     // potential (or null)
  const TV* ani_n;   // [3n] unit axes (or null)
  const TV* ani_p;   // [n] per-node prefactor 2Ku/(mu0 Ms) (or null)
  TV ani_p0;         // scalar prefactor when ani_p == null
  const TV* H0;      // [3n] (or null)
  TV h0x, h0y, h0z;
  const TV* Ht;      // [3n] time-dependent applied field at this evaluation's time (or null)
  TV htx, hty, htz;  // its uniform part
  const TV* m;       // stage input (AoS)
  TV* out;           // mode 0: H ; mode 1: rhs ; mode 2: next stage m
  TV* mn;            // RK state (mode 2)
  TV* acc;           // RK accumulator (mode 2)
  TV pref, alpha, precess, stab;
  TV c_next, w_acc, dt6;
  int mode, stage;
  // spin torques: Zhang-Li operator (row-scaled, rows sum to zero; null: no STT) and its
  // output in mode 0 (zout, may be null); SOT polarisation (null: no SOT)
  const TM* Kz;
  TV* zout;
  TV prefZ, stt_a, stt_b;
  const TV* sot_p;
  TV c_fl, c_dl;
};

// Work data of the adjoint and tangent products (adjoint.cu), built on first use.
template <class TV, class TM>
struct LLGAdjoint {
  bool ready = false;
  DevBuf<TM> KexT, KdT;            // transposed exchange (1 plane) and DMI (9 planes)
  DevBuf<double> KexTsum, KdTsum;  // their row sums
  DevBuf<TV> Y[4], Hs[4], dY[2], u, w, a, ap, lam, acc, K, dK, dH;
  DevBuf<double> part;
};

// Options and outcome of one implicit BDF attempt (implicit.cu); the fields mirror
// spx_bdf_opts / spx_bdf_result of the C ABI.
struct ImplicitOpts {
  double rtol = 1e-6, atol = 1e-6;                                          // TS error tolerances
  double snes_rtol = 1e-2, snes_atol = 1e-4, snes_stol = 1e-8, snes_divtol = 1e4;
  double ksp_rtol = 1e-4, ksp_atol = 1e-50, ksp_dtol = 1e5;
  double ls_alpha = 1e-4, ls_minlambda = 1e-12, ls_maxstep = 1e8;
  int snes_max_it = 8, ksp_max_it = 200, ksp_restart = 30, ls_max_it = 40;
  int use_pc = 1;
};

struct ImplicitResult {
  double wlte = -1.0;   // weighted RMS local error estimate (< 0: none)
  int snes_reason = 0;  // > 0 converged, < 0 diverged (PETSc's SNESConvergedReason values)
  int order = 0;        // order of the error estimate for the step adaptor
  int restarted = 0;    // 1: no history, a backward-Euler half step came first
  int newton_its = 0, linear_its = 0, fevals = 0;
};

// History and work vectors of the implicit driver
template <class TV>
struct ImplicitWork {
  DevBuf<TV> hist[2];  // y_{n-1}, y_{n-2} (newest first)
  double t[2] = {0.0, 0.0};
  int n = 0;           // past points held (0: the next attempt restarts)
  DevBuf<TV> half, cand, pred, base, f, F, G, W, Y, t1, t2, V;
  DevBuf<double> part, mpart, dev;
  bool has_cand = false, cand_restart = false;
  double cand_t = 0.0, cand_th = 0.0, cand_t0 = 0.0;
  int64_t fevals = 0;
};

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
  DevBuf<TM> Kz;              // Zhang-Li operator / V_i on the node pattern (STT)
  DevBuf<TV> Zm, sotp;        // Z(M_state) (Jv / PC state), SOT polarisation
  bool has_stt = false, has_sot = false;
  double prefZ = 0.0, stt_a = 0.0, stt_b = 0.0, c_fl = 0.0, c_dl = 0.0, c3 = 0.0, c4 = 0.0;
  DevBuf<double> red;
  int64_t steps = 0, rhs_evals = 0;
  mutable int64_t launches = 0;
  // CUDA graphs of one RK4 step (set_graph): CG_HIST captures, one per phase of the Krylov
  // extrapolation ring (each step advances every slot's ring by one, period CG_HIST), replayed
  // in turn; dropped when dt, a field parameter or the solver state outside the graphs changes
  bool graph_on = false, graph_ok = false;
  cudaStream_t gstream = nullptr;
  cudaGraphExec_t gexec[CG_HIST] = {};
  int gphase = 0, gwarm = 0;
  double gdt = 0.0;
  int64_t gepoch = -1, graph_replays = 0;
  std::string graph_error;
  void graph_reset();
  // one classic RK4 step; htu (host [4][3]) / htn (device [4][3N]) optional per-stage
  // time-dependent fields (stage times t, t + dt/2, t + dt/2, t + dt)
  void step_once(double dt, cudaStream_t s, const double* htu = nullptr, const TV* htn = nullptr);
  // time-dependent applied field (EffectiveField.H_time_func, llg_module_GPU.py:909-956,
  // 998-1000): the value at the current time, added by heff / rhs / the Jacobian state
  double ht[3] = {0.0, 0.0, 0.0};
  DevBuf<TV> ht_nodes;  // [3N] nodal part (empty: none)
  void set_time_field(const double* h3, const TV* h_nodes, cudaStream_t s);
  // embedded explicit Runge-Kutta (drivers.cu): Dormand-Prince 5(4) with first-same-as-last,
  // the scheme of the reference's PETSc TS rk/5dp (llg_module_GPU.py:1724-1787)
  DevBuf<TV> rk_k[7], rk_y, rk_ynew;
  DevBuf<double> rk_part;
  bool rk_fsal = false;
  // one attempt of size dt from the state m: rk_ynew = 5th-order solution, returns the
  // weighted RMS norm of the embedded error (tol_i = atol + rtol max(|y5_i|, |y4_i|)).
  // htu (host [7][3]) / htn (device [7][3N]): per-stage time fields at t + c_i dt, or null.
  double rk_attempt(double dt, double rtol, double atol, const double* htu, const TV* htn, bool reuse_fsal,
                    cudaStream_t s);
  void rk_accept(cudaStream_t s);  // m = rk_ynew; k1 of the next attempt = k7 (FSAL)
  // implicit BDF(2) driver (implicit.cu): one attempt of size dt from (t, m), Newton-Krylov
  // stage solves; htu (host [2][3]) / htn (device [2][3N]) the time field at t + dt/2 and
  // t + dt, or null.  bdf_accept makes the candidate the state and shifts the history.
  ImplicitWork<TV> im;
  ImplicitResult bdf_attempt(double t, double dt, const ImplicitOpts& o, const double* htu, const TV* htn,
                             cudaStream_t s);
  void bdf_accept(cudaStream_t s);
  void bdf_reset() { im.n = 0; im.has_cand = false; }
  void im_alloc();
  void im_lin(int nv, const TV* const* v, const double* c, TV* out, cudaStream_t s);
  double im_dot(const TV* a, const TV* b, cudaStream_t s);
  void im_apply_A(double shift, const TV* v, TV* out, cudaStream_t s);
  void im_apply_P(const TV* x, TV* y, bool use_pc, cudaStream_t s);
  double im_residual(double shift, const TV* y, TV* F, cudaStream_t s);
  int im_gmres(double shift, const TV* b, TV* x, const ImplicitOpts& o, int* its, cudaStream_t s);
  int im_newton(double shift, TV* y, const ImplicitOpts& o, int* nits, int* lits, cudaStream_t s);
  LLGCtx() = default;
  LLGCtx(const LLGCtx&) = delete;
  LLGCtx& operator=(const LLGCtx&) = delete;
  ~LLGCtx();
  std::vector<double> diag_lin_host;        // [3N] diagonal of exchange + DMI (no anisotropy)
  std::vector<double> X_host, n_int_host;   // kept when DMI is on (adjoint set-up)
  std::vector<int32_t> tets_host;
  LLGAdjoint<TV, TM> adj;

  void create(DemagCtx<TV, TM>* dm, const double* X, int64_t N, const int32_t* tets, int64_t E,
              const LLGParams& p, cudaStream_t s);
  StageArgs<TV, TM> args(const TV* min, TV* out, int mode, bool with_demag) const;
  void launch_stage(const StageArgs<TV, TM>& a, bool with_demag, cudaStream_t s) const;
  void heff(const TV* m, TV* H, bool with_demag, cudaStream_t s);
  void rhs(const TV* m, TV* out, cudaStream_t s);
  void step_rk4(double dt, int64_t nsteps, cudaStream_t s);
  void update_jac_state(const TV* m, cudaStream_t s);
  void jv(const TV* v, TV* out, cudaStream_t s);
  // mode 0: LLG (+ STT terms when STT is on, JvContextSTT); 2: SOT column-wise build
  // (JvContextSOT.update_pc_full_fast_gpu(shift, use_abs_diag)), use_abs_kappa = use_abs_diag
  void pc_build(double shift, int include_stab, int use_abs_kappa, cudaStream_t s);
  // Z(m) = (J . grad) m / V_i (ZhangLiGPU.compute_vec)
  void zhang_li(const TV* m, TV* out, cudaStream_t s);
  void set_sot(double Hdl, double Hfl, const double* p_nodes, cudaStream_t s);
  void pc_apply(const TV* x, TV* y, cudaStream_t s);
  // adjoint / tangent products (adjoint.cu).  gKu [N] and gH0 [3] are FP64 device
  // accumulators (+=), either may be null.
  void adjoint_setup(cudaStream_t s);
  // out = J(m)^T w for the field H = H_eff(m) given; slot: CG slot of the demag solves
  void rhs_vjp(const TV* m, const TV* H, const TV* w, TV* out, double* gKu, double* gH0, int slot, cudaStream_t s);
  // lam_out = (d m_(n+1) / d m_n)^T lam_in for one RK4 step of size dt from mn
  void step_vjp(const TV* mn, double dt, const TV* lam_in, TV* lam_out, double* gKu, double* gH0, cudaStream_t s);
  // one RK4 step of the primal and of the tangent: m_out = step(mn), dm_out = d step . (dm, dKu, dH0)
  void step_jvp(const TV* mn, const TV* dm, const double* dKu, const double dH0[3], double dt, TV* m_out, TV* dm_out,
                cudaStream_t s);
  void set_ku_map(const double* Ku_nodes, cudaStream_t s);
  // energy minimiser (minimize.cu): d = projected field at m (m normalised first when asked),
  // out5 = (E [J], max |d|, s.y, s.s, y.y) with s, y relative to (m_old, d_old) when given
  DevBuf<double> minvol, minpart;
  DevBuf<TV> minH;
  void min_eval(TV* m, const TV* m_old, const TV* d_old, TV* d, bool normalize, double out5[5], cudaStream_t s);
  void min_trial(const TV* m_old, const TV* d_old, double alpha, TV* m_t, TV* d_t, double out5[5], cudaStream_t s);
};

template <class A, class B>
void convert(int64_t n, const A* src, B* dst, cudaStream_t s);

// max over nodes of |a_i - b_i| for AoS FP64 device vectors [n][3] (drivers.cu)
double node_diff_max(int64_t n, const double* a, const double* b, cudaStream_t s);

template <class TV, class TM>
double demag_energy(DemagCtx<TV, TM>& d, const TV* m, const TV* H, cudaStream_t s);

}  // namespace spx
