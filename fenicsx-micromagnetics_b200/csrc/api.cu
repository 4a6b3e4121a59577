// extern "C" entry points of libspx (declared in include/spx.h).
#include <algorithm>
#include <cstring>
#include <memory>

#include "../../include/spx.h"
#include "llg.cuh"

namespace spx {
namespace {
thread_local std::string g_last_error;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }
std::atomic<int64_t> g_fail_alloc_min_bytes{0};
std::atomic<int32_t> g_fail_alloc_count{0};
}  // namespace spx

using namespace spx;

#define API_BEGIN try {
#define API_END                                       \
  }                                                   \
  catch (const spx::Error& e) {                       \
    spx::set_last_error(e.what());                    \
    return e.code;                                    \
  }                                                   \
  catch (const std::bad_alloc&) {                     \
    spx::set_last_error("host allocation failed");    \
    return SPX_ERR_OOM;                               \
  }                                                   \
  catch (const std::exception& e) {                   \
    spx::set_last_error(e.what());                    \
    return SPX_ERR_INTERNAL;                          \
  }                                                   \
  return SPX_OK;

#define REQUIRE(p) SPX_CHECK((p) != nullptr, #p " must not be NULL")

static cudaStream_t S(spx_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// H-matrix packing precision (SPX_PREC_F32_F16 included)
static Prec to_hprec(int32_t p) {
  SPX_CHECK(p >= 0 && p <= 3, "H-matrix precision must be SPX_PREC_F64, _F32, _MIXED or _F32_F16");
  return static_cast<Prec>(p);
}

static Prec to_prec(int32_t p) {
  SPX_CHECK(p >= 0 && p <= 2, "precision must be SPX_PREC_F64, SPX_PREC_F32 or SPX_PREC_MIXED");
  return static_cast<Prec>(p);
}

static void check_mesh(const double* X, int64_t N, const int32_t* tets, int64_t E) {
  REQUIRE(X);
  REQUIRE(tets);
  SPX_CHECK(N > 3 && E > 0, "mesh needs at least 4 vertices and one tetrahedron");
  for (int64_t k = 0; k < 4 * E; ++k) SPX_CHECK(tets[k] >= 0 && tets[k] < N, "tet vertex id out of range");
}

static HBuildConfig to_hcfg(const spx_hmat_config* c) {
  HBuildConfig h;
  if (!c) return h;
  SPX_CHECK(c->epsilon > 0.0, "epsilon must be positive");
  SPX_CHECK(c->eta > 0.0, "eta must be positive");
  SPX_CHECK(c->leaf_size >= 1 && c->leaf_size <= 1024, "leaf_size must be in [1, 1024]");
  SPX_CHECK(c->max_temporary_block_bytes >= 8, "max_temporary_block_bytes is too small");
  h.epsilon = c->epsilon;
  h.eta = c->eta;
  h.leaf_size = c->leaf_size;
  h.max_rank = c->max_rank > 0 ? c->max_rank : -1;
  h.max_temporary_block_bytes = c->max_temporary_block_bytes;
  if (c->batch_bytes > 0) h.batch_bytes = c->batch_bytes;
  SPX_CHECK((c->flags & ~SPX_HMAT_RECOMPRESS) == 0, "unknown spx_hmat_config.flags bits");
  h.recompress = (c->flags & SPX_HMAT_RECOMPRESS) != 0;
  return h;
}

static void require_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    throw Error(ERR_NO_DEVICE, "no CUDA device is visible");
  }
}

struct spx_boundary_s {
  BoundaryDev bd;
};
struct spx_hmat_s {
  HMatrix own;             // the matrix of a handle made by spx_hmat_build / spx_hmat_import
  HMatrix* ext = nullptr;  // a borrowed view: the matrix of a demag object (which owns this handle)
  HMatrix& h() { return ext ? *ext : own; }
  // near field as CSR, computed by spx_hmat_export_sizes for spx_hmat_export
  std::vector<int32_t> near_indptr, near_indices;
  std::vector<double> near_data;
};
// ---- type-erased demag / LLG handles (precision chosen at create)
struct DemagBase {
  virtual ~DemagBase() = default;
  // handles lent out by spx_demag_hmat / spx_demag_ensemble_hmat (views of matrices this object
  // owns; they live as long as it does)
  std::vector<std::unique_ptr<spx_hmat_s>> views;
  spx_hmat view_of(HMatrix* H) {
    for (auto& v : views)
      if (v->ext == H) return v.get();
    views.push_back(std::make_unique<spx_hmat_s>());
    views.back()->ext = H;
    return views.back().get();
  }
  virtual int64_t N() const = 0;
  virtual void apply(const double* m, double* H, cudaStream_t s) = 0;
  virtual void potentials(double* u1, double* phi, cudaStream_t s) = 0;
  virtual double energy(const double* m, const double* H, cudaStream_t s) = 0;
  virtual CgStats last1() const = 0;
  virtual CgStats last2() const = 0;
  virtual void info(int64_t* N, int64_t* Nb, int64_t* NI, int64_t* bytes) const = 0;
  virtual HMatrix* hmat() = 0;
  virtual Profiler& prof() = 0;
  virtual void counters(unsigned long long a[4], unsigned long long b[4]) = 0;
  virtual void residuals(double a[2], double b[2]) = 0;
  virtual int amg_levels(int64_t* out, int maxl) = 0;
  virtual void set_tolerances(double r1, double r2, double at, int m1, int m2) = 0;
  virtual void apply_transpose(const double* w, double* out, cudaStream_t s) = 0;
  virtual void ensemble_info(int64_t* out6) const = 0;
  virtual HMatrix* shared_hmat(int idx) = 0;
};

template <class TV, class TM>
struct DemagImpl : DemagBase {
  DemagCtx<TV, TM> d;
  DevBuf<TV> tm, th;
  int64_t N() const override { return d.N; }
  void apply(const double* m, double* H, cudaStream_t s) override {
    if (sizeof(TV) == sizeof(double)) {
      d.potential(reinterpret_cast<const TV*>(m), s, true);
      d.field(reinterpret_cast<TV*>(H), s);
    } else {
      const int64_t n3 = 3 * d.N;
      if (!tm.n) { tm.alloc(n3); th.alloc(n3); }
      convert<double, TV>(n3, m, tm.p, s);
      d.potential(tm.p, s, true);
      d.field(th.p, s);
      convert<TV, double>(n3, th.p, H, s);
    }
  }
  void potentials(double* u1, double* phi, cudaStream_t s) override {
    if (u1) convert<TV, double>(d.N, d.u1.p, u1, s);
    if (phi) convert<TV, double>(d.N, d.phi.p, phi, s);
  }
  double energy(const double* m, const double* H, cudaStream_t s) override {
    if (sizeof(TV) == sizeof(double))
      return demag_energy<TV, TM>(d, reinterpret_cast<const TV*>(m), reinterpret_cast<const TV*>(H), s);
    const int64_t n3 = 3 * d.N;
    if (!tm.n) { tm.alloc(n3); th.alloc(n3); }
    convert<double, TV>(n3, m, tm.p, s);
    convert<double, TV>(n3, H, th.p, s);
    return demag_energy<TV, TM>(d, tm.p, th.p, s);
  }
  CgStats last1() const override { return d.last1; }
  CgStats last2() const override { return d.last2; }
  void info(int64_t* N, int64_t* Nb, int64_t* NI, int64_t* bytes) const override {
    if (N) *N = d.N;
    if (Nb) *Nb = d.Nb;
    if (NI) *NI = d.NI;
    if (bytes) *bytes = d.device_bytes();
  }
  HMatrix* hmat() override { return d.opt.backend == 1 ? &d.H : nullptr; }
  Profiler& prof() override { return d.prof; }
  void counters(unsigned long long a[4], unsigned long long b[4]) override {
    auto rd = [](DevBuf<unsigned long long>& src, unsigned long long* dst) {
      if (src.n) SPX_CUDA(cudaMemcpy(dst, src.p, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    };
    rd(d.cg1.iters_acc, a);
    rd(d.cg2.iters_acc, b);
  }
  void residuals(double a[2], double b[2]) override {
    auto rd = [](DevBuf<double>& src, double* dst) {
      if (src.n) SPX_CUDA(cudaMemcpy(dst, src.p, 2 * sizeof(double), cudaMemcpyDeviceToHost));
    };
    rd(d.cg1.res_acc, a);
    rd(d.cg2.res_acc, b);
  }
  int amg_levels(int64_t* out, int maxl) override {
    const AmgDevice* a = d.cg1.amg.get();
    if (!a) return 0;
    for (int l = 0; l < a->nlev && l < maxl; ++l) {
      out[4 * l + 0] = a->sizes[l];
      out[4 * l + 1] = a->nnz[l];
      out[4 * l + 2] = a->pnnz[l];
      out[4 * l + 3] = a->rnnz[l];
    }
    return a->nlev;
  }
  void set_tolerances(double r1, double r2, double at, int m1, int m2) override {
    ++d.epoch;  // captured step graphs hold the old tolerances
    d.opt.rtol_u1 = r1; d.opt.rtol_u2 = r2; d.opt.atol = at;
    d.opt.maxit_u1 = m1; d.opt.maxit_u2 = m2;
  }
  HMatrix* shared_hmat(int idx) override {
    if (idx < 0 || idx >= static_cast<int>(d.blk.shared.size())) return nullptr;
    return d.blk.shared[idx].H.get();
  }
  void ensemble_info(int64_t* o) const override {
    const BlockBoundary& b = d.blk;
    o[0] = b.nsamples;
    o[1] = b.ndense;
    o[2] = b.dense_entries;
    o[3] = b.Hm ? b.Hm->Nb : 0;
    o[4] = b.Hm ? b.Hm->bytes_far : 0;
    o[5] = b.Hm ? b.Hm->bytes_near : 0;
  }
  void apply_transpose(const double* w, double* out, cudaStream_t s) override {
    if (sizeof(TV) == sizeof(double)) {
      d.apply_transpose(reinterpret_cast<const TV*>(w), reinterpret_cast<TV*>(out), false, -1, s);
    } else {
      const int64_t n3 = 3 * d.N;
      if (!tm.n) { tm.alloc(n3); th.alloc(n3); }
      convert<double, TV>(n3, w, tm.p, s);
      d.apply_transpose(tm.p, th.p, false, -1, s);
      convert<TV, double>(n3, th.p, out, s);
    }
  }
};

struct spx_demag_s {
  std::unique_ptr<DemagBase> impl;
};

struct LLGBase {
  virtual ~LLGBase() = default;
  virtual void heff(const double* m, double* H, bool with_demag, cudaStream_t s) = 0;
  virtual void rhs(const double* m, double* r, cudaStream_t s) = 0;
  virtual void update_jac_state(const double* m, cudaStream_t s) = 0;
  virtual void jv(const double* v, double* o, cudaStream_t s) = 0;
  virtual void pc_build(double shift, int inc, int absk, cudaStream_t s) = 0;
  virtual void pc_apply(const double* x, double* y, cudaStream_t s) = 0;
  virtual void set_state(const double* m, cudaStream_t s) = 0;
  virtual void get_state(double* m, cudaStream_t s) = 0;
  virtual void step(double dt, int64_t n, cudaStream_t s) = 0;
  virtual void run_host(const double* in, double* out, double dt, int64_t n) = 0;
  virtual void set_uniform_field(double x, double y, double z) = 0;
  virtual void stats(int64_t* steps, int64_t* rhs, int64_t* launches) const = 0;
  virtual void rhs_vjp(const double* m, const double* w, double* out, double* gKu, double* gH0, cudaStream_t s) = 0;
  virtual void step_vjp(const double* mn, double dt, const double* lin, double* lout, double* gKu, double* gH0,
                        cudaStream_t s) = 0;
  virtual void step_jvp(const double* mn, const double* dm, const double* dKu, const double* dH0, double dt,
                        double* mo, double* dmo, cudaStream_t s) = 0;
  virtual void set_ku_map(const double* ku) = 0;
  virtual void zhang_li(const double* m, double* out, cudaStream_t s) = 0;
  virtual void set_sot(double Hdl, double Hfl, const double* p) = 0;
  virtual void min_eval(double* m, double* d, int normalize, double* out5, cudaStream_t s) = 0;
  virtual void min_trial(const double* m_old, const double* d_old, double alpha, double* mt, double* dt,
                         double* out5, cudaStream_t s) = 0;
  virtual void set_graph(int on) = 0;
  virtual void graph_stats(int64_t* replays, int32_t* active) const = 0;
  virtual std::string graph_error() const = 0;
  virtual void set_time_field(const double* h3, const double* hn, cudaStream_t s) = 0;
  virtual void step_time_field(double dt, const double* htu, const double* htn, cudaStream_t s) = 0;
  virtual double rk_attempt(double dt, double rtol, double atol, const double* htu, const double* htn, bool reuse,
                            cudaStream_t s) = 0;
  virtual void rk_accept(cudaStream_t s) = 0;
  virtual ImplicitResult bdf_attempt(double t, double dt, const ImplicitOpts& o, const double* htu,
                                     const double* htn, cudaStream_t s) = 0;
  virtual void bdf_accept(cudaStream_t s) = 0;
  virtual void bdf_reset() = 0;
};

template <class TV, class TM>
struct LLGImpl : LLGBase {
  LLGCtx<TV, TM> l;
  DevBuf<TV> ta, tb;
  DevBuf<double> hstage;
  static constexpr bool f64 = sizeof(TV) == sizeof(double);
  const TV* in(const double* p, cudaStream_t s) {
    if (f64) return reinterpret_cast<const TV*>(p);
    if (!ta.n) ta.alloc(3 * l.N);
    convert<double, TV>(3 * l.N, p, ta.p, s);
    return ta.p;
  }
  TV* outbuf(double* p) {
    if (f64) return reinterpret_cast<TV*>(p);
    if (!tb.n) tb.alloc(3 * l.N);
    return tb.p;
  }
  void out(double* p, cudaStream_t s) {
    if (!f64) convert<TV, double>(3 * l.N, tb.p, p, s);
  }
  void heff(const double* m, double* H, bool wd, cudaStream_t s) override {
    TV* o = outbuf(H);
    l.heff(in(m, s), o, wd, s);
    out(H, s);
  }
  void rhs(const double* m, double* r, cudaStream_t s) override {
    TV* o = outbuf(r);
    l.rhs(in(m, s), o, s);
    out(r, s);
  }
  void update_jac_state(const double* m, cudaStream_t s) override { l.update_jac_state(in(m, s), s); }
  void jv(const double* v, double* o, cudaStream_t s) override {
    TV* q = outbuf(o);
    l.jv(in(v, s), q, s);
    out(o, s);
  }
  void pc_build(double shift, int inc, int absk, cudaStream_t s) override { l.pc_build(shift, inc, absk, s); }
  void pc_apply(const double* x, double* y, cudaStream_t s) override {
    TV* q = outbuf(y);
    l.pc_apply(in(x, s), q, s);
    out(y, s);
  }
  void set_state(const double* m, cudaStream_t s) override {
    l.rk_fsal = false;
    l.bdf_reset();
    convert<double, TV>(3 * l.N, m, l.m.p, s);
  }
  void get_state(double* m, cudaStream_t s) override { convert<TV, double>(3 * l.N, l.m.p, m, s); }
  void step(double dt, int64_t n, cudaStream_t s) override {
    l.rk_fsal = false;
    l.bdf_reset();
    l.step_rk4(dt, n, s);
  }
  DevBuf<TV> tstage;
  // nodal stage fields [nst][3N] in the pipeline's vector type (FP64 pipelines use the caller's)
  const TV* stage_fields(const double* hn, int nst, cudaStream_t s) {
    if (!hn) return nullptr;
    if (f64) return reinterpret_cast<const TV*>(hn);
    if (tstage.n < static_cast<size_t>(nst * 3 * l.N)) tstage.alloc(static_cast<size_t>(nst) * 3 * l.N);
    convert<double, TV>(nst * 3 * l.N, hn, tstage.p, s);
    return tstage.p;
  }
  void set_time_field(const double* h3, const double* hn, cudaStream_t s) override {
    l.set_time_field(h3, stage_fields(hn, 1, s), s);
  }
  void step_time_field(double dt, const double* htu, const double* htn, cudaStream_t s) override {
    l.graph_reset();
    l.rk_fsal = false;
    l.bdf_reset();
    l.step_once(dt, s, htu, stage_fields(htn, 4, s));
  }
  double rk_attempt(double dt, double rtol, double atol, const double* htu, const double* htn, bool reuse,
                    cudaStream_t s) override {
    return l.rk_attempt(dt, rtol, atol, htu, stage_fields(htn, 7, s), reuse, s);
  }
  void rk_accept(cudaStream_t s) override {
    l.rk_accept(s);
    l.bdf_reset();
  }
  ImplicitResult bdf_attempt(double t, double dt, const ImplicitOpts& o, const double* htu, const double* htn,
                             cudaStream_t s) override {
    return l.bdf_attempt(t, dt, o, htu, stage_fields(htn, 2, s), s);
  }
  void bdf_accept(cudaStream_t s) override { l.bdf_accept(s); }
  void bdf_reset() override { l.bdf_reset(); }
  void run_host(const double* hin, double* hout, double dt, int64_t n) override {
    const int64_t n3 = 3 * l.N;
    cudaStream_t s = 0;
    if (!hstage.n) hstage.alloc(n3);
    SPX_CUDA(cudaMemcpyAsync(hstage.p, hin, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    convert<double, TV>(n3, hstage.p, l.m.p, s);
    l.bdf_reset();
    l.step_rk4(dt, n, s);
    convert<TV, double>(n3, l.m.p, hstage.p, s);
    SPX_CUDA(cudaMemcpyAsync(hout, hstage.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    SPX_CUDA(cudaStreamSynchronize(s));
  }
  void set_uniform_field(double x, double y, double z) override {
    l.graph_reset();
    l.rk_fsal = false;
    l.H0.release();
    l.h0[0] = x; l.h0[1] = y; l.h0[2] = z;
  }
  void stats(int64_t* st, int64_t* r, int64_t* la) const override {
    if (st) *st = l.steps;
    if (r) *r = l.rhs_evals;
    if (la) *la = l.launches;
  }
  DevBuf<TV> tc, td, te;
  TV* scratch(DevBuf<TV>& b) {
    if (!b.n) b.alloc(3 * l.N);
    return b.p;
  }
  // FP64 -> TV copy into a given scratch (FP64 pipelines use the caller's buffer)
  const TV* in_to(const double* p, DevBuf<TV>& b, cudaStream_t s) {
    if (f64) return reinterpret_cast<const TV*>(p);
    convert<double, TV>(3 * l.N, p, scratch(b), s);
    return b.p;
  }
  TV* out_of(double* p, DevBuf<TV>& b) { return f64 ? reinterpret_cast<TV*>(p) : scratch(b); }
  void back(double* p, DevBuf<TV>& b, cudaStream_t s) {
    if (!f64) convert<TV, double>(3 * l.N, b.p, p, s);
  }
  void rhs_vjp(const double* m, const double* w, double* o, double* gKu, double* gH0, cudaStream_t s) override {
    l.adjoint_setup(s);
    const TV* mm = in_to(m, ta, s);
    const TV* ww = in_to(w, tc, s);
    TV* oo = out_of(o, tb);
    l.heff(mm, l.adj.Hs[0].p, true, s);
    l.rhs_vjp(mm, l.adj.Hs[0].p, ww, oo, gKu, gH0, -1, s);
    back(o, tb, s);
  }
  void step_vjp(const double* mn, double dt, const double* lin, double* lout, double* gKu, double* gH0,
                cudaStream_t s) override {
    const TV* mm = in_to(mn, ta, s);
    const TV* li = in_to(lin, tc, s);
    TV* lo = out_of(lout, tb);
    l.step_vjp(mm, dt, li, lo, gKu, gH0, s);
    back(lout, tb, s);
  }
  void step_jvp(const double* mn, const double* dm, const double* dKu, const double* dH0, double dt, double* mo,
                double* dmo, cudaStream_t s) override {
    const TV* mm = in_to(mn, ta, s);
    const TV* dd = in_to(dm, tc, s);
    TV* o1 = out_of(mo, tb);
    TV* o2 = out_of(dmo, td);
    l.step_jvp(mm, dd, dKu, dH0, dt, o1, o2, s);
    back(mo, tb, s);
    back(dmo, td, s);
  }
  void set_ku_map(const double* ku) override {
    l.graph_reset();
    l.rk_fsal = false;
    l.set_ku_map(ku, 0);
  }
  void zhang_li(const double* m, double* o, cudaStream_t s) override {
    TV* q = outbuf(o);
    l.zhang_li(in(m, s), q, s);
    out(o, s);
  }
  void set_sot(double Hdl, double Hfl, const double* p) override {
    l.graph_reset();
    l.rk_fsal = false;
    l.set_sot(Hdl, Hfl, p, 0);
  }
  void min_eval(double* m, double* d, int normalize, double* out5, cudaStream_t s) override {
    TV* mm = f64 ? reinterpret_cast<TV*>(m) : const_cast<TV*>(in_to(m, ta, s));
    TV* dd = out_of(d, td);
    l.min_eval(mm, nullptr, nullptr, dd, normalize != 0, out5, s);
    if (!f64 && normalize) convert<TV, double>(3 * l.N, mm, m, s);
    back(d, td, s);
    if (!f64) SPX_CUDA(cudaStreamSynchronize(s));
  }
  void min_trial(const double* m_old, const double* d_old, double alpha, double* mt, double* dt, double* out5,
                 cudaStream_t s) override {
    const TV* mo = in_to(m_old, ta, s);
    const TV* dold = in_to(d_old, tc, s);
    TV* m1 = out_of(mt, tb);
    TV* d1 = out_of(dt, td);
    l.min_trial(mo, dold, alpha, m1, d1, out5, s);
    back(mt, tb, s);
    back(dt, td, s);
    if (!f64) SPX_CUDA(cudaStreamSynchronize(s));
  }
  void set_graph(int on) override {
    l.graph_reset();
    l.graph_on = on != 0;
    l.graph_error.clear();
  }
  void graph_stats(int64_t* replays, int32_t* active) const override {
    if (replays) *replays = l.graph_replays;
    if (active) *active = (l.graph_on && l.graph_ok) ? 1 : 0;
  }
  std::string graph_error() const override { return l.graph_error; }
};

struct spx_llg_s {
  std::unique_ptr<LLGBase> impl;
  int64_t N = 0;
};

namespace spx {
template <class T>
__global__ void k_gemv_rows(int64_t Nb, const double* __restrict__ B, const double* __restrict__ x,
                            double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t i = w; i < Nb; i += nw) {
    double acc = 0.0;
    for (int64_t j = lane; j < Nb; j += 32) acc += B[i * Nb + j] * x[j];
    acc = warp_sum(acc);
    if (lane == 0) y[i] = acc;
  }
}
}  // namespace spx

template <class TV, class TM>
static std::unique_ptr<LLGBase> make_llg(spx_demag d, const double* X, int64_t N, const int32_t* tets, int64_t E,
                                         const LLGParams& q) {
  auto l = std::make_unique<LLGImpl<TV, TM>>();
  DemagCtx<TV, TM>* dm = nullptr;
  if (d) {
    auto* impl = dynamic_cast<DemagImpl<TV, TM>*>(d->impl.get());
    SPX_CHECK(impl != nullptr, "internal: demag precision mismatch");
    dm = &impl->d;
  }
  l->l.create(dm, X, N, tets, E, q, 0);
  return l;
}


namespace spx {
int barrier_timeout_probe(int nblocks, long long limit, int* timed_out_ctas);  // failure_probe.cu
double barrier_time_us(int nblocks, int threads, int nbar);                  // failure_probe.cu
void pcg_phase_times(double* ns32, int64_t* n32);                           // amg.cu
extern std::atomic<int> g_pcg_timing;                                       // amg.cu
}

extern "C" {

const char* spx_last_error(void) { return spx::g_last_error.c_str(); }
int spx_version(void) { return 10000; }

int spx_device_count(int32_t* n) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    c = 0;
  }
  if (n) *n = c;
  return SPX_OK;
}

int spx_boundary_sizes(const double* X, int64_t N, const int32_t* tets, int64_t E, int64_t* Nb, int64_t* Nt) {
  API_BEGIN
  check_mesh(X, N, tets, E);
  HostBoundary b;
  build_boundary(X, N, tets, E, b);
  if (Nb) *Nb = b.Nb;
  if (Nt) *Nt = b.Nt;
  API_END
}

int spx_boundary_data(const double* X, int64_t N, const int32_t* tets, int64_t E, int32_t* bverts, int32_t* tri_lid,
                      double* Xb, double* ntri, double* area, double* omega_sum) {
  API_BEGIN
  check_mesh(X, N, tets, E);
  HostBoundary b;
  build_boundary(X, N, tets, E, b);
  if (bverts) std::memcpy(bverts, b.bverts.data(), b.bverts.size() * sizeof(int32_t));
  if (tri_lid) std::memcpy(tri_lid, b.tri_lid.data(), b.tri_lid.size() * sizeof(int32_t));
  if (Xb) std::memcpy(Xb, b.Xb.data(), b.Xb.size() * sizeof(double));
  if (ntri) std::memcpy(ntri, b.ntri.data(), b.ntri.size() * sizeof(double));
  if (area) std::memcpy(area, b.area.data(), b.area.size() * sizeof(double));
  if (omega_sum) std::memcpy(omega_sum, b.omega_sum.data(), b.omega_sum.size() * sizeof(double));
  API_END
}

int spx_fem_sizes(const double* X, int64_t N, const int32_t* tets, int64_t E, int64_t* nnz) {
  API_BEGIN
  check_mesh(X, N, tets, E);
  HostFem f;
  assemble_fem(X, N, tets, E, f);
  REQUIRE(nnz);
  *nnz = f.rowptr[N];
  API_END
}

int spx_fem_assemble(const double* X, int64_t N, const int32_t* tets, int64_t E, int64_t* rowptr, int32_t* col,
                     double* A, double* Div, double* G, double* vol) {
  API_BEGIN
  check_mesh(X, N, tets, E);
  HostFem f;
  assemble_fem(X, N, tets, E, f);
  if (rowptr) std::memcpy(rowptr, f.rowptr.data(), f.rowptr.size() * sizeof(int64_t));
  if (col) std::memcpy(col, f.col.data(), f.col.size() * sizeof(int32_t));
  if (A) std::memcpy(A, f.A.data(), f.A.size() * sizeof(double));
  if (Div) std::memcpy(Div, f.Div.data(), f.Div.size() * sizeof(double));
  if (G) std::memcpy(G, f.G.data(), f.G.size() * sizeof(double));
  if (vol) std::memcpy(vol, f.vol.data(), f.vol.size() * sizeof(double));
  API_END
}

int spx_cluster_tree(const double* pts, int64_t n, int32_t leaf_size, int32_t* perm) {
  API_BEGIN
  REQUIRE(pts);
  REQUIRE(perm);
  ClusterTree t;
  build_cluster_tree(pts, n, leaf_size, t);
  std::memcpy(perm, t.perm.data(), t.perm.size() * sizeof(int32_t));
  API_END
}

int spx_boundary_create(const double* X, int64_t N, const int32_t* tets, int64_t E, spx_boundary* out) {
  API_BEGIN
  REQUIRE(out);
  *out = nullptr;
  check_mesh(X, N, tets, E);
  require_device();
  auto b = std::make_unique<spx_boundary_s>();
  b->bd.create(X, N, tets, E);
  *out = b.release();
  API_END
}

int spx_boundary_destroy(spx_boundary b) {
  API_BEGIN
  delete b;
  API_END
}

int spx_boundary_info(spx_boundary b, int64_t* Nb, int64_t* Nt, int32_t* maxinc) {
  API_BEGIN
  REQUIRE(b);
  if (Nb) *Nb = b->bd.host.Nb;
  if (Nt) *Nt = b->bd.host.Nt;
  if (maxinc) *maxinc = b->bd.maxinc;
  API_END
}

int spx_lindholm_pairs(spx_boundary b, const double* x0, const int32_t* tri, int64_t P, double* w, spx_stream_t s) {
  API_BEGIN
  REQUIRE(b);
  SPX_CHECK(P >= 0, "P must be non-negative");
  if (P == 0) return SPX_OK;
  REQUIRE(x0);
  REQUIRE(tri);
  REQUIRE(w);
  launch_lindholm_pairs(P, x0, tri, b->bd.T.p, b->bd.host.Nt, w, S(s));
  API_END
}

int spx_lindholm_fill_block(spx_boundary b, const int32_t* rows, int64_t m, const int32_t* cols, int64_t n,
                            double* out, spx_stream_t s) {
  API_BEGIN
  REQUIRE(b);
  SPX_CHECK(m >= 0 && n >= 0 && m < (1ll << 31) && n < (1ll << 31), "block size out of range");
  if (m == 0 || n == 0) return SPX_OK;
  REQUIRE(rows);
  REQUIRE(cols);
  REQUIRE(out);
  b->bd.fill_block(rows, m, cols, n, out, S(s));
  API_END
}

int spx_dense_b_assemble(spx_boundary b, double* B, spx_stream_t s) {
  API_BEGIN
  REQUIRE(b);
  REQUIRE(B);
  b->bd.dense_B(B, S(s));
  API_END
}


int spx_dense_b_apply(const double* B, int64_t Nb, const double* x, double* y, spx_stream_t s) {
  API_BEGIN
  REQUIRE(B);
  REQUIRE(x);
  REQUIRE(y);
  SPX_CHECK(Nb > 0, "Nb must be positive");
  k_gemv_rows<double><<<grid_for(Nb * 32, 256, 148 * 64), 256, 0, S(s)>>>(Nb, B, x, y);
  SPX_LAUNCH_CHECK();
  API_END
}

int spx_hmat_build(spx_boundary b, const spx_hmat_config* cfg, spx_hmat* out) {
  API_BEGIN
  REQUIRE(b);
  REQUIRE(out);
  *out = nullptr;
  auto h = std::make_unique<spx_hmat_s>();
  h->own.build(b->bd, to_hcfg(cfg), 0);
  h->own.pack(to_hprec(cfg ? cfg->precision : 0), 0);
  *out = h.release();
  API_END
}

int spx_hmat_export_sizes(spx_hmat hm, int64_t* nfar, int64_t* u_entries, int64_t* v_entries, int64_t* near_nnz) {
  API_BEGIN
  REQUIRE(hm);
  int64_t f = 0, u = 0, v = 0;
  hmat_far_sizes(hm->h(), f, u, v);
  hmat_near_csr(hm->h(), hm->near_indptr, hm->near_indices, hm->near_data);
  if (nfar) *nfar = f;
  if (u_entries) *u_entries = u;
  if (v_entries) *v_entries = v;
  if (near_nnz) *near_nnz = static_cast<int64_t>(hm->near_data.size());
  API_END
}

int spx_hmat_export(spx_hmat hm, int32_t* perm, double* diag_jump, int64_t* far_meta5, double* relres, double* U,
                    double* V, int32_t* near_indptr, int32_t* near_indices, double* near_data) {
  API_BEGIN
  REQUIRE(hm);
  const HMatrix& H = hm->h();
  SPX_CHECK(hm->near_indptr.size() == static_cast<size_t>(H.Nb + 1),
            "call spx_hmat_export_sizes before spx_hmat_export");
  if (perm) std::memcpy(perm, H.tree.perm.data(), H.Nb * sizeof(int32_t));
  if (diag_jump) {  // original boundary order
    std::vector<double> dp(H.Nb);
    SPX_CUDA(cudaMemcpy(dp.data(), H.diag_perm.p, H.Nb * sizeof(double), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < H.Nb; ++i) diag_jump[H.tree.perm[i]] = dp[i];
  }
  hmat_export_far(H, far_meta5, relres, U, V);
  if (near_indptr) std::memcpy(near_indptr, hm->near_indptr.data(), hm->near_indptr.size() * sizeof(int32_t));
  if (near_indices) std::memcpy(near_indices, hm->near_indices.data(), hm->near_indices.size() * sizeof(int32_t));
  if (near_data) std::memcpy(near_data, hm->near_data.data(), hm->near_data.size() * sizeof(double));
  hm->near_indptr.clear();
  hm->near_indices.clear();
  hm->near_data.clear();
  API_END
}

int spx_hmat_import(spx_boundary b, const spx_hmat_config* cfg, const int32_t* perm, const double* diag_jump,
                    int64_t nfar, const int64_t* far_meta5, const double* relres, const double* U, const double* V,
                    const int32_t* near_indptr, const int32_t* near_indices, const double* near_data,
                    spx_hmat* out) {
  API_BEGIN
  REQUIRE(b);
  REQUIRE(out);
  *out = nullptr;
  REQUIRE(near_indptr);
  SPX_CHECK(nfar >= 0 && (nfar == 0 || (far_meta5 && U && V)), "far blocks need meta, U and V");
  SPX_CHECK(near_indptr[0] == 0 && (near_indptr[b->bd.host.Nb] == 0 || (near_indices && near_data)),
            "near CSR needs indices and data");
  auto h = std::make_unique<spx_hmat_s>();
  hmat_import(h->own, b->bd, to_hcfg(cfg), to_hprec(cfg ? cfg->precision : 0), nfar, far_meta5, relres, U, V,
              near_indptr, near_indices, near_data, perm, diag_jump, 0);
  *out = h.release();
  API_END
}

int spx_hmat_stats(spx_hmat hm, int64_t* st, double* secs) {
  API_BEGIN
  REQUIRE(hm);
  const HStats& s = hm->h().stats;
  if (st) {
    const int64_t v[16] = {s.dense_blocks, s.low_rank_blocks, s.rejected_low_rank_blocks,
                           s.forced_subdivisions_memory, s.compression_tolerance_subdivisions,
                           s.max_observed_rank, s.sum_observed_rank, s.block_entry_evaluations, s.near_entries,
                           s.far_entries, s.n_far, s.n_near, s.aca_steps, s.waves, hm->h().Nb, 0};
    std::memcpy(st, v, sizeof(v));
  }
  if (secs) *secs = s.build_seconds;
  API_END
}

int spx_hmat_num_blocks(spx_hmat hm, int64_t* n) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(n);
  *n = static_cast<int64_t>(hm->h().blocks.size());
  API_END
}

int spx_hmat_blocks(spx_hmat hm, int64_t* out6, int64_t cap) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(out6);
  SPX_CHECK(cap >= static_cast<int64_t>(hm->h().blocks.size()), "capacity smaller than the number of blocks");
  int64_t k = 0;
  for (const HBlock& b : hm->h().blocks) {
    out6[6 * k] = b.rs; out6[6 * k + 1] = b.re; out6[6 * k + 2] = b.cs; out6[6 * k + 3] = b.ce;
    out6[6 * k + 4] = b.type; out6[6 * k + 5] = b.rank;
    ++k;
  }
  API_END
}

int spx_hmat_perm(spx_hmat hm, int32_t* perm) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(perm);
  std::memcpy(perm, hm->h().tree.perm.data(), hm->h().tree.perm.size() * sizeof(int32_t));
  API_END
}

int spx_hmat_apply(spx_hmat hm, const double* x, double* y, spx_stream_t s) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(x);
  REQUIRE(y);
  hm->h().apply_f64(x, y, S(s));
  API_END
}

int spx_hmat_apply_multi(spx_hmat hm, const double* X, double* Y, int32_t nrhs, spx_stream_t s) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(X);
  REQUIRE(Y);
  SPX_CHECK(nrhs >= 1, "nrhs must be at least 1");
  std::vector<int64_t> off(nrhs);
  for (int32_t r = 0; r < nrhs; ++r) off[r] = static_cast<int64_t>(r) * hm->h().Nb;
  hm->h().apply_multi<double>(X, nullptr, off.data(), Y, nullptr, nullptr, nullptr, nrhs, S(s));
  API_END
}

int spx_hmat_apply_transpose(spx_hmat hm, const double* x, double* y, spx_stream_t s) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(x);
  REQUIRE(y);
  hm->h().transposed(S(s)).apply_f64(x, y, S(s));
  API_END
}

int spx_hmat_apply_noalloc(spx_hmat hm, const double* x, double* y, spx_stream_t s) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(x);
  REQUIRE(y);
  hmat_apply_noalloc(hm->h(), x, y, S(s));
  API_END
}

int spx_hmat_repack(spx_hmat hm, int32_t precision) {
  API_BEGIN
  REQUIRE(hm);
  hm->h().pack(to_hprec(precision), 0);
  API_END
}

int spx_hmat_far_factors(spx_hmat hm, int64_t index, double* Ut, double* V) {
  API_BEGIN
  REQUIRE(hm);
  SPX_CHECK(index >= 0 && index < static_cast<int64_t>(hm->h().blocks.size()), "block index out of range");
  const HBlock& b = hm->h().blocks[index];
  SPX_CHECK(b.type == 1, "block is not a far (low-rank) block");
  const int64_t m = b.re - b.rs, n = b.ce - b.cs, k = b.rank;
  if (Ut) SPX_CUDA(cudaMemcpy(Ut, hm->h().far_pool64.p + b.off_u, k * m * sizeof(double), cudaMemcpyDeviceToHost));
  if (V) SPX_CUDA(cudaMemcpy(V, hm->h().far_pool64.p + b.off_v, k * n * sizeof(double), cudaMemcpyDeviceToHost));
  API_END
}

int spx_hmat_memory(spx_hmat hm, int64_t* far_bytes, int64_t* near_bytes, int64_t* total) {
  API_BEGIN
  REQUIRE(hm);
  if (far_bytes) *far_bytes = hm->h().bytes_far;
  if (near_bytes) *near_bytes = hm->h().bytes_near;
  if (total) *total = hm->h().device_bytes();
  API_END
}

int spx_debug_barrier_probe(int32_t nblocks, int64_t limit, int32_t* status, int32_t* timed_out_ctas) {
  API_BEGIN
  REQUIRE(status);
  REQUIRE(timed_out_ctas);
  int t = 0;
  *status = spx::barrier_timeout_probe(nblocks, static_cast<long long>(limit), &t);
  *timed_out_ctas = t;
  API_END
}

int spx_debug_barrier_time(int32_t nblocks, int32_t threads, int32_t nbarriers, double* us_per_barrier) {
  API_BEGIN
  REQUIRE(us_per_barrier);
  *us_per_barrier = spx::barrier_time_us(nblocks, threads, nbarriers);
  API_END
}

int spx_device_l2_persisting(int64_t* current_bytes, int64_t* max_bytes) {
  API_BEGIN
  REQUIRE(current_bytes); REQUIRE(max_bytes);
  int dev = 0, mx = 0;
  SPX_CUDA(cudaGetDevice(&dev));
  SPX_CUDA(cudaDeviceGetAttribute(&mx, cudaDevAttrMaxPersistingL2CacheSize, dev));
  size_t cur = 0;
  SPX_CUDA(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
  *current_bytes = static_cast<int64_t>(cur);
  *max_bytes = mx;
  API_END
}

int spx_debug_pcg_timing(int32_t enable) {
  API_BEGIN
  spx::g_pcg_timing.store(enable != 0 ? 1 : 0);
  API_END
}

int spx_debug_pcg_phase_times(double* ns32, int64_t* counts32) {
  API_BEGIN
  REQUIRE(ns32); REQUIRE(counts32);
  spx::pcg_phase_times(ns32, counts32);
  API_END
}

int spx_hmat_recompress(spx_hmat hm, int64_t* out3, double* max_rel_err) {
  API_BEGIN
  REQUIRE(hm);
  HMatrix& H = hm->h();
  SPX_CHECK(H.far_pool64.n > 0 || H.stats.n_far == 0, "this H-matrix has no FP64 factors (merged)");
  const Prec p = H.prec;
  const RecompressStats st = H.recompress(0);
  H.pack(p, 0);
  if (out3) {
    out3[0] = st.entries_before;
    out3[1] = st.entries_after;
    out3[2] = st.rewritten;
  }
  if (max_rel_err) *max_rel_err = st.truncation_error_max;
  API_END
}

// time of one 8-state apply (ms, median of 3 after a warm-up) with the current setting
static float time_multi8(HMatrix& H) {
  const int64_t Nb = H.Nb;
  DevBuf<double> X(8 * Nb), Y(8 * Nb);
  X.zero(0);
  std::vector<int64_t> off(8);
  for (int r = 0; r < 8; ++r) off[r] = r * Nb;
  cudaEvent_t a, b;
  SPX_CUDA(cudaEventCreate(&a));
  SPX_CUDA(cudaEventCreate(&b));
  H.apply_multi<double>(X.p, nullptr, off.data(), Y.p, nullptr, nullptr, nullptr, 8, 0);
  std::vector<float> t;
  for (int k = 0; k < 3; ++k) {
    SPX_CUDA(cudaEventRecord(a, 0));
    H.apply_multi<double>(X.p, nullptr, off.data(), Y.p, nullptr, nullptr, nullptr, 8, 0);
    SPX_CUDA(cudaEventRecord(b, 0));
    SPX_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    SPX_CUDA(cudaEventElapsedTime(&ms, a, b));
    t.push_back(ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  std::sort(t.begin(), t.end());
  return t[1];
}

int spx_hmat_tensor_cores(spx_hmat hm, int32_t enable, int64_t* plan_bytes) {
  API_BEGIN
  REQUIRE(hm);
  HMatrix& H = hm->h();
  SPX_CHECK(enable >= 0 && enable <= 2, "enable must be 0, 1 or 2 (autotune)");
  if (enable) {
    SPX_CHECK(H.packed && (H.prec == Prec::F32 || H.prec == Prec::F64 || H.prec == Prec::SPLIT),
              "the tensor-core multi-state apply needs an F64, F32 or F32_F16 packing");
    if (enable == 1) {
      if (!H.tc) tc_build(H, 0);
    } else {  // autotune: CUDA-core kernels vs tensor-core tiles of 512 / 2048 K elements
      H.tc.reset();
      float best = H.prec == Prec::SPLIT ? 1e30f : time_multi8(H);
      int best_k = 0;
      for (int ks : {16, 64}) {  // stages of 32 K elements
        tc_build(H, 0, ks);
        const float t = time_multi8(H);
        SPX_CHECK(tc_error(H, 0) == 0, "tensor-core apply timed out during autotuning");
        if (t < best) {
          best = t;
          best_k = ks;
        }
        H.tc.reset();
      }
      if (best_k > 0) tc_build(H, 0, best_k);
    }
  } else {
    H.tc.reset();
  }
  if (plan_bytes) *plan_bytes = tc_bytes(H);
  API_END
}

int spx_hmat_tc_status(spx_hmat hm, int32_t* status) {
  API_BEGIN
  REQUIRE(hm); REQUIRE(status);
  HMatrix& H = hm->h();
  *status = tc_error(H, 0);
  API_END
}

int spx_debug_fail_alloc(int64_t min_bytes, int32_t count) {
  API_BEGIN
  SPX_CHECK(min_bytes >= 0 && count >= 0, "min_bytes and count must be non-negative");
  spx::g_fail_alloc_min_bytes.store(min_bytes);
  spx::g_fail_alloc_count.store(count);
  API_END
}

int spx_debug_noalloc_cap(int64_t bytes) {
  API_BEGIN
  SPX_CHECK(bytes >= 0, "bytes must be non-negative");
  spx::g_noalloc_cap.store(bytes);
  API_END
}

int spx_hmat_destroy(spx_hmat hm) {
  API_BEGIN
  SPX_CHECK(!hm || !hm->ext, "this H-matrix handle belongs to a demag object (destroy the demag object instead)");
  delete hm;
  API_END
}

struct EnsembleSpec {
  int64_t nsamples;
  const int64_t* offsets;
  int64_t dense_max_nb;
};

static int demag_create(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms,
                        const spx_demag_options* opt, HMatrix* preset, spx_demag* out,
                        const EnsembleSpec* ens = nullptr) {
  API_BEGIN
  REQUIRE(out);
  *out = nullptr;
  check_mesh(X, N, tets, E);
  require_device();
  SPX_CHECK(Ms > 0.0, "Ms must be positive");
  DemagOptions o;
  if (opt) {
    SPX_CHECK(opt->backend == 0 || opt->backend == 1, "backend must be 0 (dense) or 1 (hmatrix)");
    SPX_CHECK(opt->warm_start >= 0 && opt->warm_start <= 3, "warm_start must be 0, 1, 2 or 3");
    o.backend = opt->backend;
    o.prec = to_prec(opt->precision);
    o.hprec = to_hprec(opt->hmat.precision);
    if (opt->rtol_u1 > 0) o.rtol_u1 = opt->rtol_u1;
    if (opt->rtol_u2 > 0) o.rtol_u2 = opt->rtol_u2;
    if (opt->atol >= 0) o.atol = opt->atol;
    if (opt->maxit_u1 > 0) o.maxit_u1 = opt->maxit_u1;
    if (opt->maxit_u2 > 0) o.maxit_u2 = opt->maxit_u2;
    o.warm_start = opt->warm_start;
    SPX_CHECK(opt->u1_preconditioner == 0 || opt->u1_preconditioner == 1,
              "u1_preconditioner must be 0 (AMG) or 1 (Jacobi)");
    o.u1_pc = opt->u1_preconditioner;
    o.hcfg = to_hcfg(&opt->hmat);
  }
  if (preset) {
    SPX_CHECK(o.backend == 1, "an H-matrix can only be given to the hmatrix backend");
    o.preset = preset;
  }
  if (ens) {
    SPX_CHECK(ens->nsamples >= 1 && ens->offsets, "an ensemble needs nsamples >= 1 and node offsets");
    SPX_CHECK(ens->dense_max_nb >= 0, "dense_max_nb must be non-negative");
    o.backend = 2;
    o.sample_offsets.assign(ens->offsets, ens->offsets + ens->nsamples + 1);
    o.dense_max_nb = ens->dense_max_nb;
  }
  auto d = std::make_unique<spx_demag_s>();
  switch (o.prec) {
    case Prec::F64: {
      auto p = std::make_unique<DemagImpl<double, double>>();
      p->d.create(X, N, tets, E, Ms, o, 0);
      d->impl = std::move(p);
      break;
    }
    case Prec::F32: {
      auto p = std::make_unique<DemagImpl<float, float>>();
      p->d.create(X, N, tets, E, Ms, o, 0);
      d->impl = std::move(p);
      break;
    }
    case Prec::MIXED: {
      auto p = std::make_unique<DemagImpl<double, float>>();
      p->d.create(X, N, tets, E, Ms, o, 0);
      d->impl = std::move(p);
      break;
    }
  }
  *out = d.release();
  API_END
}

int spx_demag_create(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms,
                     const spx_demag_options* opt, spx_demag* out) {
  return demag_create(X, N, tets, E, Ms, opt, nullptr, out);
}

int spx_demag_create_ensemble(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms,
                              const spx_demag_options* opt, int64_t nsamples, const int64_t* node_offsets,
                              int64_t dense_max_nb, spx_demag* out) {
  const EnsembleSpec e{nsamples, node_offsets, dense_max_nb};
  return demag_create(X, N, tets, E, Ms, opt, nullptr, out, &e);
}

int spx_demag_ensemble_info(spx_demag d, int64_t* out6) {
  API_BEGIN
  REQUIRE(d); REQUIRE(out6);
  d->impl->ensemble_info(out6);
  API_END
}

int spx_demag_create_with_hmat(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms,
                               const spx_demag_options* opt, spx_hmat hm, spx_demag* out) {
  if (!hm) {
    spx::set_last_error("null H-matrix handle");
    return SPX_ERR_INVALID;
  }
  if (hm->ext) {
    spx::set_last_error("the H-matrix handle belongs to a demag object");
    return SPX_ERR_INVALID;
  }
  return demag_create(X, N, tets, E, Ms, opt, &hm->own, out);
}

int spx_demag_apply(spx_demag d, const double* m, double* H, spx_stream_t s) {
  API_BEGIN
  REQUIRE(d); REQUIRE(m); REQUIRE(H);
  d->impl->apply(m, H, S(s));
  API_END
}

int spx_demag_potentials(spx_demag d, double* u1, double* u2, spx_stream_t s) {
  API_BEGIN
  REQUIRE(d);
  const int64_t N = d->impl->N();
  DevBuf<double> a(N);
  d->impl->potentials(a.p, u2, S(s));  // u2 temporarily holds phi
  if (u1) SPX_CUDA(cudaMemcpyAsync(u1, a.p, N * sizeof(double), cudaMemcpyDeviceToDevice, S(s)));
  if (u2) {
    std::vector<double> ha(N), hb(N);
    SPX_CUDA(cudaMemcpyAsync(ha.data(), a.p, N * sizeof(double), cudaMemcpyDeviceToHost, S(s)));
    SPX_CUDA(cudaMemcpyAsync(hb.data(), u2, N * sizeof(double), cudaMemcpyDeviceToHost, S(s)));
    SPX_CUDA(cudaStreamSynchronize(S(s)));
    for (int64_t i = 0; i < N; ++i) hb[i] -= ha[i];
    SPX_CUDA(cudaMemcpyAsync(u2, hb.data(), N * sizeof(double), cudaMemcpyHostToDevice, S(s)));
  }
  SPX_CUDA(cudaStreamSynchronize(S(s)));
  API_END
}

int spx_demag_energy(spx_demag d, const double* m, const double* H, double* E, spx_stream_t s) {
  API_BEGIN
  REQUIRE(d); REQUIRE(m); REQUIRE(H); REQUIRE(E);
  *E = d->impl->energy(m, H, S(s));
  API_END
}

int spx_demag_stats(spx_demag d, int64_t* i1, int64_t* i2, double* r1, double* r2) {
  API_BEGIN
  REQUIRE(d);
  const CgStats a = d->impl->last1(), b = d->impl->last2();
  if (i1) *i1 = a.iterations;
  if (i2) *i2 = b.iterations;
  if (r1) *r1 = a.rel_residual;
  if (r2) *r2 = b.rel_residual;
  API_END
}

int spx_demag_info(spx_demag d, int64_t* N, int64_t* Nb, int64_t* NI, int64_t* bytes) {
  API_BEGIN
  REQUIRE(d);
  d->impl->info(N, Nb, NI, bytes);
  API_END
}

int spx_demag_hmat(spx_demag d, spx_hmat* h) {
  API_BEGIN
  REQUIRE(d);
  REQUIRE(h);
  HMatrix* H = d->impl->hmat();
  SPX_CHECK(H != nullptr, "demag uses the dense boundary operator");
  *h = d->impl->view_of(H);
  API_END
}

int spx_demag_ensemble_hmat(spx_demag d, int32_t group, spx_hmat* h) {
  API_BEGIN
  REQUIRE(d);
  REQUIRE(h);
  HMatrix* H = d->impl->shared_hmat(group);
  SPX_CHECK(H != nullptr, "no H-matrix shared by several samples with this index");
  *h = d->impl->view_of(H);
  API_END
}

int spx_demag_profile_begin(spx_demag d) {
  API_BEGIN
  REQUIRE(d);
  d->impl->prof().begin();
  API_END
}

int spx_demag_profile_end(spx_demag d, double* ms8, int64_t* l8, int64_t* g8) {
  API_BEGIN
  REQUIRE(d); REQUIRE(ms8); REQUIRE(l8); REQUIRE(g8);
  d->impl->prof().end(ms8, l8, g8);
  API_END
}

int spx_demag_counters(spx_demag d, int64_t* c1, int64_t* c2) {
  API_BEGIN
  REQUIRE(d);
  unsigned long long a[4] = {0, 0, 0, 0}, b[4] = {0, 0, 0, 0};
  d->impl->counters(a, b);
  for (int k = 0; k < 4; ++k) {
    if (c1) c1[k] = static_cast<int64_t>(a[k]);
    if (c2) c2[k] = static_cast<int64_t>(b[k]);
  }
  API_END
}

int spx_demag_residuals(spx_demag d, double* r1, double* r2) {
  API_BEGIN
  REQUIRE(d);
  double a[2] = {0, 0}, b[2] = {0, 0};
  d->impl->residuals(a, b);
  for (int k = 0; k < 2; ++k) {
    if (r1) r1[k] = a[k];
    if (r2) r2[k] = b[k];
  }
  API_END
}

int spx_demag_amg_levels(spx_demag d, int64_t* levels4, int32_t max_levels, int32_t* nlev) {
  API_BEGIN
  REQUIRE(d);
  REQUIRE(nlev);
  SPX_CHECK(max_levels >= 0 && (levels4 || max_levels == 0), "levels4 must hold 4 * max_levels entries");
  *nlev = d->impl->amg_levels(levels4, max_levels);
  API_END
}

int spx_demag_set_tolerances(spx_demag d, double rtol_u1, double rtol_u2, double atol, int32_t maxit_u1,
                             int32_t maxit_u2) {
  API_BEGIN
  REQUIRE(d);
  SPX_CHECK(rtol_u1 > 0.0 && rtol_u2 > 0.0 && atol >= 0.0, "tolerances must be positive");
  SPX_CHECK(maxit_u1 > 0 && maxit_u2 > 0, "iteration limits must be positive");
  d->impl->set_tolerances(rtol_u1, rtol_u2, atol, maxit_u1, maxit_u2);
  API_END
}

int spx_demag_apply_transpose(spx_demag d, const double* w, double* out, spx_stream_t s) {
  API_BEGIN
  REQUIRE(d); REQUIRE(w); REQUIRE(out);
  d->impl->apply_transpose(w, out, S(s));
  API_END
}

int spx_demag_destroy(spx_demag d) {
  API_BEGIN
  delete d;
  API_END
}

static LLGParams to_params(const spx_llg_params* p) {
  LLGParams q;
  REQUIRE(p);
  SPX_CHECK(p->Ms > 0.0, "Ms must be positive");
  q.Ms = p->Ms; q.gamma = p->gamma; q.alpha = p->alpha; q.do_precess = p->do_precess;
  q.Aex = p->Aex; q.Ku = p->Ku; q.Ku_nodes = p->Ku_nodes; q.n_ani = p->n_ani;
  q.D_int = p->D_int; q.n_int = p->n_int; q.H0_nodes = p->H0_nodes; q.D_bulk = p->D_bulk;
  for (int c = 0; c < 3; ++c) q.H0_uniform[c] = p->H0_uniform[c];
  q.use_demag = p->use_demag;
  q.stt_J = p->stt_J; q.stt_P = p->stt_P; q.stt_beta = p->stt_beta; q.stt_dir = p->stt_dir;
  q.sot_Hdl = p->sot_Hdl; q.sot_Hfl = p->sot_Hfl; q.sot_p = p->sot_p;
  SPX_CHECK(!((q.Ku != 0.0 || q.Ku_nodes) && !q.n_ani), "anisotropy needs easy axes (n_ani)");
  return q;
}

int spx_llg_create(spx_demag d, const double* X, int64_t N, const int32_t* tets, int64_t E,
                   const spx_llg_params* p, spx_llg* out) {
  API_BEGIN
  REQUIRE(out);
  *out = nullptr;
  check_mesh(X, N, tets, E);
  require_device();
  LLGParams q = to_params(p);
  auto l = std::make_unique<spx_llg_s>();
  l->N = N;
  int prec = p->precision;
  if (d) {
    if (dynamic_cast<DemagImpl<double, double>*>(d->impl.get())) prec = 0;
    else if (dynamic_cast<DemagImpl<float, float>*>(d->impl.get())) prec = 1;
    else prec = 2;
    SPX_CHECK(d->impl->N() == N, "demag and LLG meshes differ");
  }
  switch (to_prec(prec)) {
    case Prec::F64: l->impl = make_llg<double, double>(d, X, N, tets, E, q); break;
    case Prec::F32: l->impl = make_llg<float, float>(d, X, N, tets, E, q); break;
    case Prec::MIXED: l->impl = make_llg<double, float>(d, X, N, tets, E, q); break;
  }
  *out = l.release();
  API_END
}

int spx_llg_heff(spx_llg l, const double* m, double* H, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(H);
  l->impl->heff(m, H, true, S(s));
  API_END
}

int spx_llg_hjac(spx_llg l, const double* m, double* H, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(H);
  l->impl->heff(m, H, false, S(s));
  API_END
}

int spx_llg_rhs(spx_llg l, const double* m, double* r, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(r);
  l->impl->rhs(m, r, S(s));
  API_END
}

int spx_llg_update_jac_state(spx_llg l, const double* m, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m);
  l->impl->update_jac_state(m, S(s));
  API_END
}

int spx_llg_jv(spx_llg l, const double* v, double* o, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(v); REQUIRE(o);
  l->impl->jv(v, o, S(s));
  API_END
}

int spx_llg_pc_build(spx_llg l, double shift, int32_t include_stab, int32_t use_abs_kappa, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l);
  l->impl->pc_build(shift, include_stab, use_abs_kappa, S(s));
  API_END
}

int spx_llg_pc_apply(spx_llg l, const double* x, double* y, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(x); REQUIRE(y);
  l->impl->pc_apply(x, y, S(s));
  API_END
}

int spx_llg_set_state(spx_llg l, const double* m, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m);
  l->impl->set_state(m, S(s));
  API_END
}

int spx_llg_get_state(spx_llg l, double* m, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m);
  l->impl->get_state(m, S(s));
  API_END
}

int spx_llg_step(spx_llg l, double dt, int64_t nsteps, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l);
  SPX_CHECK(nsteps >= 0, "nsteps must be non-negative");
  SPX_CHECK(dt > 0.0, "dt must be positive");
  l->impl->step(dt, nsteps, S(s));
  API_END
}

int spx_llg_run_host(spx_llg l, const double* m_in, double* m_out, double dt, int64_t nsteps) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m_in); REQUIRE(m_out);
  SPX_CHECK(dt > 0.0 && nsteps >= 0, "dt must be positive and nsteps non-negative");
  l->impl->run_host(m_in, m_out, dt, nsteps);
  API_END
}

int spx_llg_set_time_field(spx_llg l, const double* h_uniform3, const double* h_nodes, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l);
  l->impl->set_time_field(h_uniform3, h_nodes, S(s));
  API_END
}

int spx_llg_step_time_field(spx_llg l, double dt, const double* h_uniform4x3, const double* h_nodes4,
                            spx_stream_t s) {
  API_BEGIN
  REQUIRE(l);
  SPX_CHECK(dt > 0.0, "dt must be positive");
  l->impl->step_time_field(dt, h_uniform4x3, h_nodes4, S(s));
  API_END
}

int spx_llg_rk_attempt(spx_llg l, int32_t scheme, double dt, double rtol, double atol, const double* h_uniform7x3,
                       const double* h_nodes7, int32_t reuse_fsal, double* err_norm, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(err_norm);
  SPX_CHECK(scheme == 0, "scheme must be 0 (Dormand-Prince 5(4))");
  SPX_CHECK(dt > 0.0, "dt must be positive");
  SPX_CHECK(rtol >= 0.0 && atol >= 0.0 && rtol + atol > 0.0, "rtol and atol must be non-negative, not both zero");
  *err_norm = l->impl->rk_attempt(dt, rtol, atol, h_uniform7x3, h_nodes7, reuse_fsal != 0, S(s));
  API_END
}

int spx_llg_rk_accept(spx_llg l, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l);
  l->impl->rk_accept(S(s));
  API_END
}

static ImplicitOpts implicit_opts(const spx_bdf_opts* p) {
  ImplicitOpts o;
  if (!p) return o;
  o.rtol = p->rtol; o.atol = p->atol;
  o.snes_rtol = p->snes_rtol; o.snes_atol = p->snes_atol; o.snes_stol = p->snes_stol; o.snes_divtol = p->snes_divtol;
  o.ksp_rtol = p->ksp_rtol; o.ksp_atol = p->ksp_atol; o.ksp_dtol = p->ksp_dtol;
  o.ls_alpha = p->ls_alpha; o.ls_minlambda = p->ls_minlambda; o.ls_maxstep = p->ls_maxstep;
  o.snes_max_it = p->snes_max_it; o.ksp_max_it = p->ksp_max_it; o.ksp_restart = p->ksp_restart;
  o.ls_max_it = p->ls_max_it; o.use_pc = p->use_pc;
  SPX_CHECK(o.rtol >= 0.0 && o.atol >= 0.0 && o.rtol + o.atol > 0.0,
            "rtol and atol must be non-negative, not both zero");
  SPX_CHECK(o.snes_max_it >= 1 && o.ksp_max_it >= 1 && o.ls_max_it >= 0, "iteration limits must be positive");
  SPX_CHECK(o.ksp_restart >= 1 && o.ksp_restart <= 100, "ksp_restart must be in [1, 100]");
  SPX_CHECK(o.ls_maxstep > 0.0 && o.ksp_dtol > 0.0, "ls_maxstep and ksp_dtol must be positive");
  return o;
}

int spx_bdf_default_opts(spx_bdf_opts* o) {
  API_BEGIN
  REQUIRE(o);
  const ImplicitOpts d;
  o->rtol = d.rtol; o->atol = d.atol;
  o->snes_rtol = d.snes_rtol; o->snes_atol = d.snes_atol; o->snes_stol = d.snes_stol; o->snes_divtol = d.snes_divtol;
  o->ksp_rtol = d.ksp_rtol; o->ksp_atol = d.ksp_atol; o->ksp_dtol = d.ksp_dtol;
  o->ls_alpha = d.ls_alpha; o->ls_minlambda = d.ls_minlambda; o->ls_maxstep = d.ls_maxstep;
  o->snes_max_it = d.snes_max_it; o->ksp_max_it = d.ksp_max_it; o->ksp_restart = d.ksp_restart;
  o->ls_max_it = d.ls_max_it; o->use_pc = d.use_pc; o->reserved = 0;
  API_END
}

int spx_llg_bdf_attempt(spx_llg l, double t, double dt, const spx_bdf_opts* o, const double* h_uniform2x3,
                        const double* h_nodes2, spx_bdf_result* r, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(r);
  SPX_CHECK(dt > 0.0 && std::isfinite(t) && std::isfinite(dt), "dt must be positive and t finite");
  const ImplicitResult x = l->impl->bdf_attempt(t, dt, implicit_opts(o), h_uniform2x3, h_nodes2, S(s));
  r->wlte = x.wlte;
  r->snes_reason = x.snes_reason;
  r->order = x.order;
  r->restarted = x.restarted;
  r->newton_its = x.newton_its;
  r->linear_its = x.linear_its;
  r->fevals = x.fevals;
  API_END
}

int spx_llg_bdf_accept(spx_llg l, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l);
  l->impl->bdf_accept(S(s));
  API_END
}

int spx_llg_bdf_reset(spx_llg l) {
  API_BEGIN
  REQUIRE(l);
  l->impl->bdf_reset();
  API_END
}

int spx_vec_node_diff_max(const double* a, const double* b, int64_t N, double* out, spx_stream_t s) {
  API_BEGIN
  REQUIRE(a); REQUIRE(b); REQUIRE(out);
  SPX_CHECK(N >= 0, "N must be non-negative");
  *out = N ? spx::node_diff_max(N, a, b, S(s)) : 0.0;
  API_END
}

int spx_llg_set_uniform_field(spx_llg l, double hx, double hy, double hz) {
  API_BEGIN
  REQUIRE(l);
  l->impl->set_uniform_field(hx, hy, hz);
  API_END
}

int spx_llg_stats(spx_llg l, int64_t* steps, int64_t* rhs, int64_t* launches) {
  API_BEGIN
  REQUIRE(l);
  l->impl->stats(steps, rhs, launches);
  API_END
}

int spx_llg_set_anisotropy_map(spx_llg l, const double* Ku_nodes) {
  API_BEGIN
  REQUIRE(l); REQUIRE(Ku_nodes);
  l->impl->set_ku_map(Ku_nodes);
  API_END
}

int spx_llg_rhs_vjp(spx_llg l, const double* m, const double* w, double* mbar, double* gKu, double* gH0,
                    spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(w); REQUIRE(mbar);
  l->impl->rhs_vjp(m, w, mbar, gKu, gH0, S(s));
  API_END
}

int spx_llg_step_vjp(spx_llg l, const double* m_n, double dt, const double* lam_in, double* lam_out, double* gKu,
                     double* gH0, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m_n); REQUIRE(lam_in); REQUIRE(lam_out);
  SPX_CHECK(dt > 0.0, "dt must be positive");
  l->impl->step_vjp(m_n, dt, lam_in, lam_out, gKu, gH0, S(s));
  API_END
}

int spx_llg_step_jvp(spx_llg l, const double* m_n, const double* dm, const double* dKu, const double* dH0, double dt,
                     double* m_out, double* dm_out, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m_n); REQUIRE(dm); REQUIRE(m_out); REQUIRE(dm_out);
  SPX_CHECK(dt > 0.0, "dt must be positive");
  l->impl->step_jvp(m_n, dm, dKu, dH0, dt, m_out, dm_out, S(s));
  API_END
}

int spx_llg_zhang_li(spx_llg l, const double* m, double* out, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(out);
  l->impl->zhang_li(m, out, S(s));
  API_END
}

int spx_llg_set_sot(spx_llg l, double H_dl, double H_fl, const double* polarization) {
  API_BEGIN
  REQUIRE(l);
  l->impl->set_sot(H_dl, H_fl, polarization);
  API_END
}

int spx_llg_min_eval(spx_llg l, double* m, double* d, int32_t normalize, double* out5, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(d); REQUIRE(out5);
  l->impl->min_eval(m, d, normalize, out5, S(s));
  API_END
}

int spx_llg_min_trial(spx_llg l, const double* m_old, const double* d_old, double alpha, double* m_trial,
                      double* d_trial, double* out5, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m_old); REQUIRE(d_old); REQUIRE(m_trial); REQUIRE(d_trial); REQUIRE(out5);
  l->impl->min_trial(m_old, d_old, alpha, m_trial, d_trial, out5, S(s));
  API_END
}

int spx_llg_set_graph(spx_llg l, int32_t enable) {
  API_BEGIN
  REQUIRE(l);
  l->impl->set_graph(enable);
  API_END
}

int spx_llg_graph_stats(spx_llg l, int64_t* replays, int32_t* active) {
  API_BEGIN
  REQUIRE(l);
  l->impl->graph_stats(replays, active);
  const std::string e = l->impl->graph_error();
  if (!e.empty()) spx::set_last_error(e);
  API_END
}

int spx_llg_destroy(spx_llg l) {
  API_BEGIN
  delete l;
  API_END
}

}  // extern "C"
