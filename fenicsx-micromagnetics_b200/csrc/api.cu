// extern "C" entry points of libspx (declared in include/spx.h).
#include <cstring>
#include <memory>

#include "../../include/spx.h"
#include "llg.cuh"

namespace spx {
namespace {
thread_local std::string g_last_error;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }
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
  HMatrix h;
};
struct spx_demag_s {
  Prec prec = Prec::F64;
  std::unique_ptr<DemagCtx<double>> d64;
  std::unique_ptr<DemagCtx<float>> d32;
  DevBuf<float> tm, th;  // FP32 staging of FP64 API vectors
  int64_t N() const { return d64 ? d64->N : d32->N; }
};
struct spx_llg_s {
  bool f32 = false;
  std::unique_ptr<LLGCtx<double>> l64;
  std::unique_ptr<LLGCtx<float>> l32;
  DevBuf<float> ta, tb;
  DevBuf<double> hstage;
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

// run op on FP64 API vectors: in -> (convert) -> op -> (convert) -> out
template <class F64, class F32>
static void llg_call(spx_llg l, const double* in, double* outp, spx_stream_t s, F64 f64, F32 f32) {
  if (!l->f32) {
    f64(*l->l64, in, outp);
  } else {
    const int64_t n3 = 3 * l->N;
    if (in) convert<double, float>(n3, in, l->ta.p, S(s));
    f32(*l->l32, in ? l->ta.p : nullptr, outp ? l->tb.p : nullptr);
    if (outp) convert<float, double>(n3, l->tb.p, outp, S(s));
  }
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
  h->h.build(b->bd, to_hcfg(cfg), 0);
  h->h.pack(to_prec(cfg ? cfg->precision : 0), 0);
  *out = h.release();
  API_END
}

int spx_hmat_stats(spx_hmat hm, int64_t* st, double* secs) {
  API_BEGIN
  REQUIRE(hm);
  const HStats& s = hm->h.stats;
  if (st) {
    const int64_t v[16] = {s.dense_blocks, s.low_rank_blocks, s.rejected_low_rank_blocks,
                           s.forced_subdivisions_memory, s.compression_tolerance_subdivisions,
                           s.max_observed_rank, s.sum_observed_rank, s.block_entry_evaluations, s.near_entries,
                           s.far_entries, s.n_far, s.n_near, s.aca_steps, s.waves, 0, 0};
    std::memcpy(st, v, sizeof(v));
  }
  if (secs) *secs = s.build_seconds;
  API_END
}

int spx_hmat_num_blocks(spx_hmat hm, int64_t* n) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(n);
  *n = static_cast<int64_t>(hm->h.blocks.size());
  API_END
}

int spx_hmat_blocks(spx_hmat hm, int64_t* out6, int64_t cap) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(out6);
  SPX_CHECK(cap >= static_cast<int64_t>(hm->h.blocks.size()), "capacity smaller than the number of blocks");
  int64_t k = 0;
  for (const HBlock& b : hm->h.blocks) {
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
  std::memcpy(perm, hm->h.tree.perm.data(), hm->h.tree.perm.size() * sizeof(int32_t));
  API_END
}

int spx_hmat_apply(spx_hmat hm, const double* x, double* y, spx_stream_t s) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(x);
  REQUIRE(y);
  hm->h.apply_f64(x, y, S(s));
  API_END
}

int spx_hmat_apply_noalloc(spx_hmat hm, const double* x, double* y, spx_stream_t s) {
  API_BEGIN
  REQUIRE(hm);
  REQUIRE(x);
  REQUIRE(y);
  hmat_apply_noalloc(hm->h, x, y, S(s));
  API_END
}

int spx_hmat_repack(spx_hmat hm, int32_t precision) {
  API_BEGIN
  REQUIRE(hm);
  hm->h.pack(to_prec(precision), 0);
  API_END
}

int spx_hmat_far_factors(spx_hmat hm, int64_t index, double* Ut, double* V) {
  API_BEGIN
  REQUIRE(hm);
  SPX_CHECK(index >= 0 && index < static_cast<int64_t>(hm->h.blocks.size()), "block index out of range");
  const HBlock& b = hm->h.blocks[index];
  SPX_CHECK(b.type == 1, "block is not a far (low-rank) block");
  const int64_t m = b.re - b.rs, n = b.ce - b.cs, k = b.rank;
  if (Ut) SPX_CUDA(cudaMemcpy(Ut, hm->h.far_pool64.p + b.off_u, k * m * sizeof(double), cudaMemcpyDeviceToHost));
  if (V) SPX_CUDA(cudaMemcpy(V, hm->h.far_pool64.p + b.off_v, k * n * sizeof(double), cudaMemcpyDeviceToHost));
  API_END
}

int spx_hmat_memory(spx_hmat hm, int64_t* far_bytes, int64_t* near_bytes, int64_t* total) {
  API_BEGIN
  REQUIRE(hm);
  if (far_bytes) *far_bytes = hm->h.bytes_far;
  if (near_bytes) *near_bytes = hm->h.bytes_near;
  if (total) *total = hm->h.device_bytes();
  API_END
}

int spx_hmat_destroy(spx_hmat hm) {
  API_BEGIN
  delete hm;
  API_END
}

int spx_demag_create(const double* X, int64_t N, const int32_t* tets, int64_t E, double Ms,
                     const spx_demag_options* opt, spx_demag* out) {
  API_BEGIN
  REQUIRE(out);
  *out = nullptr;
  check_mesh(X, N, tets, E);
  require_device();
  SPX_CHECK(Ms > 0.0, "Ms must be positive");
  DemagOptions o;
  if (opt) {
    SPX_CHECK(opt->backend == 0 || opt->backend == 1, "backend must be 0 (dense) or 1 (hmatrix)");
    o.backend = opt->backend;
    o.prec = to_prec(opt->precision);
    if (opt->rtol_u1 > 0) o.rtol_u1 = opt->rtol_u1;
    if (opt->rtol_u2 > 0) o.rtol_u2 = opt->rtol_u2;
    if (opt->atol >= 0) o.atol = opt->atol;
    if (opt->maxit_u1 > 0) o.maxit_u1 = opt->maxit_u1;
    if (opt->maxit_u2 > 0) o.maxit_u2 = opt->maxit_u2;
    o.warm_start = opt->warm_start;
    o.hcfg = to_hcfg(&opt->hmat);
  }
  auto d = std::make_unique<spx_demag_s>();
  d->prec = o.prec;
  if (o.prec == Prec::F64) {
    d->d64 = std::make_unique<DemagCtx<double>>();
    d->d64->create(X, N, tets, E, Ms, o, 0);
  } else {
    d->d32 = std::make_unique<DemagCtx<float>>();
    d->d32->create(X, N, tets, E, Ms, o, 0);
    d->tm.alloc(3 * N);
    d->th.alloc(3 * N);
  }
  *out = d.release();
  API_END
}

int spx_demag_apply(spx_demag d, const double* m, double* H, spx_stream_t s) {
  API_BEGIN
  REQUIRE(d);
  REQUIRE(m);
  REQUIRE(H);
  if (d->d64) {
    d->d64->potential(m, S(s), true);
    d->d64->field(H, S(s));
  } else {
    const int64_t n3 = 3 * d->d32->N;
    convert<double, float>(n3, m, d->tm.p, S(s));
    d->d32->potential(d->tm.p, S(s), true);
    d->d32->field(d->th.p, S(s));
    convert<float, double>(n3, d->th.p, H, S(s));
  }
  API_END
}

int spx_demag_potentials(spx_demag d, double* u1, double* u2, spx_stream_t s) {
  API_BEGIN
  REQUIRE(d);
  const int64_t N = d->N();
  DevBuf<double> t(N);
  if (d->d64) {
    if (u1) SPX_CUDA(cudaMemcpyAsync(u1, d->d64->u1.p, N * sizeof(double), cudaMemcpyDeviceToDevice, S(s)));
    if (u2) {
      SPX_CUDA(cudaMemcpyAsync(u2, d->d64->phi.p, N * sizeof(double), cudaMemcpyDeviceToDevice, S(s)));
    }
  } else {
    if (u1) convert<float, double>(N, d->d32->u1.p, u1, S(s));
    if (u2) convert<float, double>(N, d->d32->phi.p, u2, S(s));
  }
  // u2 = phi - u1
  if (u2) {
    std::vector<double> a(N), b(N);
    if (d->d64) SPX_CUDA(cudaMemcpyAsync(a.data(), d->d64->u1.p, N * sizeof(double), cudaMemcpyDeviceToHost, S(s)));
    else {
      convert<float, double>(N, d->d32->u1.p, t.p, S(s));
      SPX_CUDA(cudaMemcpyAsync(a.data(), t.p, N * sizeof(double), cudaMemcpyDeviceToHost, S(s)));
    }
    SPX_CUDA(cudaMemcpyAsync(b.data(), u2, N * sizeof(double), cudaMemcpyDeviceToHost, S(s)));
    SPX_CUDA(cudaStreamSynchronize(S(s)));
    for (int64_t i = 0; i < N; ++i) b[i] -= a[i];
    SPX_CUDA(cudaMemcpyAsync(u2, b.data(), N * sizeof(double), cudaMemcpyHostToDevice, S(s)));
    SPX_CUDA(cudaStreamSynchronize(S(s)));
  }
  API_END
}

int spx_demag_energy(spx_demag d, const double* m, const double* H, double* E, spx_stream_t s) {
  API_BEGIN
  REQUIRE(d);
  REQUIRE(m);
  REQUIRE(H);
  REQUIRE(E);
  if (d->d64) {
    *E = demag_energy<double>(*d->d64, m, H, S(s));
  } else {
    const int64_t n3 = 3 * d->d32->N;
    convert<double, float>(n3, m, d->tm.p, S(s));
    convert<double, float>(n3, H, d->th.p, S(s));
    *E = demag_energy<float>(*d->d32, d->tm.p, d->th.p, S(s));
  }
  API_END
}

int spx_demag_stats(spx_demag d, int64_t* i1, int64_t* i2, double* r1, double* r2) {
  API_BEGIN
  REQUIRE(d);
  const CgStats a = d->d64 ? d->d64->last1 : d->d32->last1;
  const CgStats b = d->d64 ? d->d64->last2 : d->d32->last2;
  if (i1) *i1 = a.iterations;
  if (i2) *i2 = b.iterations;
  if (r1) *r1 = a.rel_residual;
  if (r2) *r2 = b.rel_residual;
  API_END
}

int spx_demag_info(spx_demag d, int64_t* N, int64_t* Nb, int64_t* NI, int64_t* bytes) {
  API_BEGIN
  REQUIRE(d);
  if (d->d64) {
    if (N) *N = d->d64->N;
    if (Nb) *Nb = d->d64->Nb;
    if (NI) *NI = d->d64->NI;
    if (bytes) *bytes = d->d64->device_bytes();
  } else {
    if (N) *N = d->d32->N;
    if (Nb) *Nb = d->d32->Nb;
    if (NI) *NI = d->d32->NI;
    if (bytes) *bytes = d->d32->device_bytes();
  }
  API_END
}

int spx_demag_hmat(spx_demag d, spx_hmat* h) {
  API_BEGIN
  REQUIRE(d);
  REQUIRE(h);
  const int be = d->d64 ? d->d64->opt.backend : d->d32->opt.backend;
  SPX_CHECK(be == 1, "demag uses the dense boundary operator");
  *h = reinterpret_cast<spx_hmat>(d->d64 ? &d->d64->H : &d->d32->H);
  API_END
}

int spx_demag_profile_begin(spx_demag d) {
  API_BEGIN
  REQUIRE(d);
  if (d->d64) d->d64->prof.begin();
  else d->d32->prof.begin();
  API_END
}

int spx_demag_profile_end(spx_demag d, double* ms8, int64_t* l8, int64_t* g8) {
  API_BEGIN
  REQUIRE(d); REQUIRE(ms8); REQUIRE(l8); REQUIRE(g8);
  if (d->d64) d->d64->prof.end(ms8, l8, g8);
  else d->d32->prof.end(ms8, l8, g8);
  API_END
}

int spx_demag_counters(spx_demag d, int64_t* c1, int64_t* c2) {
  API_BEGIN
  REQUIRE(d);
  unsigned long long a[4] = {0, 0, 0, 0}, b[4] = {0, 0, 0, 0};
  auto rd = [](DevBuf<unsigned long long>& src, unsigned long long* dst) {
    if (src.n) SPX_CUDA(cudaMemcpy(dst, src.p, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  };
  if (d->d64) { rd(d->d64->cg1.iters_acc, a); rd(d->d64->cg2.iters_acc, b); }
  else { rd(d->d32->cg1.iters_acc, a); rd(d->d32->cg2.iters_acc, b); }
  for (int k = 0; k < 4; ++k) {
    if (c1) c1[k] = static_cast<int64_t>(a[k]);
    if (c2) c2[k] = static_cast<int64_t>(b[k]);
  }
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
  q.D_int = p->D_int; q.n_int = p->n_int; q.H0_nodes = p->H0_nodes;
  for (int c = 0; c < 3; ++c) q.H0_uniform[c] = p->H0_uniform[c];
  q.use_demag = p->use_demag;
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
  const bool f32 = d ? (d->d32 != nullptr) : (p->precision != 0);
  l->f32 = f32;
  if (!f32) {
    l->l64 = std::make_unique<LLGCtx<double>>();
    l->l64->create(d ? d->d64.get() : nullptr, X, N, tets, E, q, 0);
  } else {
    l->l32 = std::make_unique<LLGCtx<float>>();
    l->l32->create(d ? d->d32.get() : nullptr, X, N, tets, E, q, 0);
    l->ta.alloc(3 * N);
    l->tb.alloc(3 * N);
  }
  l->hstage.alloc(3 * N);
  *out = l.release();
  API_END
}

int spx_llg_heff(spx_llg l, const double* m, double* H, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(H);
  llg_call(l, m, H, s, [&](LLGCtx<double>& c, const double* a, double* b) { c.heff(a, b, true, S(s)); },
           [&](LLGCtx<float>& c, const float* a, float* b) { c.heff(a, b, true, S(s)); });
  API_END
}

int spx_llg_hjac(spx_llg l, const double* m, double* H, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(H);
  llg_call(l, m, H, s, [&](LLGCtx<double>& c, const double* a, double* b) { c.heff(a, b, false, S(s)); },
           [&](LLGCtx<float>& c, const float* a, float* b) { c.heff(a, b, false, S(s)); });
  API_END
}

int spx_llg_rhs(spx_llg l, const double* m, double* r, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m); REQUIRE(r);
  llg_call(l, m, r, s, [&](LLGCtx<double>& c, const double* a, double* b) { c.rhs(a, b, S(s)); },
           [&](LLGCtx<float>& c, const float* a, float* b) { c.rhs(a, b, S(s)); });
  API_END
}

int spx_llg_update_jac_state(spx_llg l, const double* m, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m);
  llg_call(l, m, nullptr, s, [&](LLGCtx<double>& c, const double* a, double*) { c.update_jac_state(a, S(s)); },
           [&](LLGCtx<float>& c, const float* a, float*) { c.update_jac_state(a, S(s)); });
  API_END
}

int spx_llg_jv(spx_llg l, const double* v, double* o, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(v); REQUIRE(o);
  llg_call(l, v, o, s, [&](LLGCtx<double>& c, const double* a, double* b) { c.jv(a, b, S(s)); },
           [&](LLGCtx<float>& c, const float* a, float* b) { c.jv(a, b, S(s)); });
  API_END
}

int spx_llg_pc_build(spx_llg l, double shift, int32_t include_stab, int32_t use_abs_kappa, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l);
  if (!l->f32) l->l64->pc_build(shift, include_stab, use_abs_kappa, S(s));
  else l->l32->pc_build(shift, include_stab, use_abs_kappa, S(s));
  API_END
}

int spx_llg_pc_apply(spx_llg l, const double* x, double* y, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(x); REQUIRE(y);
  llg_call(l, x, y, s, [&](LLGCtx<double>& c, const double* a, double* b) { c.pc_apply(a, b, S(s)); },
           [&](LLGCtx<float>& c, const float* a, float* b) { c.pc_apply(a, b, S(s)); });
  API_END
}

int spx_llg_set_state(spx_llg l, const double* m, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m);
  if (!l->f32) SPX_CUDA(cudaMemcpyAsync(l->l64->m.p, m, 3 * l->N * sizeof(double), cudaMemcpyDeviceToDevice, S(s)));
  else convert<double, float>(3 * l->N, m, l->l32->m.p, S(s));
  API_END
}

int spx_llg_get_state(spx_llg l, double* m, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m);
  if (!l->f32) SPX_CUDA(cudaMemcpyAsync(m, l->l64->m.p, 3 * l->N * sizeof(double), cudaMemcpyDeviceToDevice, S(s)));
  else convert<float, double>(3 * l->N, l->l32->m.p, m, S(s));
  API_END
}

int spx_llg_step(spx_llg l, double dt, int64_t nsteps, spx_stream_t s) {
  API_BEGIN
  REQUIRE(l);
  SPX_CHECK(nsteps >= 0, "nsteps must be non-negative");
  SPX_CHECK(dt > 0.0, "dt must be positive");
  if (!l->f32) l->l64->step_rk4(dt, nsteps, S(s));
  else l->l32->step_rk4(dt, nsteps, S(s));
  API_END
}

int spx_llg_run_host(spx_llg l, const double* m_in, double* m_out, double dt, int64_t nsteps) {
  API_BEGIN
  REQUIRE(l); REQUIRE(m_in); REQUIRE(m_out);
  SPX_CHECK(dt > 0.0 && nsteps >= 0, "dt must be positive and nsteps non-negative");
  const int64_t n3 = 3 * l->N;
  cudaStream_t s = 0;
  SPX_CUDA(cudaMemcpyAsync(l->hstage.p, m_in, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
  if (!l->f32) {
    SPX_CUDA(cudaMemcpyAsync(l->l64->m.p, l->hstage.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    l->l64->step_rk4(dt, nsteps, s);
    SPX_CUDA(cudaMemcpyAsync(l->hstage.p, l->l64->m.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  } else {
    convert<double, float>(n3, l->hstage.p, l->l32->m.p, s);
    l->l32->step_rk4(dt, nsteps, s);
    convert<float, double>(n3, l->l32->m.p, l->hstage.p, s);
  }
  SPX_CUDA(cudaMemcpyAsync(m_out, l->hstage.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  API_END
}

int spx_llg_set_uniform_field(spx_llg l, double hx, double hy, double hz) {
  API_BEGIN
  REQUIRE(l);
  if (!l->f32) {
    l->l64->H0.release();
    l->l64->h0[0] = hx; l->l64->h0[1] = hy; l->l64->h0[2] = hz;
  } else {
    l->l32->H0.release();
    l->l32->h0[0] = hx; l->l32->h0[1] = hy; l->l32->h0[2] = hz;
  }
  API_END
}

int spx_llg_stats(spx_llg l, int64_t* steps, int64_t* rhs, int64_t* launches) {
  API_BEGIN
  REQUIRE(l);
  if (!l->f32) {
    if (steps) *steps = l->l64->steps;
    if (rhs) *rhs = l->l64->rhs_evals;
    if (launches) *launches = l->l64->launches;
  } else {
    if (steps) *steps = l->l32->steps;
    if (rhs) *rhs = l->l32->rhs_evals;
    if (launches) *launches = l->l32->launches;
  }
  API_END
}

int spx_llg_destroy(spx_llg l) {
  API_BEGIN
  delete l;
  API_END
}

}  // extern "C"
