// Time integration drivers on the device: the time-dependent applied field, the embedded
// Dormand-Prince 5(4) step of the reference's explicit relaxation, and the max |dm| / dt
// reduction of its dm/dt stopping test.
//
// Reference: LLG_GPU._ensure_solver_explicit / relax_explicit
// (gpu/solvers/llg_module_GPU.py:1724-1970) drive PETSc TS "rk" of type "5dp" with the
// "basic" step adaptor, and StopByMaxDmdtFDGPU (:314-382) stops on max_i |m_i - m_prev_i| /
// (t - t_prev) in deg/ns.  Here each attempt's stages run as fused stage kernels (mode 1:
// the LLG right-hand side, demag and time field included) plus one linear-combination kernel
// per stage; the error norm is a fixed-order reduction read back as one scalar per attempt.
// The accept / reject / step-size logic is host code (spinfemx_b200/llg.py), as in PETSc.
//
// Dormand-Prince 5(4) tableau: J. R. Dormand and P. J. Prince, "A family of embedded
// Runge-Kutta formulae", J. Comput. Appl. Math. 6 (1980) 19-26 (the coefficients every
// DP5 implementation uses; the 5th-order row is the 7th stage's input, first same as last).
#include "llg.cuh"

namespace spx {

namespace {

constexpr double DP_C[7] = {0.0, 1.0 / 5.0, 3.0 / 10.0, 4.0 / 5.0, 8.0 / 9.0, 1.0, 1.0};
constexpr double DP_A[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5.0, 0, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
    {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
// 4th-order weights (the embedded solution)
constexpr double DP_BS[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0, -92097.0 / 339200.0,
                             187.0 / 2100.0, 1.0 / 40.0};
constexpr int ERR_GRID = 592;  // partial sums of the error norm (4 x 148 CTAs, fixed)

template <class TV>
struct Comb {
  const TV* k[7];
  TV c[7];
  int nk;
};

// out = m + sum_j c_j k_j
template <class TV>
__global__ void k_rk_combine(int64_t n3, const TV* __restrict__ m, Comb<TV> cb, TV* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x) {
    TV v = m[i];
    for (int j = 0; j < cb.nk; ++j)
      if (cb.c[j] != TV(0)) v += cb.c[j] * cb.k[j][i];
    out[i] = v;
  }
}

// partial sums of (e_i / tol_i)^2 with e = sum_j c_j k_j (c = dt (b - b*)), y5 = ynew,
// y4 = y5 - e, tol_i = atol + rtol max(|y5_i|, |y4_i|)
template <class TV>
__global__ void k_rk_err(int64_t n3, const TV* __restrict__ ynew, Comb<TV> cb, double rtol, double atol,
                         double* __restrict__ part) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x) {
    double e = 0.0;
    for (int j = 0; j < cb.nk; ++j) e += static_cast<double>(cb.c[j]) * static_cast<double>(cb.k[j][i]);
    const double y5 = static_cast<double>(ynew[i]);
    const double y4 = y5 - e;
    const double tol = atol + rtol * fmax(fabs(y5), fabs(y4));
    const double r = e / tol;
    acc += r * r;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void k_sum_fixed(int n, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) out[0] = s;
}

// per-CTA max over nodes of |a_i - b_i| (AoS [n][3])
__global__ void k_node_diff_max(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                                double* __restrict__ part) {
  __shared__ double sh[32];
  double mx = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double dx = a[3 * i] - b[3 * i], dy = a[3 * i + 1] - b[3 * i + 1], dz = a[3 * i + 2] - b[3 * i + 2];
    mx = fmax(mx, sqrt(dx * dx + dy * dy + dz * dz));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = mx;
  __syncthreads();
  if (wid == 0) {
    mx = lane < static_cast<int>((blockDim.x + 31) >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) part[blockIdx.x] = mx;
  }
}

}  // namespace

template <class TV, class TM>
void LLGCtx<TV, TM>::set_time_field(const double* h3, const TV* h_nodes, cudaStream_t s) {
  graph_reset();
  rk_fsal = false;
  ht[0] = h3 ? h3[0] : 0.0;
  ht[1] = h3 ? h3[1] : 0.0;
  ht[2] = h3 ? h3[2] : 0.0;
  if (h_nodes) {
    if (ht_nodes.n != static_cast<size_t>(3 * N)) ht_nodes.alloc(3 * N);
    SPX_CUDA(cudaMemcpyAsync(ht_nodes.p, h_nodes, 3 * N * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  } else {
    ht_nodes.release();
  }
}

template <class TV, class TM>
double LLGCtx<TV, TM>::rk_attempt(double dt, double rtol, double atol, const double* htu, const TV* htn,
                                  bool reuse_fsal, cudaStream_t s) {
  const int64_t n3 = 3 * N;
  for (int j = 0; j < 7; ++j)
    if (rk_k[j].n != static_cast<size_t>(n3)) rk_k[j].alloc(n3);
  if (rk_y.n != static_cast<size_t>(n3)) rk_y.alloc(n3);
  if (rk_ynew.n != static_cast<size_t>(n3)) rk_ynew.alloc(n3);
  if (rk_part.n != static_cast<size_t>(ERR_GRID + 1)) rk_part.alloc(ERR_GRID + 1);
  const bool time_field = htu || htn;
  auto eval = [&](const TV* y, TV* k, int st) {
    if (use_demag) demag->potential(y, s, false, -1);
    StageArgs<TV, TM> a = args(y, k, 1, use_demag);
    if (time_field) {
      a.htx = htu ? static_cast<TV>(htu[3 * st]) : TV(0);
      a.hty = htu ? static_cast<TV>(htu[3 * st + 1]) : TV(0);
      a.htz = htu ? static_cast<TV>(htu[3 * st + 2]) : TV(0);
      a.Ht = htn ? htn + n3 * st : nullptr;
    }
    launch_stage(a, use_demag, s);
    ++rhs_evals;
  };
  const unsigned g = grid_for(n3, 256, 4 * num_sms());
  if (!(reuse_fsal && rk_fsal)) eval(m.p, rk_k[0].p, 0);
  for (int st = 1; st < 7; ++st) {
    Comb<TV> cb{};
    cb.nk = st;
    for (int j = 0; j < st; ++j) {
      cb.k[j] = rk_k[j].p;
      cb.c[j] = static_cast<TV>(dt * DP_A[st][j]);
    }
    TV* y = st == 6 ? rk_ynew.p : rk_y.p;
    k_rk_combine<TV><<<g, 256, 0, s>>>(n3, m.p, cb, y);
    SPX_LAUNCH_CHECK();
    eval(y, rk_k[st].p, st);
  }
  Comb<TV> ce{};
  ce.nk = 7;
  for (int j = 0; j < 7; ++j) {
    ce.k[j] = rk_k[j].p;
    ce.c[j] = static_cast<TV>(dt * ((j < 6 ? DP_A[6][j] : 0.0) - DP_BS[j]));
  }
  k_rk_err<TV><<<ERR_GRID, 256, 0, s>>>(n3, rk_ynew.p, ce, rtol, atol, rk_part.p);
  SPX_LAUNCH_CHECK();
  k_sum_fixed<<<1, 256, 0, s>>>(ERR_GRID, rk_part.p, rk_part.p + ERR_GRID);
  SPX_LAUNCH_CHECK();
  double sum = 0.0;
  SPX_CUDA(cudaMemcpyAsync(&sum, rk_part.p + ERR_GRID, sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  launches += 6 + 2 + (reuse_fsal && rk_fsal ? 6 : 7);
  return std::sqrt(sum / static_cast<double>(n3));
}

template <class TV, class TM>
void LLGCtx<TV, TM>::rk_accept(cudaStream_t s) {
  (void)s;
  graph_reset();
  std::swap(m, rk_ynew);
  std::swap(rk_k[0], rk_k[6]);
  rk_fsal = true;
  ++steps;
}

#define SPX_DRV_INST(TV, TM)                                                                                   \
  template void LLGCtx<TV, TM>::set_time_field(const double*, const TV*, cudaStream_t);                          \
  template double LLGCtx<TV, TM>::rk_attempt(double, double, double, const double*, const TV*, bool, cudaStream_t); \
  template void LLGCtx<TV, TM>::rk_accept(cudaStream_t);
SPX_DRV_INST(double, double)
SPX_DRV_INST(float, float)
SPX_DRV_INST(double, float)
#undef SPX_DRV_INST

double node_diff_max(int64_t n, const double* a, const double* b, cudaStream_t s) {
  constexpr int G = 296;
  DevBuf<double> part(G + 1);
  k_node_diff_max<<<G, 256, 0, s>>>(n, a, b, part.p);
  SPX_LAUNCH_CHECK();
  std::vector<double> h(G);
  SPX_CUDA(cudaMemcpyAsync(h.data(), part.p, G * sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  double mx = 0.0;
  for (double v : h) mx = std::max(mx, v);
  return mx;
}

}  // namespace spx
