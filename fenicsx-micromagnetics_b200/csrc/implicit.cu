// Implicit relaxation driver on the device: variable-step BDF(2) whose stage equations
// F(y) = shift y + base - f(t1, y) = 0 are solved by Newton with quadratic backtracking and
// left-preconditioned restarted GMRES on the matrix-free operator shift I - J(y).
//
// Reference: LLG_GPU._ensure_solver / relax (gpu/solvers/llg_module_GPU.py:2052-2381), which
// drives PETSc TS "bdf" (order 2, TSAdapt "basic"), SNES newtonls + line search "bt" of order
// 2, KSP gmres with the python PC of JvContext (:1412-1547: the per-node 3x3 inverse of
// shift I - J_i, rebuilt with the Jacobian state in every IJacobian call), operator
// y = shift x - J x (JvContext.mult :1510-1517) and residual ydot - f (ifunction :1328-1340).
//
// Device work: the right-hand side (fused stage kernel, demag included), the Jacobian-vector
// product (k_jv, local: no demag), the block preconditioner, and the Krylov vector algebra
// below.  Every reduction runs over a fixed grid of partial sums with a fixed-order final
// sum, so results are run-to-run identical.  Scalars (Hessenberg column, norms) are read back
// once per GMRES iteration; the Givens rotations, the back substitution, the line search and
// the BDF coefficients are host arithmetic, as in PETSc.
//
// Algorithms: variable-step BDF through the Lagrange polynomial on the step's nodes; GMRES
// (Saad & Schultz, SIAM J. Sci. Stat. Comput. 7 (1986) 856-869) with classical Gram-Schmidt
// and Givens rotations; backtracking line search with a quadratic model (Dennis & Schnabel,
// "Numerical Methods for Unconstrained Optimization and Nonlinear Equations", 1983, 6.3).
#include "llg.cuh"

#include <cmath>

namespace spx {

namespace {

constexpr int IM_GRID = 592;   // partial sums per reduction (4 x 148 CTAs)
constexpr int IM_THREADS = 256;
constexpr int MDOT_CHUNK = 8;  // basis vectors per multi-dot CTA row

template <class TV>
struct Lin4 {
  const TV* v[4];
  double c[4];
  int n;
};

// out = sum_j c_j v_j (out may alias an input)
template <class TV>
__global__ void k_lin(int64_t n, Lin4<TV> a, TV* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int j = 0; j < a.n; ++j) v += a.c[j] * static_cast<double>(a.v[j][i]);
    out[i] = static_cast<TV>(v);
  }
}

// part[blk] = partial sum of a_i b_i
template <class TV>
__global__ void k_dot_part(int64_t n, const TV* __restrict__ a, const TV* __restrict__ b, double* __restrict__ part) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    acc += static_cast<double>(a[i]) * static_cast<double>(b[i]);
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// part[j][blk] = partial sums of <V_j, w> for j in [8 y, 8 y + 8) and j < nv
template <class TV>
__global__ void k_mdot_part(int64_t n, const TV* __restrict__ V, int64_t ld, int nv, const TV* __restrict__ w,
                            double* __restrict__ part) {
  __shared__ double sh[MDOT_CHUNK][32];
  const int j0 = blockIdx.y * MDOT_CHUNK;
  const int nj = min(MDOT_CHUNK, nv - j0);
  double acc[MDOT_CHUNK];
#pragma unroll
  for (int u = 0; u < MDOT_CHUNK; ++u) acc[u] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double wi = static_cast<double>(w[i]);
#pragma unroll
    for (int u = 0; u < MDOT_CHUNK; ++u)
      if (u < nj) acc[u] += static_cast<double>(V[(j0 + u) * ld + i]) * wi;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int u = 0; u < MDOT_CHUNK; ++u) {
    const double v = warp_sum(acc[u]);
    if (lane == 0) sh[u][wid] = v;
  }
  __syncthreads();
  if (wid < nj) {
    const int nw = (blockDim.x + 31) >> 5;
    double v = lane < nw ? sh[wid][lane] : 0.0;
    v = warp_sum(v);
    if (lane == 0) part[(int64_t)(j0 + wid) * gridDim.x + blockIdx.x] = v;
  }
}

// out[row] = sum of part[row][0..G) (one CTA per row, fixed order)
__global__ void k_rows_sum(int G, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < G; i += blockDim.x) s += part[(int64_t)blockIdx.x * G + i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// w -= sum_j h_j V_j and part[blk] = partial sum of the new w_i^2
template <class TV>
__global__ void k_maxpy_norm(int64_t n, const TV* __restrict__ V, int64_t ld, int nv, const double* __restrict__ h,
                             TV* __restrict__ w, double* __restrict__ part) {
  __shared__ double sh[32];
  __shared__ double hs[128];
  for (int j = threadIdx.x; j < nv; j += blockDim.x) hs[j] = h[j];
  __syncthreads();
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = static_cast<double>(w[i]);
    for (int j = 0; j < nv; ++j) v -= hs[j] * static_cast<double>(V[j * ld + i]);
    const TV t = static_cast<TV>(v);
    w[i] = t;
    acc += static_cast<double>(t) * static_cast<double>(t);
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// y += sum_j c_j V_j
template <class TV>
__global__ void k_maxpy(int64_t n, const TV* __restrict__ V, int64_t ld, int nv, const double* __restrict__ c,
                        TV* __restrict__ y) {
  __shared__ double cs[128];
  for (int j = threadIdx.x; j < nv; j += blockDim.x) cs[j] = c[j];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = static_cast<double>(y[i]);
    for (int j = 0; j < nv; ++j) v += cs[j] * static_cast<double>(V[j * ld + i]);
    y[i] = static_cast<TV>(v);
  }
}

// x *= 1 / sqrt(nrm2[0]) (zeros when the norm is zero: a breakdown vector is never used)
template <class TV>
__global__ void k_scale_inv_norm(int64_t n, const double* __restrict__ nrm2, TV* __restrict__ x) {
  const double q = nrm2[0];
  const double s = q > 0.0 ? 1.0 / sqrt(q) : 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = static_cast<TV>(s * static_cast<double>(x[i]));
}

// part[blk] = partial sum of (c (y_i - p_i) / (atol + rtol max(|y_i|, |m_i|)))^2
template <class TV>
__global__ void k_lte_part(int64_t n, const TV* __restrict__ y, const TV* __restrict__ p, const TV* __restrict__ m,
                           double c, double rtol, double atol, double* __restrict__ part) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double yi = static_cast<double>(y[i]);
    const double e = c * (yi - static_cast<double>(p[i]));
    const double tol = atol + rtol * fmax(fabs(yi), fabs(static_cast<double>(m[i])));
    const double r = e / tol;
    acc += r * r;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// Lagrange basis on nodes ts[0..k): values and derivatives at x
void lagrange_values(double x, const double* ts, int k, double* out) {
  for (int j = 0; j < k; ++j) {
    double v = 1.0;
    for (int m = 0; m < k; ++m)
      if (m != j) v *= (x - ts[m]) / (ts[j] - ts[m]);
    out[j] = v;
  }
}

void lagrange_derivs(double x, const double* ts, int k, double* out) {
  for (int j = 0; j < k; ++j) {
    double d = 0.0;
    for (int m = 0; m < k; ++m) {
      if (m == j) continue;
      double p = 1.0 / (ts[j] - ts[m]);
      for (int q = 0; q < k; ++q)
        if (q != j && q != m) p *= (x - ts[q]) / (ts[j] - ts[q]);
      d += p;
    }
    out[j] = d;
  }
}

}  // namespace

// ------------------------------------------------------------------ vector algebra helpers

template <class TV, class TM>
void LLGCtx<TV, TM>::im_lin(int nv, const TV* const* v, const double* c, TV* out, cudaStream_t s) {
  Lin4<TV> a{};
  a.n = nv;
  for (int j = 0; j < nv; ++j) {
    a.v[j] = v[j];
    a.c[j] = c[j];
  }
  k_lin<TV><<<grid_for(3 * N, IM_THREADS, 4 * num_sms()), IM_THREADS, 0, s>>>(3 * N, a, out);
  SPX_LAUNCH_CHECK();
  ++launches;
}

template <class TV, class TM>
double LLGCtx<TV, TM>::im_dot(const TV* a, const TV* b, cudaStream_t s) {
  k_dot_part<TV><<<IM_GRID, IM_THREADS, 0, s>>>(3 * N, a, b, im.part.p);
  SPX_LAUNCH_CHECK();
  k_rows_sum<<<1, IM_THREADS, 0, s>>>(IM_GRID, im.part.p, im.dev.p);
  SPX_LAUNCH_CHECK();
  launches += 2;
  double h = 0.0;
  SPX_CUDA(cudaMemcpyAsync(&h, im.dev.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  return h;
}

template <class TV, class TM>
void LLGCtx<TV, TM>::im_apply_A(double shift, const TV* v, TV* out, cudaStream_t s) {
  jv(v, im.t1.p, s);
  const TV* vs[2] = {v, im.t1.p};
  const double cs[2] = {shift, -1.0};
  im_lin(2, vs, cs, out, s);
  ++launches;
}

template <class TV, class TM>
void LLGCtx<TV, TM>::im_apply_P(const TV* x, TV* y, bool use_pc, cudaStream_t s) {
  if (use_pc) {
    pc_apply(x, y, s);
    ++launches;
  } else {
    SPX_CUDA(cudaMemcpyAsync(y, x, 3 * N * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  }
}

template <class TV, class TM>
double LLGCtx<TV, TM>::im_residual(double shift, const TV* y, TV* F, cudaStream_t s) {
  rhs(y, im.f.p, s);
  ++launches;
  ++im.fevals;
  const TV* vs[3] = {y, im.base.p, im.f.p};
  const double cs[3] = {shift, 1.0, -1.0};
  im_lin(3, vs, cs, F, s);
  return std::sqrt(im_dot(F, F, s));
}

// ------------------------------------------------------------------ GMRES

template <class TV, class TM>
int LLGCtx<TV, TM>::im_gmres(double shift, const TV* b, TV* x, const ImplicitOpts& o, int* its_out, cudaStream_t s) {
  const int64_t n3 = 3 * N;
  const int R = o.ksp_restart;
  const int64_t ld = n3;
  TV* V = im.V.p;
  const unsigned gl = grid_for(n3, IM_THREADS, 4 * num_sms());
  SPX_CUDA(cudaMemsetAsync(x, 0, n3 * sizeof(TV), s));
  im_apply_P(b, V, o.use_pc != 0, s);
  std::vector<double> Hh(static_cast<size_t>(R + 1) * R, 0.0), cs(R, 0.0), sn(R, 0.0), g(R + 1, 0.0), hcol(R + 2);
  auto H = [&](int i, int j) -> double& { return Hh[static_cast<size_t>(i) * R + j]; };
  int its = 0, reason = 0;
  bool first = true;
  double rnorm0 = 0.0, ttol = 0.0;
  while (true) {
    const double beta = std::sqrt(im_dot(V, V, s));
    if (first) {
      rnorm0 = beta;
      ttol = std::max(o.ksp_rtol * rnorm0, o.ksp_atol);
      first = false;
    }
    if (!std::isfinite(beta)) { reason = -9; break; }
    if (beta <= ttol) { reason = beta <= o.ksp_atol ? 3 : 2; break; }
    if (beta >= o.ksp_dtol * rnorm0) { reason = -4; break; }
    {
      const TV* vs[1] = {V};
      const double c1[1] = {1.0 / beta};
      im_lin(1, vs, c1, V, s);
    }
    std::fill(Hh.begin(), Hh.end(), 0.0);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int loc = 0;
    while (reason == 0 && loc < R && its < o.ksp_max_it) {
      TV* w = V + static_cast<int64_t>(loc + 1) * ld;
      im_apply_A(shift, V + static_cast<int64_t>(loc) * ld, im.t2.p, s);
      im_apply_P(im.t2.p, w, o.use_pc != 0, s);
      const int nv = loc + 1;
      dim3 gm(IM_GRID, (nv + MDOT_CHUNK - 1) / MDOT_CHUNK);
      k_mdot_part<TV><<<gm, IM_THREADS, 0, s>>>(n3, V, ld, nv, w, im.mpart.p);
      SPX_LAUNCH_CHECK();
      k_rows_sum<<<nv, IM_THREADS, 0, s>>>(IM_GRID, im.mpart.p, im.dev.p);
      SPX_LAUNCH_CHECK();
      k_maxpy_norm<TV><<<IM_GRID, IM_THREADS, 0, s>>>(n3, V, ld, nv, im.dev.p, w, im.part.p);
      SPX_LAUNCH_CHECK();
      k_rows_sum<<<1, IM_THREADS, 0, s>>>(IM_GRID, im.part.p, im.dev.p + nv);
      SPX_LAUNCH_CHECK();
      k_scale_inv_norm<TV><<<gl, IM_THREADS, 0, s>>>(n3, im.dev.p + nv, w);
      SPX_LAUNCH_CHECK();
      launches += 5;
      SPX_CUDA(cudaMemcpyAsync(hcol.data(), im.dev.p, (nv + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
      SPX_CUDA(cudaStreamSynchronize(s));
      const double tt = std::sqrt(hcol[nv]);
      for (int i = 0; i < nv; ++i) H(i, loc) = hcol[i];
      H(loc + 1, loc) = tt;
      const double hapbnd = std::min(std::fabs(tt / g[loc]), 1e-30);
      const bool hapend = tt < hapbnd;
      for (int i = 0; i < loc; ++i) {
        const double a0 = H(i, loc), a1 = H(i + 1, loc);
        H(i, loc) = cs[i] * a0 + sn[i] * a1;
        H(i + 1, loc) = cs[i] * a1 - sn[i] * a0;
      }
      double res = 0.0;
      if (!hapend) {
        const double a0 = H(loc, loc), a1 = H(loc + 1, loc);
        const double d = std::sqrt(a0 * a0 + a1 * a1);
        if (d == 0.0) {
          reason = -2;
          break;
        }
        cs[loc] = a0 / d;
        sn[loc] = a1 / d;
        g[loc + 1] = -(sn[loc] * g[loc]);
        g[loc] = cs[loc] * g[loc];
        H(loc, loc) = cs[loc] * a0 + sn[loc] * a1;
        res = std::fabs(g[loc + 1]);
      }
      ++loc;
      ++its;
      if (!std::isfinite(res)) reason = -9;
      else if (res <= ttol) reason = res <= o.ksp_atol ? 3 : 2;
      else if (res >= o.ksp_dtol * rnorm0) reason = -4;
      if (hapend) {
        if (reason == 0) reason = 5;
        break;
      }
    }
    if (loc > 0 && reason != -2) {
      std::vector<double> y(loc, 0.0);
      for (int k = loc - 1; k >= 0; --k) {
        double t = g[k];
        for (int j = k + 1; j < loc; ++j) t -= H(k, j) * y[j];
        y[k] = t / H(k, k);
      }
      SPX_CUDA(cudaMemcpyAsync(im.dev.p, y.data(), loc * sizeof(double), cudaMemcpyHostToDevice, s));
      k_maxpy<TV><<<gl, IM_THREADS, 0, s>>>(n3, V, ld, loc, im.dev.p, x);
      SPX_LAUNCH_CHECK();
      ++launches;
      // the host vector y must outlive the copy
      SPX_CUDA(cudaStreamSynchronize(s));
    }
    if (reason != 0) break;
    if (its >= o.ksp_max_it) {
      reason = -3;
      break;
    }
    // restart from the explicit residual P^-1 (b - A x)
    im_apply_A(shift, x, im.t2.p, s);
    const TV* vs[2] = {b, im.t2.p};
    const double c2[2] = {1.0, -1.0};
    im_lin(2, vs, c2, im.t2.p, s);
    im_apply_P(im.t2.p, V, o.use_pc != 0, s);
  }
  *its_out = its;
  return reason;
}

// ------------------------------------------------------------------ Newton

template <class TV, class TM>
int LLGCtx<TV, TM>::im_newton(double shift, TV* y, const ImplicitOpts& o, int* nits, int* lits, cudaStream_t s) {
  const int64_t n3 = 3 * N;
  *nits = 0;
  *lits = 0;
  double fnorm = im_residual(shift, y, im.F.p, s);
  if (!std::isfinite(fnorm)) return -4;
  const double fnorm0 = fnorm, ttol = fnorm * o.snes_rtol;
  if (fnorm < o.snes_atol) return 2;
  for (int it = 0; it < o.snes_max_it; ++it) {
    // IJacobian: Jacobian state at y and the block preconditioner for this shift
    update_jac_state(y, s);
    if (o.use_pc) pc_build(shift, 1, 1, s);
    launches += 2;
    int kits = 0;
    const int kr = im_gmres(shift, im.F.p, im.Y.p, o, &kits, s);
    *lits += kits;
    *nits = it + 1;
    if (kr < 0 && kr != -3) return -3;
    // line search along -Y
    const double xnorm = std::sqrt(im_dot(y, y, s));
    double ynorm = std::sqrt(im_dot(im.Y.p, im.Y.p, s));
    if (ynorm == 0.0) return o.snes_stol * xnorm > ynorm ? 4 : -6;
    if (ynorm > o.ls_maxstep) {
      const TV* vs[1] = {im.Y.p};
      const double c[1] = {o.ls_maxstep / ynorm};
      im_lin(1, vs, c, im.Y.p, s);
      ynorm = o.ls_maxstep;
    }
    const double f = fnorm * fnorm;
    im_apply_A(shift, im.Y.p, im.t2.p, s);
    double slope = im_dot(im.F.p, im.t2.p, s);
    if (slope > 0.0) slope = -slope;
    if (slope == 0.0) slope = -1.0;
    double lam = 1.0;
    auto trial = [&](double l) {
      const TV* vs[2] = {y, im.Y.p};
      const double c[2] = {1.0, -l};
      im_lin(2, vs, c, im.W.p, s);
      const double gn = im_residual(shift, im.W.p, im.G.p, s);
      return gn * gn;
    };
    double g = trial(lam);
    bool ok = false, nan = !std::isfinite(g);
    if (!nan && 0.5 * g <= 0.5 * f + lam * o.ls_alpha * slope) {
      ok = true;
    } else if (!nan && !(o.snes_stol * xnorm > ynorm)) {
      for (int c = 0; c <= o.ls_max_it; ++c) {
        if (lam <= o.ls_minlambda) break;
        double lt = -slope * lam * lam / (g - f - 2.0 * lam * slope);
        if (lt > 0.5 * lam) lt = 0.5 * lam;
        lam = lt <= 0.1 * lam ? 0.1 * lam : lt;
        g = trial(lam);
        if (!std::isfinite(g)) {
          nan = true;
          break;
        }
        if (0.5 * g < 0.5 * f + lam * o.ls_alpha * slope) {
          ok = true;
          break;
        }
      }
    }
    if (!ok) return o.snes_stol * xnorm > ynorm ? 4 : -6;
    SPX_CUDA(cudaMemcpyAsync(y, im.W.p, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
    std::swap(im.F, im.G);
    fnorm = std::sqrt(g);
    const double xn = std::sqrt(im_dot(y, y, s));
    if (!std::isfinite(fnorm)) return -4;
    if (fnorm < o.snes_atol) return 2;
    if (fnorm <= ttol) return 3;
    if (ynorm < o.snes_stol * xn) return 4;
    if (fnorm > o.snes_divtol * fnorm0) return -10;
  }
  return -5;
}

// ------------------------------------------------------------------ BDF attempt / accept

template <class TV, class TM>
void LLGCtx<TV, TM>::im_alloc() {
  const size_t n3 = static_cast<size_t>(3 * N);
  for (DevBuf<TV>* b : {&im.hist[0], &im.hist[1], &im.half, &im.cand, &im.pred, &im.base, &im.f, &im.F, &im.G,
                        &im.W, &im.Y, &im.t1, &im.t2})
    if (b->n != n3) b->alloc(n3);
  if (im.part.n != static_cast<size_t>(IM_GRID)) im.part.alloc(IM_GRID);
  if (im.dev.n != 256) im.dev.alloc(256);
}

template <class TV, class TM>
ImplicitResult LLGCtx<TV, TM>::bdf_attempt(double t, double dt, const ImplicitOpts& o, const double* htu,
                                           const TV* htn, cudaStream_t s) {
  SPX_CHECK(o.ksp_restart >= 1 && o.ksp_restart <= 100, "ksp_restart must be in [1, 100]");
  im_alloc();
  const int64_t n3 = 3 * N;
  const size_t vneed = static_cast<size_t>(o.ksp_restart + 1) * n3;
  if (im.V.n != vneed) im.V.alloc(vneed);
  const size_t mneed = static_cast<size_t>(o.ksp_restart + 1) * IM_GRID;
  if (im.mpart.n < mneed) im.mpart.alloc(mneed);
  graph_reset();
  rk_fsal = false;
  im.has_cand = false;
  const bool time_field = htu || htn;
  auto set_field = [&](int st) {
    if (!time_field) return;
    const double zero[3] = {0.0, 0.0, 0.0};
    set_time_field(htu ? htu + 3 * st : zero, htn ? htn + n3 * st : nullptr, s);
  };
  ImplicitResult r{};
  r.wlte = -1.0;
  const double t1 = t + dt;
  // stage nodes: times and vectors (newest first), predictor nodes
  double ts[3], tp[3];
  const TV* ys[3];
  const TV* yp[3];
  int k = 0, kp = 0;
  r.restarted = im.n == 0;
  if (r.restarted) {
    // backward-Euler half step to t + dt/2 from the predictor m
    const double th = t + 0.5 * dt;
    set_field(0);
    double a[2];
    const double tn[2] = {th, t};
    lagrange_derivs(th, tn, 2, a);
    {
      const TV* vs[1] = {m.p};
      const double c[1] = {a[1]};
      im_lin(1, vs, c, im.base.p, s);
    }
    SPX_CUDA(cudaMemcpyAsync(im.half.p, m.p, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
    int ni = 0, li = 0;
    r.snes_reason = im_newton(a[0], im.half.p, o, &ni, &li, s);
    r.newton_its += ni;
    r.linear_its += li;
    if (r.snes_reason < 0) {
      r.order = 2;
      r.fevals = static_cast<int>(im.fevals);
      im.fevals = 0;
      return r;
    }
    ts[0] = th; ys[0] = im.half.p;
    ts[1] = t;  ys[1] = m.p;
    k = 2;
    for (int j = 0; j < 2; ++j) { tp[j] = ts[j]; yp[j] = ys[j]; }
    kp = 2;
  } else {
    ts[0] = t;  ys[0] = m.p;
    ts[1] = im.t[0]; ys[1] = im.hist[0].p;
    k = 2;
    tp[0] = t; yp[0] = m.p;
    tp[1] = im.t[0]; yp[1] = im.hist[0].p;
    kp = 2;
    if (im.n >= 2) {
      tp[2] = im.t[1];
      yp[2] = im.hist[1].p;
      kp = 3;
    }
  }
  // BDF coefficients on [t1, nodes...]: shift = L_0'(t1), base = sum_j L_j'(t1) y_j
  double nodes[4], a[4], lv[3];
  nodes[0] = t1;
  for (int j = 0; j < k; ++j) nodes[j + 1] = ts[j];
  lagrange_derivs(t1, nodes, k + 1, a);
  {
    double c[3];
    for (int j = 0; j < k; ++j) c[j] = a[j + 1];
    im_lin(k, ys, c, im.base.p, s);
  }
  lagrange_values(t1, tp, kp, lv);
  im_lin(kp, yp, lv, im.pred.p, s);
  SPX_CUDA(cudaMemcpyAsync(im.cand.p, im.pred.p, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  set_field(1);
  int ni = 0, li = 0;
  r.snes_reason = im_newton(a[0], im.cand.p, o, &ni, &li, s);
  r.newton_its += ni;
  r.linear_its += li;
  r.order = kp;
  r.fevals = static_cast<int>(im.fevals);
  im.fevals = 0;
  if (r.snes_reason < 0) return r;
  double t_old = tp[0];
  for (int j = 1; j < kp; ++j) t_old = std::min(t_old, tp[j]);
  const double c = dt / (t1 - t_old);
  k_lte_part<TV><<<IM_GRID, IM_THREADS, 0, s>>>(n3, im.cand.p, im.pred.p, m.p, c, o.rtol, o.atol, im.part.p);
  SPX_LAUNCH_CHECK();
  k_rows_sum<<<1, IM_THREADS, 0, s>>>(IM_GRID, im.part.p, im.dev.p);
  SPX_LAUNCH_CHECK();
  launches += 2;
  double sum = 0.0;
  SPX_CUDA(cudaMemcpyAsync(&sum, im.dev.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  r.wlte = std::sqrt(sum / static_cast<double>(n3));
  im.has_cand = true;
  im.cand_t = t1;
  im.cand_restart = r.restarted != 0;
  im.cand_th = ts[0];
  im.cand_t0 = t;
  return r;
}

template <class TV, class TM>
void LLGCtx<TV, TM>::bdf_accept(cudaStream_t s) {
  (void)s;
  SPX_CHECK(im.has_cand, "no converged BDF attempt to accept");
  graph_reset();
  rk_fsal = false;
  if (im.cand_restart) {
    // history: the half step (t + dt/2) and the old state (t)
    std::swap(im.hist[0], im.half);
    std::swap(im.hist[1], m);
    im.t[0] = im.cand_th;
    im.t[1] = im.cand_t0;
  } else {
    std::swap(im.hist[1], im.hist[0]);
    std::swap(im.hist[0], m);
    im.t[1] = im.t[0];
    im.t[0] = im.cand_t0;
  }
  std::swap(m, im.cand);
  im.n = 2;
  im.has_cand = false;
  ++steps;
}

#define SPX_IM_INST(TV, TM)                                                                                        \
  template ImplicitResult LLGCtx<TV, TM>::bdf_attempt(double, double, const ImplicitOpts&, const double*, const TV*, \
                                                      cudaStream_t);                                               \
  template void LLGCtx<TV, TM>::bdf_accept(cudaStream_t);
SPX_IM_INST(double, double)
SPX_IM_INST(float, float)
SPX_IM_INST(double, float)
#undef SPX_IM_INST

}  // namespace spx
