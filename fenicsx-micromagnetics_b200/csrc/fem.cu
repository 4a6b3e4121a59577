// FEM operators, persistent CG and the FEM/BEM demag pipeline on the device.
//
// Pipeline per call (DemagFieldLindholmGPU.compute_vec, gpu/fields/Demag_Lindholm_GPU.py:643-670):
//   b  = Ms int grad v . m                      k_div   (+ sum b for the null space)
//   u1 : A u1 = b - mean(b), u1 -= mean(u1)     k_cg    (:569-582; PETSc CG+GAMG there)
//   g  = B u1|bnd                               dense GEMV or H-matrix (:585-616)
//   u2 : A_II u_I = -A_IB g, u2|bnd = g          k_cg    (:618-640)
//   phi = u1 + u2 ;  H = G phi / V_i            k_grad  (:659-670)
// The Dirichlet problem is solved on the interior unknowns only; DOLFINx's identity
// rows for the boundary dofs (assemble_matrix with bcs) give the same interior
// solution.  CG stops when ||r||_2 <= max(rtol ||b||_2, atol) (unpreconditioned
// residual, the KSP default test with a zero initial guess) or after maxit.
#include <algorithm>
#include <cmath>

#include "fem.cuh"

namespace spx {

// ------------------------------------------------------------------ SELL kernels
// one warp per 32-row slice; thread = row
#define SELL_ROW_LOOP(nslices, ...)                                                    \
  {                                                                                     \
    const int lane_ = threadIdx.x & 31;                                                 \
    const int64_t gw_ = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;           \
    const int64_t nw_ = (gridDim.x * (int64_t)blockDim.x) >> 5;                          \
    for (int64_t sl_ = gw_; sl_ < (nslices); sl_ += nw_) {                              \
      const int64_t row = sl_ * 32 + lane_;                                             \
      const int64_t base_ = sp[sl_];                                                    \
      const int width = static_cast<int>((sp[sl_ + 1] - base_) >> 5);                   \
      __VA_ARGS__                                                                       \
    }                                                                                   \
  }

template <class T>
__global__ void k_div(int64_t n, int64_t nslices, const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                      const T* __restrict__ D, int64_t L, const T* __restrict__ m, T* __restrict__ b,
                      double* __restrict__ bsum) {
  __shared__ double sh[32];
  double part = 0.0;
  SELL_ROW_LOOP(nslices, {
    if (row < n) {
      T acc = 0;
      for (int k = 0; k < width; ++k) {
        const int64_t idx = base_ + ((int64_t)k << 5) + lane_;
        const int64_t j = col[idx];
        acc += D[idx] * m[3 * j] + D[L + idx] * m[3 * j + 1] + D[2 * L + idx] * m[3 * j + 2];
      }
      b[row] = acc;
      part += static_cast<double>(acc);
    }
  })
  const double t = block_sum(part, sh);
  if (threadIdx.x == 0 && bsum) atomicAdd(bsum, t);
}

template <class T>
__global__ void k_grad(int64_t n, int64_t nslices, const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                       const T* __restrict__ Gv, int64_t L, const T* __restrict__ phi, T* __restrict__ H) {
  SELL_ROW_LOOP(nslices, {
    if (row < n) {
      T hx = 0, hy = 0, hz = 0;
      for (int k = 0; k < width; ++k) {
        const int64_t idx = base_ + ((int64_t)k << 5) + lane_;
        const T p = phi[col[idx]];
        hx += Gv[idx] * p;
        hy += Gv[L + idx] * p;
        hz += Gv[2 * L + idx] * p;
      }
      H[3 * row] = hx;
      H[3 * row + 1] = hy;
      H[3 * row + 2] = hz;
    }
  })
}

template <class T>
__global__ void k_u2rhs(int64_t n, int64_t nslices, const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                        const T* __restrict__ v, const T* __restrict__ g, T* __restrict__ b) {
  SELL_ROW_LOOP(nslices, {
    if (row < n) {
      T acc = 0;
      for (int k = 0; k < width; ++k) {
        const int64_t idx = base_ + ((int64_t)k << 5) + lane_;
        acc += v[idx] * g[col[idx]];
      }
      b[row] = -acc;
    }
  })
}

template <class T>
__global__ void k_phi_interior(int64_t NI, const int32_t* __restrict__ interior, const T* __restrict__ u1,
                               const T* __restrict__ xI, T* __restrict__ phi) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < NI) {
    const int32_t g = interior[i];
    phi[g] = u1[g] + xI[i];
  }
}

template <class T>
__global__ void k_gather_idx(int64_t n, const int32_t* __restrict__ idx, const T* __restrict__ src, T* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

// dense B (FP64, row-major Nb x Nb): warp per row; g = B xb ; phi[bverts] = u1 + g
template <class T>
__global__ void k_dense_gemv(int64_t Nb, const double* __restrict__ B, const T* __restrict__ xb,
                             const int32_t* __restrict__ bverts, const T* __restrict__ u1, T* __restrict__ phi,
                             T* __restrict__ gB) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t i = w; i < Nb; i += nw) {
    const double* row = B + i * Nb;
    double acc = 0.0;
    for (int64_t j = lane; j < Nb; j += 32) acc += row[j] * static_cast<double>(xb[j]);
    acc = warp_sum(acc);
    if (lane == 0) {
      const T y = static_cast<T>(acc);
      gB[i] = y;
      if (phi) phi[bverts[i]] = u1[bverts[i]] + y;
    }
  }
}

// ------------------------------------------------------------------ persistent pipelined CG
template <class T>
struct CgParams {
  int64_t n, nslices;
  const int64_t* sp;
  const int32_t* col;
  const T* val;
  const T* sdinv;
  const T* diag;
  const T* b;
  T* x;
  T *r, *w0, *w1, *p, *s, *z, *y;
  double* red;  // [0..11] 3 slots x (gamma, delta, rho, -); [12] sum b; [13] ||b||^2; [14] sum x
  unsigned int* bar;
  int* err;
  int* iters;
  double* resid;
  unsigned long long* iters_acc;  // [0] inner iterations, [1] outer steps, [2] solves (accumulated)
  double rtol, atol;
  int maxit, warm, project;
};

template <class T>
__device__ __forceinline__ T spmv_row(const CgParams<T>& P, int64_t base, int width, int lane, const T* v) {
  T acc = 0;
  for (int k = 0; k < width; ++k) {
    const int64_t idx = base + ((int64_t)k << 5) + lane;
    acc += P.val[idx] * v[P.col[idx]];
  }
  return acc;
}

template <class T>
__global__ void __launch_bounds__(256) k_cg(CgParams<T> P) {
  __shared__ double sh[32];
  const unsigned nb = gridDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  unsigned int* cnt = P.bar;
  unsigned int* gen = P.bar + 1;
  const int64_t n = P.n;
#define ROWS_BEGIN                                                  \
  for (int64_t sl = gw; sl < P.nslices; sl += nw) {                 \
    const int64_t row = sl * 32 + lane;                             \
    const int64_t base = P.sp[sl];                                  \
    const int width = static_cast<int>((P.sp[sl + 1] - base) >> 5); \
    (void)base; (void)width;                                        \
    if (row < n) {
#define ROWS_END \
  }              \
  }

  // phase 0: sum of b (null space)
  if (P.project) {
    double part = 0.0;
    ROWS_BEGIN part += static_cast<double>(P.b[row]);
    ROWS_END
    const double t = block_sum(part, sh);
    if (threadIdx.x == 0) atomicAdd(P.red + 12, t);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  const double meanb = P.project ? P.red[12] / static_cast<double>(n) : 0.0;
  // phase 1: b^ (kept in r), y0, ||b||^2
  {
    double bb = 0.0;
    ROWS_BEGIN
      const double bv = static_cast<double>(P.b[row]) - meanb;
      P.r[row] = static_cast<T>(bv) * P.sdinv[row];
      P.y[row] = P.warm ? P.x[row] / P.sdinv[row] : T(0);
      bb += bv * bv;
    ROWS_END
    const double t = block_sum(bb, sh);
    if (threadIdx.x == 0) atomicAdd(P.red + 13, t);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  // phase 2: r0 = b^ - A^ y0
  if (P.warm) {
    ROWS_BEGIN P.r[row] -= spmv_row(P, base, width, lane, P.y);
    ROWS_END
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  // phase 3: w0 = A^ r0, slot 0 <- (r,r), (w,r), rho
  {
    double g = 0.0, dl = 0.0, rh = 0.0;
    ROWS_BEGIN
      const T w = spmv_row(P, base, width, lane, P.r);
      P.w0[row] = w;
      const double rv = static_cast<double>(P.r[row]);
      g += rv * rv;
      dl += static_cast<double>(w) * rv;
      rh += static_cast<double>(P.diag[row]) * rv * rv;
    ROWS_END
    g = block_sum(g, sh);
    dl = block_sum(dl, sh);
    rh = block_sum(rh, sh);
    if (threadIdx.x == 0) {
      atomicAdd(P.red + 0, g);
      atomicAdd(P.red + 1, dl);
      atomicAdd(P.red + 2, rh);
    }
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  const double bb = P.red[13];
  const double tol2 = fmax(P.rtol * P.rtol * bb, P.atol * P.atol);
  double gprev = 1.0, aprev = 1.0, rho = 0.0;
  int it = 0;
  for (;; ++it) {
    const int sl = it % 3;
    const double gm = P.red[4 * sl], dl = P.red[4 * sl + 1];
    rho = P.red[4 * sl + 2];
    if (rho <= tol2 || it >= P.maxit || !(gm > 0.0)) break;
    if (blockIdx.x == 0 && threadIdx.x < 4) P.red[4 * ((it + 2) % 3) + threadIdx.x] = 0.0;
    double beta, alpha;
    if (it == 0) {
      beta = 0.0;
      alpha = gm / dl;
    } else {
      beta = gm / gprev;
      alpha = gm / (dl - beta * gm / aprev);
    }
    const T a = static_cast<T>(alpha), bt = static_cast<T>(beta);
    const T* wc = (it & 1) ? P.w1 : P.w0;
    T* wn = (it & 1) ? P.w0 : P.w1;
    double g2 = 0.0, d2 = 0.0, r2 = 0.0;
    ROWS_BEGIN
      const T nv = spmv_row(P, base, width, lane, wc);
      const T wv = wc[row];
      const T rv = P.r[row];
      T zv, sv, pv;
      if (it == 0) {
        zv = nv; sv = wv; pv = rv;
      } else {
        zv = nv + bt * P.z[row];
        sv = wv + bt * P.s[row];
        pv = rv + bt * P.p[row];
      }
      P.z[row] = zv;
      P.s[row] = sv;
      P.p[row] = pv;
      P.y[row] += a * pv;
      const T rn = rv - a * sv;
      const T wnv = wv - a * zv;
      P.r[row] = rn;
      wn[row] = wnv;
      const double rd = static_cast<double>(rn);
      g2 += rd * rd;
      d2 += static_cast<double>(wnv) * rd;
      r2 += static_cast<double>(P.diag[row]) * rd * rd;
    ROWS_END
    g2 = block_sum(g2, sh);
    d2 = block_sum(d2, sh);
    r2 = block_sum(r2, sh);
    if (threadIdx.x == 0) {
      const int ns = (it + 1) % 3;
      atomicAdd(P.red + 4 * ns, g2);
      atomicAdd(P.red + 4 * ns + 1, d2);
      atomicAdd(P.red + 4 * ns + 2, r2);
    }
    gprev = gm;
    aprev = alpha;
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  // epilogue: x = D^-1/2 y (- mean)
  double sx = 0.0;
  ROWS_BEGIN
    const T xv = P.y[row] * P.sdinv[row];
    P.x[row] = xv;
    sx += static_cast<double>(xv);
  ROWS_END
  if (P.project) {
    sx = block_sum(sx, sh);
    if (threadIdx.x == 0) atomicAdd(P.red + 14, sx);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
    const T mx = static_cast<T>(P.red[14] / static_cast<double>(n));
    ROWS_BEGIN P.x[row] -= mx;
    ROWS_END
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *P.iters = it;
    *P.resid = bb > 0.0 ? sqrt(rho / bb) : 0.0;
    atomicAdd(P.iters_acc, (unsigned long long)it);
    atomicAdd(P.iters_acc + 1, 1ull);
    atomicAdd(P.iters_acc + 2, 1ull);
  }
#undef ROWS_BEGIN
#undef ROWS_END
}

// ------------------------------------------------------------------ mixed-precision IR solve
// FP32 systems: FP64 outer iterative refinement (true residual with FP64 values, FP64
// solution kept between calls for warm starts) around an FP32 inner single-reduction
// (Chronopoulos-Gear) CG, all inside one cooperative launch.  Per inner iteration two
// grid barriers; per outer iteration three.
struct CgIrParams {
  int64_t n, nslices;
  const int64_t* sp;
  const int32_t* col;
  const float* v32;
  const double* v64;
  const double* sdinv;
  const double* diag;
  const float* b;
  float* x;
  double *bh, *y;
  float *r, *p, *q, *s, *d;
  double* red;  // [0] sum b, [1] ||b||^2, [2] sum x, [4..5] outer rho, [8..13] inner (gamma, delta) x 3
  unsigned int* bar;
  int* err;
  int* iters;
  double* resid;
  unsigned long long* iters_acc;
  double rtol, atol, inner_rtol;
  int maxit, max_outer, inner_maxit, warm, project;
};

__global__ void __launch_bounds__(256) k_cg_ir(CgIrParams P) {
  __shared__ double sh[32];
  const unsigned nb = gridDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  unsigned int* cnt = P.bar;
  unsigned int* gen = P.bar + 1;
  const int64_t n = P.n;
#define IR_ROWS_BEGIN                                               \
  for (int64_t sl = gw; sl < P.nslices; sl += nw) {                 \
    const int64_t row = sl * 32 + lane;                             \
    const int64_t base = P.sp[sl];                                  \
    const int width = static_cast<int>((P.sp[sl + 1] - base) >> 5); \
    (void)base; (void)width;                                        \
    if (row < n) {
#define IR_ROWS_END \
  }                 \
  }
  if (P.project) {
    double part = 0.0;
    IR_ROWS_BEGIN part += static_cast<double>(P.b[row]);
    IR_ROWS_END
    part = block_sum(part, sh);
    if (threadIdx.x == 0) atomicAdd(P.red + 0, part);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  const double meanb = P.project ? P.red[0] / static_cast<double>(n) : 0.0;
  {
    double bb = 0.0;
    IR_ROWS_BEGIN
      const double bv = static_cast<double>(P.b[row]) - meanb;
      P.bh[row] = bv * P.sdinv[row];
      if (!P.warm) P.y[row] = 0.0;
      bb += bv * bv;
    IR_ROWS_END
    bb = block_sum(bb, sh);
    if (threadIdx.x == 0) atomicAdd(P.red + 1, bb);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  const double bb = P.red[1];
  const double tol2 = fmax(P.rtol * P.rtol * bb, P.atol * P.atol);
  int total = 0;
  double rho = 0.0;
  int outers = 0;
  for (int outer = 0; outer < P.max_outer; ++outer) {
    ++outers;
    const int so = 4 + (outer & 1);
    // true residual in FP64; inner start r = p = r64 (float), d = 0
    {
      double rh = 0.0, g = 0.0;
      if (blockIdx.x == 0 && threadIdx.x == 0) P.red[4 + ((outer + 1) & 1)] = 0.0;
      IR_ROWS_BEGIN
        double acc = 0.0;
        for (int k = 0; k < width; ++k) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          acc += P.v64[idx] * P.y[P.col[idx]];
        }
        const double r64 = P.bh[row] - acc;
        rh += P.diag[row] * r64 * r64;
        const float rf = static_cast<float>(r64);
        P.r[row] = rf;
        P.d[row] = 0.0f;
        g += static_cast<double>(rf) * rf;
      IR_ROWS_END
      rh = block_sum(rh, sh);
      if (threadIdx.x == 0) atomicAdd(P.red + so, rh);
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
    }
    rho = P.red[so];
    if (rho <= tol2 || total >= P.maxit) break;
    // s = A r, slot 0 <- (r,r), (r,s)
    {
      double g = 0.0, dl = 0.0;
      IR_ROWS_BEGIN
        float acc = 0.0f;
        for (int k = 0; k < width; ++k) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          acc += P.v32[idx] * P.r[P.col[idx]];
        }
        P.s[row] = acc;
        const double rv = P.r[row];
        g += rv * rv;
        dl += rv * static_cast<double>(acc);
      IR_ROWS_END
      g = block_sum(g, sh);
      dl = block_sum(dl, sh);
      if (threadIdx.x == 0) {
        atomicAdd(P.red + 8, g);
        atomicAdd(P.red + 9, dl);
      }
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
    }
    const double g0 = P.red[8];
    const double itol2 = P.inner_rtol * P.inner_rtol * g0;
    double gprev = 1.0, aprev = 1.0;
    for (int it = 0;; ++it) {
      const int sl = it % 3;
      const double gm = P.red[8 + 2 * sl], dl = P.red[9 + 2 * sl];
      if (gm <= itol2 || it >= P.inner_maxit || total >= P.maxit || !(gm > 0.0) || !(dl > 0.0)) break;
      if (blockIdx.x == 0 && threadIdx.x < 2) P.red[8 + 2 * ((it + 2) % 3) + threadIdx.x] = 0.0;
      double beta, alpha;
      if (it == 0) {
        beta = 0.0;
        alpha = gm / dl;
      } else {
        beta = gm / gprev;
        alpha = gm / (dl - beta * gm / aprev);
      }
      const float a = static_cast<float>(alpha), bt = static_cast<float>(beta);
      IR_ROWS_BEGIN
        const float rv = P.r[row], sv = P.s[row];
        const float pv = (it == 0) ? rv : rv + bt * P.p[row];
        const float qv = (it == 0) ? sv : sv + bt * P.q[row];
        P.p[row] = pv;
        P.q[row] = qv;
        P.d[row] += a * pv;
        P.r[row] = rv - a * qv;
      IR_ROWS_END
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
      double g2 = 0.0, d2 = 0.0;
      IR_ROWS_BEGIN
        float acc = 0.0f;
        for (int k = 0; k < width; ++k) {
          const int64_t idx = base + ((int64_t)k << 5) + lane;
          acc += P.v32[idx] * P.r[P.col[idx]];
        }
        P.s[row] = acc;
        const double rv = P.r[row];
        g2 += rv * rv;
        d2 += rv * static_cast<double>(acc);
      IR_ROWS_END
      g2 = block_sum(g2, sh);
      d2 = block_sum(d2, sh);
      if (threadIdx.x == 0) {
        const int ns = (it + 1) % 3;
        atomicAdd(P.red + 8 + 2 * ns, g2);
        atomicAdd(P.red + 9 + 2 * ns, d2);
      }
      gprev = gm;
      aprev = alpha;
      ++total;
      if (!grid_barrier(cnt, gen, nb, P.err)) return;
    }
    // y += d ; reset the inner slots for the next refinement step
    if (blockIdx.x == 0 && threadIdx.x < 6) P.red[8 + threadIdx.x] = 0.0;
    IR_ROWS_BEGIN P.y[row] += static_cast<double>(P.d[row]);
    IR_ROWS_END
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
  }
  double sx = 0.0;
  IR_ROWS_BEGIN sx += P.y[row] * P.sdinv[row];
  IR_ROWS_END
  double mx = 0.0;
  if (P.project) {
    sx = block_sum(sx, sh);
    if (threadIdx.x == 0) atomicAdd(P.red + 2, sx);
    if (!grid_barrier(cnt, gen, nb, P.err)) return;
    mx = P.red[2] / static_cast<double>(n);
  }
  IR_ROWS_BEGIN
    const double xv = P.y[row] * P.sdinv[row] - mx;
    P.x[row] = static_cast<float>(xv);
    P.y[row] = xv / P.sdinv[row];
  IR_ROWS_END
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *P.iters = total;
    *P.resid = bb > 0.0 ? sqrt(rho / bb) : 0.0;
    atomicAdd(P.iters_acc, (unsigned long long)total);
    atomicAdd(P.iters_acc + 1, (unsigned long long)outers);
    atomicAdd(P.iters_acc + 2, 1ull);
  }
#undef IR_ROWS_BEGIN
#undef IR_ROWS_END
}

template <class T>
void CgSystem<T>::setup(const HostSell& s, const std::vector<double>& vals_sell, const std::vector<double>& d) {
  n = s.nrows;
  P.upload(s);
  // scaled values: A_ij / sqrt(d_i d_j); rows are SELL rows, columns are system indices
  std::vector<T> v(vals_sell.size()), sd(n), dd(n);
  for (int64_t i = 0; i < n; ++i) {
    SPX_CHECK(d[i] > 0.0, "CG system has a non-positive diagonal");
    sd[i] = static_cast<T>(1.0 / std::sqrt(d[i]));
    dd[i] = static_cast<T>(d[i]);
  }
  for (int64_t sl = 0; sl < s.nslices; ++sl) {
    const int64_t w = (s.slice_ptr[sl + 1] - s.slice_ptr[sl]) / SELL_C;
    for (int64_t k = 0; k < w; ++k)
      for (int l = 0; l < SELL_C; ++l) {
        const int64_t idx = s.slice_ptr[sl] + k * SELL_C + l;
        const int64_t row = sl * SELL_C + l;
        if (row >= n) { v[idx] = T(0); continue; }
        const int64_t c = s.col[idx];
        v[idx] = static_cast<T>(vals_sell[idx] / std::sqrt(d[row] * d[c]));
      }
  }
  vals.upload(v);
  sdinv.upload(sd);
  diag.upload(dd);
  work.alloc(7 * static_cast<size_t>(n));
  if (sizeof(T) == sizeof(float)) {
    std::vector<double> v64(v.size()), sd64(n), d64(d.begin(), d.begin() + n);
    for (int64_t i = 0; i < n; ++i) sd64[i] = 1.0 / std::sqrt(d[i]);
    for (int64_t sl = 0; sl < s.nslices; ++sl) {
      const int64_t w = (s.slice_ptr[sl + 1] - s.slice_ptr[sl]) / SELL_C;
      for (int64_t k = 0; k < w; ++k)
        for (int l = 0; l < SELL_C; ++l) {
          const int64_t idx = s.slice_ptr[sl] + k * SELL_C + l;
          const int64_t row = sl * SELL_C + l;
          v64[idx] = (row < n) ? vals_sell[idx] / std::sqrt(d[row] * d[s.col[idx]]) : 0.0;
        }
    }
    vals64.upload(v64);
    sdinv64.upload(sd64);
    diag64.upload(d64);
    y64.alloc(n);
    y64.zero();
    bh64.alloc(n);
  }
  red.alloc(16);
  red.zero();
  iters_acc.alloc(4);
  iters_acc.zero();
  bar.alloc(2);
  err.alloc(1);
  iters.alloc(1);
  resid.alloc(1);
  int dev;
  SPX_CUDA(cudaGetDevice(&dev));
  int per_sm = 0;
  SPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg<T>, 256, 0));
  if (sizeof(T) == sizeof(float)) {
    int per_sm_ir = 0;
    SPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_ir, k_cg_ir, 256, 0));
    per_sm = std::min(per_sm, per_sm_ir);
  }
  SPX_CHECK(per_sm > 0, "CG kernel cannot be resident");
  const int64_t want = (s.nslices * 32 + 255) / 256;
  grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)per_sm * num_sms(dev))));
}

template <class T>
CgStats CgSystem<T>::solve(const T* b, T* x, double rtol, double atol, int maxit, bool warm, bool project,
                           cudaStream_t st, bool sync_stats) {
  CgParams<T> p;
  p.n = n;
  p.nslices = P.nslices;
  p.sp = P.slice_ptr.p;
  p.col = P.col.p;
  p.val = vals.p;
  p.sdinv = sdinv.p;
  p.diag = diag.p;
  p.b = b;
  p.x = x;
  T* W = work.p;
  p.r = W; p.w0 = W + n; p.w1 = W + 2 * n; p.p = W + 3 * n; p.s = W + 4 * n; p.z = W + 5 * n; p.y = W + 6 * n;
  p.red = red.p;
  p.bar = bar.p;
  p.err = err.p;
  p.iters = iters.p;
  p.resid = resid.p;
  p.iters_acc = iters_acc.p;
  p.rtol = rtol;
  p.atol = atol;
  p.maxit = maxit;
  p.warm = warm ? 1 : 0;
  p.project = project ? 1 : 0;
  SPX_CUDA(cudaMemsetAsync(red.p, 0, red.bytes(), st));
  SPX_CUDA(cudaMemsetAsync(bar.p, 0, bar.bytes(), st));
  SPX_CUDA(cudaMemsetAsync(err.p, 0, err.bytes(), st));
  if (sizeof(T) == sizeof(float)) {
    CgIrParams q;
    q.n = n; q.nslices = P.nslices; q.sp = P.slice_ptr.p; q.col = P.col.p;
    q.v32 = reinterpret_cast<const float*>(vals.p); q.v64 = vals64.p; q.sdinv = sdinv64.p; q.diag = diag64.p;
    q.b = reinterpret_cast<const float*>(b); q.x = reinterpret_cast<float*>(x);
    q.bh = bh64.p; q.y = y64.p;
    float* Wf = reinterpret_cast<float*>(work.p);
    q.r = Wf; q.p = Wf + n; q.q = Wf + 2 * n; q.s = Wf + 3 * n; q.d = Wf + 4 * n;
    q.red = red.p; q.bar = bar.p; q.err = err.p; q.iters = iters.p; q.resid = resid.p;
    q.iters_acc = iters_acc.p;
    q.rtol = rtol; q.atol = atol; q.inner_rtol = inner_rtol;
    q.maxit = maxit; q.max_outer = max_outer; q.inner_maxit = maxit; q.warm = warm ? 1 : 0;
    q.project = project ? 1 : 0;
    void* a2[] = {&q};
    SPX_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_cg_ir), dim3(grid), dim3(256), a2, 0, st));
  } else {
    void* args[] = {&p};
    SPX_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_cg<T>), dim3(grid), dim3(256), args, 0, st));
  }
  CgStats out;
  if (sync_stats) {
    int h_err = 0, h_it = 0;
    double h_res = 0.0;
    SPX_CUDA(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SPX_CUDA(cudaMemcpyAsync(&h_it, iters.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SPX_CUDA(cudaMemcpyAsync(&h_res, resid.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    SPX_CUDA(cudaStreamSynchronize(st));
    if (h_err) throw Error(ERR_TIMEOUT, "CG grid barrier timed out");
    out.iterations = h_it;
    out.rel_residual = h_res;
    out.converged = (h_res <= rtol || h_it < maxit) ? 1 : 0;
  }
  return out;
}

template struct CgSystem<double>;
template struct CgSystem<float>;

// ------------------------------------------------------------------ demag context
template <class T>
void DemagCtx<T>::create(const double* X, int64_t N_, const int32_t* tets, int64_t E_, double Ms_,
                         const DemagOptions& o, cudaStream_t s) {
  SPX_CUDA(cudaGetDevice(&device));
  N = N_;
  E = E_;
  Ms = Ms_;
  opt = o;
  bd.create(X, N, tets, E);
  Nb = bd.host.Nb;
  assemble_fem(X, N, tets, E, fem);
  const int64_t nnz = fem.rowptr[N];
  // full pattern
  std::vector<int32_t> all(N);
  for (int64_t i = 0; i < N; ++i) all[i] = static_cast<int32_t>(i);
  build_sell(fem.rowptr, fem.col, all, nullptr, hsell);
  P.upload(hsell, s);
  const int64_t L = hsell.slice_ptr.back();
  {
    std::vector<T> v;
    sell_values<T>(hsell, fem.Div.data(), 3, true, nnz, Ms, v);
    Div.upload(v, s);
    // G / vol_i : scale per CSR row
    std::vector<double> g = fem.G;
    for (int64_t i = 0; i < N; ++i)
      for (int64_t k = fem.rowptr[i]; k < fem.rowptr[i + 1]; ++k)
        for (int c = 0; c < 3; ++c) g[3 * k + c] /= fem.vol[i];
    sell_values<T>(hsell, g.data(), 3, true, nnz, 1.0, v);
    Gv.upload(v, s);
  }
  vol.upload(fem.vol, s);
  // u1 system: full stiffness
  {
    std::vector<double> a;
    sell_values<double>(hsell, fem.A.data(), 1, true, nnz, 1.0, a);
    std::vector<double> d(N);
    for (int64_t i = 0; i < N; ++i)
      for (int64_t k = fem.rowptr[i]; k < fem.rowptr[i + 1]; ++k)
        if (fem.col[k] == i) d[i] = fem.A[k];
    cg1.setup(hsell, a, d);
  }
  // interior / boundary split for u2
  std::vector<int32_t> bmap(N, -1), imap(N, -1), inter;
  for (int64_t k = 0; k < Nb; ++k) bmap[bd.host.bverts[k]] = static_cast<int32_t>(k);
  for (int64_t i = 0; i < N; ++i)
    if (bmap[i] < 0) {
      imap[i] = static_cast<int32_t>(inter.size());
      inter.push_back(static_cast<int32_t>(i));
    }
  NI = static_cast<int64_t>(inter.size());
  interior.upload(inter, s);
  bverts.upload(bd.host.bverts, s);
  if (NI > 0) {
    HostSell sII, sIB;
    build_sell(fem.rowptr, fem.col, inter, &imap, sII);
    build_sell(fem.rowptr, fem.col, inter, &bmap, sIB);
    std::vector<double> aII, aIB;
    sell_values<double>(sII, fem.A.data(), 1, true, nnz, 1.0, aII);
    std::vector<T> vIB;
    sell_values<T>(sIB, fem.A.data(), 1, true, nnz, 1.0, vIB);
    std::vector<double> d(NI);
    for (int64_t q = 0; q < NI; ++q) {
      const int64_t i = inter[q];
      for (int64_t k = fem.rowptr[i]; k < fem.rowptr[i + 1]; ++k)
        if (fem.col[k] == i) d[q] = fem.A[k];
    }
    cg2.setup(sII, aII, d);
    PIB.upload(sIB, s);
    AIB.upload(vIB, s);
  }
  // boundary operator
  if (opt.backend == 0) {
    SPX_CHECK(Nb * Nb * 8 <= (int64_t)64 * 1024 * 1024 * 1024, "dense boundary operator too large");
    Bdense.alloc(static_cast<size_t>(Nb * Nb));
    bd.dense_B(Bdense.p, s);
  } else {
    H.build(bd, opt.hcfg, s);
    H.pack(opt.prec, s);
  }
  b.alloc(N); u1.alloc(N); phi.alloc(N); gB.alloc(Nb); xb.alloc(Nb); yb.alloc(Nb);
  bI.alloc(std::max<int64_t>(NI, 1));
  xI.alloc(std::max<int64_t>(NI, 1));
  u1.zero(s);
  xI.zero(s);
  sum.alloc(4);
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class T>
void DemagCtx<T>::potential(const T* m, cudaStream_t s, bool sync_stats) {
  const int threads = 256;
  const unsigned gsl = grid_for(P.nslices * 32, threads);
  prof.mark(PC_DIV, s);
  k_div<T><<<gsl, threads, 0, s>>>(N, P.nslices, P.slice_ptr.p, P.col.p, Div.p, P.len, m, b.p, nullptr);
  SPX_LAUNCH_CHECK();
  prof.mark(PC_DIV, s);
  prof.launches[PC_DIV] += 1;
  prof.mark(PC_CG1, s);
  last1 = cg1.solve(b.p, u1.p, opt.rtol_u1, opt.atol, opt.maxit_u1, opt.warm_start != 0, true, s, sync_stats);
  prof.mark(PC_CG1, s);
  prof.launches[PC_CG1] += 1;
  prof.mark(PC_BND, s);
  if (opt.backend == 0) {
    k_gather_idx<T><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, bverts.p, u1.p, xb.p);
    SPX_LAUNCH_CHECK();
    k_dense_gemv<T><<<grid_for(Nb * 32, 256), 256, 0, s>>>(Nb, Bdense.p, xb.p, bverts.p, u1.p, phi.p, gB.p);
    SPX_LAUNCH_CHECK();
    prof.launches[PC_BND] += 2;
  } else {
    H.apply_gather<T>(u1.p, bverts.p, phi.p, u1.p, gB.p, s);
    prof.launches[PC_BND] += H.n_far > 0 ? 3 : 2;
  }
  prof.mark(PC_BND, s);
  if (NI > 0) {
    prof.mark(PC_U2RHS, s);
    k_u2rhs<T><<<grid_for(PIB.nslices * 32, threads), threads, 0, s>>>(NI, PIB.nslices, PIB.slice_ptr.p,
                                                                         PIB.col.p, AIB.p, gB.p, bI.p);
    SPX_LAUNCH_CHECK();
    prof.mark(PC_U2RHS, s);
    prof.launches[PC_U2RHS] += 1;
    // ||b|| of the reference's full u2 system includes the boundary rows (b[bnd] = g);
    // the interior test is slightly stricter, which only tightens the solve.
    prof.mark(PC_CG2, s);
    last2 = cg2.solve(bI.p, xI.p, opt.rtol_u2, opt.atol, opt.maxit_u2, opt.warm_start != 0, false, s, sync_stats);
    prof.mark(PC_CG2, s);
    prof.launches[PC_CG2] += 1;
    prof.mark(PC_PHI, s);
    k_phi_interior<T><<<grid_for(NI, 256), 256, 0, s>>>(NI, interior.p, u1.p, xI.p, phi.p);
    SPX_LAUNCH_CHECK();
    prof.mark(PC_PHI, s);
    prof.launches[PC_PHI] += 1;
  }
  launches += 4 + (opt.backend == 0 ? 2 : (H.n_far > 0 ? 3 : 2)) + (NI > 0 ? 3 : 0) - 1;
  ++applies;
}

template <class T>
void DemagCtx<T>::field(T* Hout, cudaStream_t s) {
  k_grad<T><<<grid_for(P.nslices * 32, 256), 256, 0, s>>>(N, P.nslices, P.slice_ptr.p, P.col.p, Gv.p, P.len,
                                                           phi.p, Hout);
  SPX_LAUNCH_CHECK();
}

template <class T>
int64_t DemagCtx<T>::device_bytes() const {
  int64_t tot = 0;
  tot += P.slice_ptr.bytes() + P.col.bytes() + Div.bytes() + Gv.bytes() + vol.bytes();
  tot += cg1.vals.bytes() + cg1.work.bytes() + cg1.P.col.bytes() + cg2.vals.bytes() + cg2.work.bytes() +
         cg2.P.col.bytes();
  tot += AIB.bytes() + PIB.col.bytes() + Bdense.bytes();
  tot += H.device_bytes();
  return tot;
}

template struct DemagCtx<double>;
template struct DemagCtx<float>;

// explicit instantiations used by llg.cu
template __global__ void k_gather_idx<double>(int64_t, const int32_t*, const double*, double*);
template __global__ void k_gather_idx<float>(int64_t, const int32_t*, const float*, float*);

}  // namespace spx
