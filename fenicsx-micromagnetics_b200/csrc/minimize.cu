// Device side of the LaBonte / Barzilai-Borwein energy minimiser
// (gpu/solvers/Minimizer_GPU.py:171-845; the step-length and acceptance logic runs on the
// host, spinfemx_b200/minimizer.py).  One call per trial state:
//   m_t = Cayley(m_old, d_old, alpha)          (_CAYLEY_KERNEL, :46-74)
//   H   = H_eff(m_t)                            (demag included; the stage kernel in mode 0)
//   d_t = H - (m_t . H) m_t                      (_PROJDIR_KERNEL, :77-88)
//   E   = mu0 Ms 1e-27 sum_i V_i m_i . (-H_i / 2 - H0_i / 2)
//         (= -1/2 mu0 Ms sum V m . H_self - mu0 Ms sum V m . H0, compute_Energy_terms_minimize_gpu,
//          gpu/solvers/llg_module_GPU.py:1079-1222, without the anisotropy offset)
//   max |d_t|, and the Barzilai-Borwein products s.y, s.s, y.y with s = m_t - m_old,
//   y = g_t - g_old = d_old - d_t
// the last three lines in one pass over the nodes, one host read of five numbers.
#include <algorithm>
#include <cmath>

#include "llg.cuh"

namespace spx {

namespace {

constexpr int MIN_GRID = 296;  // 2 CTAs per SM

template <class TV>
__global__ void k_cayley(int64_t n, const TV* __restrict__ m, const TV* __restrict__ d, double alpha,
                         TV* __restrict__ y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double mx = m[3 * i], my = m[3 * i + 1], mz = m[3 * i + 2];
  const double dx = d[3 * i], dy = d[3 * i + 1], dz = d[3 * i + 2];
  const double cx = 0.5 * alpha * (my * dz - mz * dy);
  const double cy = 0.5 * alpha * (mz * dx - mx * dz);
  const double cz = 0.5 * alpha * (mx * dy - my * dx);
  const double bx = mx + cy * mz - cz * my, by = my + cz * mx - cx * mz, bz = mz + cx * my - cy * mx;
  const double cbx = cy * bz - cz * by, cby = cz * bx - cx * bz, cbz = cx * by - cy * bx;
  const double cdb = cx * bx + cy * by + cz * bz, c2 = cx * cx + cy * cy + cz * cz;
  const double inv = 1.0 / (1.0 + c2);
  y[3 * i] = static_cast<TV>((bx + cbx + cx * cdb) * inv);
  y[3 * i + 1] = static_cast<TV>((by + cby + cy * cdb) * inv);
  y[3 * i + 2] = static_cast<TV>((bz + cbz + cz * cdb) * inv);
}

template <class TV>
__global__ void k_normalize(int64_t n, TV* __restrict__ m) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = m[3 * i], y = m[3 * i + 1], z = m[3 * i + 2];
  const double r = std::max(std::sqrt(x * x + y * y + z * z), 1e-30);
  m[3 * i] = static_cast<TV>(x / r);
  m[3 * i + 1] = static_cast<TV>(y / r);
  m[3 * i + 2] = static_cast<TV>(z / r);
}

// per-CTA partials: [0] energy sum, [1] max |d|, [2] s.y, [3] s.s, [4] y.y
template <class TV>
__global__ void __launch_bounds__(256) k_min_reduce(int64_t n, const TV* __restrict__ m, const TV* __restrict__ H,
                                                    const TV* __restrict__ H0n, double h0x, double h0y, double h0z,
                                                    const double* __restrict__ vol, const TV* __restrict__ m_old,
                                                    const TV* __restrict__ d_old, TV* __restrict__ d,
                                                    double* __restrict__ part) {
  __shared__ double sh[32];
  double e = 0.0, dmax = 0.0, sty = 0.0, sts = 0.0, yty = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double mx = m[3 * i], my = m[3 * i + 1], mz = m[3 * i + 2];
    const double hx = H[3 * i], hy = H[3 * i + 1], hz = H[3 * i + 2];
    const double ax = H0n ? static_cast<double>(H0n[3 * i]) : h0x;
    const double ay = H0n ? static_cast<double>(H0n[3 * i + 1]) : h0y;
    const double az = H0n ? static_cast<double>(H0n[3 * i + 2]) : h0z;
    e += vol[i] * (mx * (-0.5 * hx - 0.5 * ax) + my * (-0.5 * hy - 0.5 * ay) + mz * (-0.5 * hz - 0.5 * az));
    const double mh = mx * hx + my * hy + mz * hz;
    const double dx = hx - mh * mx, dy = hy - mh * my, dz = hz - mh * mz;
    d[3 * i] = static_cast<TV>(dx);
    d[3 * i + 1] = static_cast<TV>(dy);
    d[3 * i + 2] = static_cast<TV>(dz);
    dmax = fmax(dmax, std::sqrt(dx * dx + dy * dy + dz * dz));
    if (m_old) {
      const double sx = mx - m_old[3 * i], sy = my - m_old[3 * i + 1], sz = mz - m_old[3 * i + 2];
      const double yx = d_old[3 * i] - dx, yy = d_old[3 * i + 1] - dy, yz = d_old[3 * i + 2] - dz;
      sty += sx * yx + sy * yy + sz * yz;
      sts += sx * sx + sy * sy + sz * sz;
      yty += yx * yx + yy * yy + yz * yz;
    }
  }
  const double vals[4] = {e, sty, sts, yty};
  const int slot[4] = {0, 2, 3, 4};
  for (int q = 0; q < 4; ++q) {
    const double t = block_sum(vals[q], sh);
    if (threadIdx.x == 0) part[5 * blockIdx.x + slot[q]] = t;
  }
  double v = dmax;  // block max
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mxv = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) mxv = fmax(mxv, sh[w]);
    part[5 * blockIdx.x + 1] = mxv;
  }
}

__global__ void k_min_final(int nparts, const double* __restrict__ part, double escale, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int b = 0; b < nparts; ++b) {
    s[0] += part[5 * b];
    s[1] = fmax(s[1], part[5 * b + 1]);
    s[2] += part[5 * b + 2];
    s[3] += part[5 * b + 3];
    s[4] += part[5 * b + 4];
  }
  out[0] = s[0] * escale;
  for (int q = 1; q < 5; ++q) out[q] = s[q];
}

}  // namespace

template <class TV, class TM>
void LLGCtx<TV, TM>::min_eval(TV* mm, const TV* m_old, const TV* d_old, TV* d, bool normalize, double out5[5],
                              cudaStream_t s) {
  const HostFem& fem = demag ? demag->fem : own_fem;
  if (!minvol.n) minvol.upload(fem.vol, s);
  if (!minpart.n) minpart.alloc(5 * MIN_GRID + 5);
  if (!minH.n) minH.alloc(3 * N);
  if (normalize) {
    k_normalize<TV><<<grid_for(N, 256), 256, 0, s>>>(N, mm);
    SPX_LAUNCH_CHECK();
  }
  heff(mm, minH.p, true, s);
  k_min_reduce<TV><<<MIN_GRID, 256, 0, s>>>(N, mm, minH.p, H0.n ? H0.p : nullptr, h0[0], h0[1], h0[2], minvol.p,
                                            m_old, d_old, d, minpart.p);
  SPX_LAUNCH_CHECK();
  const double mu0 = 4e-7 * 3.141592653589793;
  k_min_final<<<1, 32, 0, s>>>(MIN_GRID, minpart.p, mu0 * prm.Ms * 1e-27, minpart.p + 5 * MIN_GRID);
  SPX_LAUNCH_CHECK();
  SPX_CUDA(cudaMemcpyAsync(out5, minpart.p + 5 * MIN_GRID, 5 * sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class TV, class TM>
void LLGCtx<TV, TM>::min_trial(const TV* m_old, const TV* d_old, double alpha, TV* m_t, TV* d_t, double out5[5],
                               cudaStream_t s) {
  k_cayley<TV><<<grid_for(N, 256), 256, 0, s>>>(N, m_old, d_old, alpha, m_t);
  SPX_LAUNCH_CHECK();
  min_eval(m_t, m_old, d_old, d_t, false, out5, s);
}

#define SPX_MIN_INST(TV, TM)                                                                                    \
  template void LLGCtx<TV, TM>::min_eval(TV*, const TV*, const TV*, TV*, bool, double*, cudaStream_t);          \
  template void LLGCtx<TV, TM>::min_trial(const TV*, const TV*, double, TV*, TV*, double*, cudaStream_t);
SPX_MIN_INST(double, double)
SPX_MIN_INST(float, float)
SPX_MIN_INST(double, float)
#undef SPX_MIN_INST

}  // namespace spx
