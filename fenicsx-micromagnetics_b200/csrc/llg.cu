// Effective field, LLG right-hand side, Jacobian-vector product, 3x3 block
// preconditioner and the fixed-step RK4 driver on the device.
//
// References (gpu/solvers/llg_module_GPU.py):
//   _LLG_RHS_KERNEL :100-122     rhs = pref (p m x H + alpha m x (m x H)) + Stab (1-|m|^2) m
//   _JAC_VEC_KERNEL :125-164     J v (H_jac excludes demag)
//   _PC_BUILD_INV3_KERNEL :167-293, _PC_APPLY_KERNEL :296-308
//   EffectiveField.compute_H_eff_vec :972-1006 = K_lin m + local terms + demag + H0
//   exchange K = diag(-2A/(mu0 Ms V_i) 1e18) * stiffness (gpu/fields/Exchange_GPU.py:53-68)
//   interfacial DMI (gpu/fields/DMI_Interfacial_GPU.py:140-172), nodal uniaxial
//   anisotropy H = 2Ku/(mu0 Ms) (m.n) n (gpu/fields/Anisotropy_GPU.py:317-342)
//
// k_stage fuses, per node and in one pass over the shared SELL pattern: the exchange
// (and DMI) SpMV on m, the demag gradient G phi / V_i, anisotropy, Zeeman, the LLG
// RHS and the RK4 stage combination.  The only other per-stage work is the demag
// potential (Div SpMV, two CG solves, boundary operator).
#include <algorithm>
#include <cmath>

#include "llg.cuh"

namespace spx {

template <class T>
struct StageArgs {
  int64_t n, nslices;
  const int64_t* sp;
  const int32_t* col;
  int64_t L;
  const T* Kex;   // [L] exchange, row-scaled
  const T* Kd;    // [9L] DMI blocks, row-scaled (or null)
  const T* Gv;    // [3L] G / vol (or null: no demag)
  const T* phi;   // potential (or null)
  const T* ani_n; // [3n] unit axes (or null)
  const T* ani_p; // [n] per-node prefactor 2Ku/(mu0 Ms) (or null)
  T ani_p0;       // scalar prefactor when ani_p == null
  const T* H0;    // [3n] (or null)
  T h0x, h0y, h0z;
  const T* m;     // stage input (AoS)
  T* out;         // mode 0: H ; mode 1: rhs ; mode 2: next stage m
  T* mn;          // RK state (mode 2)
  T* acc;         // RK accumulator (mode 2)
  T pref, alpha, precess, stab;
  T c_next, w_acc, dt6;
  int mode, stage;
};

template <class T, bool DMI, bool DEMAG, bool ANI>
__global__ void __launch_bounds__(256) k_stage(StageArgs<T> a) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t sl = gw; sl < a.nslices; sl += nw) {
    const int64_t i = sl * 32 + lane;
    if (i >= a.n) continue;
    const int64_t base = a.sp[sl];
    const int width = static_cast<int>((a.sp[sl + 1] - base) >> 5);
    T hx = 0, hy = 0, hz = 0;
    for (int k = 0; k < width; ++k) {
      const int64_t idx = base + ((int64_t)k << 5) + lane;
      const int64_t j = a.col[idx];
      const T mx = a.m[3 * j], my = a.m[3 * j + 1], mz = a.m[3 * j + 2];
      const T e = a.Kex[idx];
      hx += e * mx;
      hy += e * my;
      hz += e * mz;
      if (DMI) {
        const T* K = a.Kd + idx;
        const int64_t L = a.L;
        hx += K[0] * mx + K[L] * my + K[2 * L] * mz;
        hy += K[3 * L] * mx + K[4 * L] * my + K[5 * L] * mz;
        hz += K[6 * L] * mx + K[7 * L] * my + K[8 * L] * mz;
      }
      if (DEMAG) {
        const T p = a.phi[j];
        hx += a.Gv[idx] * p;
        hy += a.Gv[a.L + idx] * p;
        hz += a.Gv[2 * a.L + idx] * p;
      }
    }
    const T mx = a.m[3 * i], my = a.m[3 * i + 1], mz = a.m[3 * i + 2];
    if (ANI) {
      const T nx = a.ani_n[3 * i], ny = a.ani_n[3 * i + 1], nz = a.ani_n[3 * i + 2];
      const T c = (a.ani_p ? a.ani_p[i] : a.ani_p0) * (mx * nx + my * ny + mz * nz);
      hx += c * nx;
      hy += c * ny;
      hz += c * nz;
    }
    if (a.H0) {
      hx += a.H0[3 * i];
      hy += a.H0[3 * i + 1];
      hz += a.H0[3 * i + 2];
    } else {
      hx += a.h0x;
      hy += a.h0y;
      hz += a.h0z;
    }
    if (a.mode == 0) {
      a.out[3 * i] = hx;
      a.out[3 * i + 1] = hy;
      a.out[3 * i + 2] = hz;
      continue;
    }
    const T cx = my * hz - mz * hy, cy = mz * hx - mx * hz, cz = mx * hy - my * hx;
    const T ccx = my * cz - mz * cy, ccy = mz * cx - mx * cz, ccz = mx * cy - my * cx;
    const T s = a.stab * (T(1) - (mx * mx + my * my + mz * mz));
    const T rx = a.pref * (a.precess * cx + a.alpha * ccx) + s * mx;
    const T ry = a.pref * (a.precess * cy + a.alpha * ccy) + s * my;
    const T rz = a.pref * (a.precess * cz + a.alpha * ccz) + s * mz;
    if (a.mode == 1) {
      a.out[3 * i] = rx;
      a.out[3 * i + 1] = ry;
      a.out[3 * i + 2] = rz;
      continue;
    }
    // RK4 stage update
    T* A = a.acc + 3 * i;
    T* M = a.mn + 3 * i;
    if (a.stage == 0) {
      A[0] = rx; A[1] = ry; A[2] = rz;
    } else if (a.stage < 3) {
      A[0] += a.w_acc * rx; A[1] += a.w_acc * ry; A[2] += a.w_acc * rz;
    }
    if (a.stage < 3) {
      a.out[3 * i] = M[0] + a.c_next * rx;
      a.out[3 * i + 1] = M[1] + a.c_next * ry;
      a.out[3 * i + 2] = M[2] + a.c_next * rz;
    } else {
      M[0] += a.dt6 * (A[0] + rx);
      M[1] += a.dt6 * (A[1] + ry);
      M[2] += a.dt6 * (A[2] + rz);
    }
  }
}

// J v with the linear field H_v = K_lin v (+ anisotropy of v)
template <class T, bool DMI, bool ANI>
__global__ void __launch_bounds__(256) k_jv(StageArgs<T> a, const T* __restrict__ Ms, const T* __restrict__ Hm,
                                            const T* __restrict__ v, T* __restrict__ out, T gamma) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t sl = gw; sl < a.nslices; sl += nw) {
    const int64_t i = sl * 32 + lane;
    if (i >= a.n) continue;
    const int64_t base = a.sp[sl];
    const int width = static_cast<int>((a.sp[sl + 1] - base) >> 5);
    T hvx = 0, hvy = 0, hvz = 0;
    for (int k = 0; k < width; ++k) {
      const int64_t idx = base + ((int64_t)k << 5) + lane;
      const int64_t j = a.col[idx];
      const T x = v[3 * j], y = v[3 * j + 1], z = v[3 * j + 2];
      const T e = a.Kex[idx];
      hvx += e * x; hvy += e * y; hvz += e * z;
      if (DMI) {
        const T* K = a.Kd + idx;
        const int64_t L = a.L;
        hvx += K[0] * x + K[L] * y + K[2 * L] * z;
        hvy += K[3 * L] * x + K[4 * L] * y + K[5 * L] * z;
        hvz += K[6 * L] * x + K[7 * L] * y + K[8 * L] * z;
      }
    }
    const T vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
    if (ANI) {
      const T nx = a.ani_n[3 * i], ny = a.ani_n[3 * i + 1], nz = a.ani_n[3 * i + 2];
      const T c = (a.ani_p ? a.ani_p[i] : a.ani_p0) * (vx * nx + vy * ny + vz * nz);
      hvx += c * nx; hvy += c * ny; hvz += c * nz;
    }
    const T mx = Ms[3 * i], my = Ms[3 * i + 1], mz = Ms[3 * i + 2];
    const T hx = Hm[3 * i], hy = Hm[3 * i + 1], hz = Hm[3 * i + 2];
    const T cvx = vy * hz - vz * hy, cvy = vz * hx - vx * hz, cvz = vx * hy - vy * hx;
    const T cmx = my * hvz - mz * hvy, cmy = mz * hvx - mx * hvz, cmz = mx * hvy - my * hvx;
    const T mdHm = mx * hx + my * hy + mz * hz;
    const T mdHv = mx * hvx + my * hvy + mz * hvz;
    const T vdHm = vx * hx + vy * hy + vz * hz;
    const T mdv = mx * vx + my * vy + mz * vz;
    const T mdmm = mx * mx + my * my + mz * mz;
    const T common = vdHm + mdHv;
    const T dampx = vx * mdHm - T(2) * hx * mdv + mx * common - hvx * mdmm;
    const T dampy = vy * mdHm - T(2) * hy * mdv + my * common - hvy * mdmm;
    const T dampz = vz * mdHm - T(2) * hz * mdv + mz * common - hvz * mdmm;
    const T coef = -gamma / (T(1) + a.alpha * a.alpha);
    const T sc = a.stab * (T(1) - mdmm);
    out[3 * i] = coef * (a.precess * (cvx + cmx) + a.alpha * dampx) + sc * vx - T(2) * a.stab * mx * mdv;
    out[3 * i + 1] = coef * (a.precess * (cvy + cmy) + a.alpha * dampy) + sc * vy - T(2) * a.stab * my * mdv;
    out[3 * i + 2] = coef * (a.precess * (cvz + cmz) + a.alpha * dampz) + sc * vz - T(2) * a.stab * mz * mdv;
  }
}

template <class T>
__global__ void k_pc_build(int64_t n, const T* __restrict__ M, const T* __restrict__ H, const T* __restrict__ D,
                           int include_stab, int use_abs_kappa, double shift, double eps_reg, double det_eps,
                           double c1, double c2, double Stab, T* __restrict__ inv) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double mx = M[3 * i], my = M[3 * i + 1], mz = M[3 * i + 2];
  const double hx = H[3 * i], hy = H[3 * i + 1], hz = H[3 * i + 2];
  const double dex = D[3 * i], dey = D[3 * i + 1], dez = D[3 * i + 2];
  const double kappa = use_abs_kappa ? (fabs(dex) + fabs(dey) + fabs(dez)) / 3.0 : (dex + dey + dez) / 3.0;
  const double mdH = mx * hx + my * hy + mz * hz;
  const double mdm = mx * mx + my * my + mz * mz;
  double J[3][3];
  J[0][0] = c2 * ((mdH - hx * mx) + kappa * (mx * mx - mdm));
  J[1][1] = c2 * ((mdH - hy * my) + kappa * (my * my - mdm));
  J[2][2] = c2 * ((mdH - hz * mz) + kappa * (mz * mz - mdm));
  J[0][1] = -c1 * (-hz - kappa * (-mz)) + c2 * ((mx * hy - 2.0 * hx * my) + kappa * (mx * my));
  J[0][2] = -c1 * (hy - kappa * my) + c2 * ((mx * hz - 2.0 * hx * mz) + kappa * (mx * mz));
  J[1][0] = -c1 * (hz - kappa * mz) + c2 * ((my * hx - 2.0 * hy * mx) + kappa * (my * mx));
  J[1][2] = -c1 * (-hx - kappa * (-mx)) + c2 * ((my * hz - 2.0 * hy * mz) + kappa * (my * mz));
  J[2][0] = -c1 * (-hy - kappa * (-my)) + c2 * ((mz * hx - 2.0 * hz * mx) + kappa * (mz * mx));
  J[2][1] = -c1 * (hx - kappa * mx) + c2 * ((mz * hy - 2.0 * hz * my) + kappa * (mz * my));
  if (include_stab) {
    const double s0 = 1.0 - mdm;
    const double m3[3] = {mx, my, mz};
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) J[r][c] += Stab * ((r == c ? s0 : 0.0) - 2.0 * m3[r] * m3[c]);
  }
  const double s = shift + eps_reg;
  double A[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[r][c] = (r == c ? s : 0.0) - J[r][c];
  double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
               A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (fabs(det) < det_eps) det += ((det + det_eps) > 0.0 ? 1.0 : -1.0) * det_eps;
  const double id = 1.0 / det;
  T* o = inv + 9 * i;
  o[0] = static_cast<T>((A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id);
  o[1] = static_cast<T>(-(A[0][1] * A[2][2] - A[0][2] * A[2][1]) * id);
  o[2] = static_cast<T>((A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id);
  o[3] = static_cast<T>(-(A[1][0] * A[2][2] - A[1][2] * A[2][0]) * id);
  o[4] = static_cast<T>((A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id);
  o[5] = static_cast<T>(-(A[0][0] * A[1][2] - A[0][2] * A[1][0]) * id);
  o[6] = static_cast<T>((A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id);
  o[7] = static_cast<T>(-(A[0][0] * A[2][1] - A[0][1] * A[2][0]) * id);
  o[8] = static_cast<T>((A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id);
}

template <class T>
__global__ void k_pc_apply(int64_t n, const T* __restrict__ inv, const T* __restrict__ x, T* __restrict__ y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T* o = inv + 9 * i;
  const T a = x[3 * i], b = x[3 * i + 1], c = x[3 * i + 2];
  y[3 * i] = o[0] * a + o[1] * b + o[2] * c;
  y[3 * i + 1] = o[3] * a + o[4] * b + o[5] * c;
  y[3 * i + 2] = o[6] * a + o[7] * b + o[8] * c;
}

// sum_i w_i m_i . H_i  (w = nodal volume)
template <class T>
__global__ void k_mdoth(int64_t n, const double* __restrict__ w, const T* __restrict__ m, const T* __restrict__ H,
                        double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += w[i] * (static_cast<double>(m[3 * i]) * H[3 * i] + static_cast<double>(m[3 * i + 1]) * H[3 * i + 1] +
                 static_cast<double>(m[3 * i + 2]) * H[3 * i + 2]);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) atomicAdd(out, s);
}

template <class A, class B>
__global__ void k_convert(int64_t n, const A* __restrict__ src, B* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = static_cast<B>(src[i]);
}

template <class A, class B>
void convert(int64_t n, const A* src, B* dst, cudaStream_t s) {
  if (n <= 0) return;
  k_convert<A, B><<<grid_for(n, 256), 256, 0, s>>>(n, src, dst);
  SPX_LAUNCH_CHECK();
}
template void convert<double, float>(int64_t, const double*, float*, cudaStream_t);
template void convert<float, double>(int64_t, const float*, double*, cudaStream_t);
template void convert<double, double>(int64_t, const double*, double*, cudaStream_t);

// ------------------------------------------------------------------ LLG context
template <class T>
void LLGCtx<T>::create(DemagCtx<T>* dm, const double* X, int64_t N_, const int32_t* tets, int64_t E,
                       const LLGParams& p, cudaStream_t s) {
  SPX_CUDA(cudaGetDevice(&device));
  prm = p;
  N = N_;
  demag = dm;
  const double mu0 = 4e-7 * 3.141592653589793;
  pref = -p.gamma / (1.0 + p.alpha * p.alpha);
  stab = p.Ms * p.gamma / (1.0 + p.alpha * p.alpha) * 0.5;
  c1 = p.gamma * p.do_precess / (1.0 + p.alpha * p.alpha);
  c2 = p.gamma * p.alpha / (1.0 + p.alpha * p.alpha);
  const HostFem* fem = nullptr;
  const HostSell* hs = nullptr;
  if (dm) {
    SPX_CHECK(dm->N == N, "demag context and LLG mesh differ");
    fem = &dm->fem;
    hs = &dm->hsell;
  } else {
    assemble_fem(X, N, tets, E, own_fem);
    std::vector<int32_t> all(N);
    for (int64_t i = 0; i < N; ++i) all[i] = static_cast<int32_t>(i);
    build_sell(own_fem.rowptr, own_fem.col, all, nullptr, own_sell);
    fem = &own_fem;
    hs = &own_sell;
  }
  P.upload(*hs, s);
  const int64_t nnz = fem->rowptr[N];
  // exchange: row-scaled stiffness (Exchange_GPU.py:62)
  std::vector<double> kex(nnz, 0.0), diag(3 * N, 0.0);
  for (int64_t i = 0; i < N; ++i) {
    const double sc = (p.Aex != 0.0) ? -2.0 * p.Aex / (mu0 * p.Ms) / fem->vol[i] / 1e-18 : 0.0;
    for (int64_t k = fem->rowptr[i]; k < fem->rowptr[i + 1]; ++k) {
      kex[k] = sc * fem->A[k];
      if (fem->col[k] == i)
        for (int c = 0; c < 3; ++c) diag[3 * i + c] += kex[k];
    }
  }
  std::vector<T> v;
  sell_values<T>(*hs, kex.data(), 1, true, nnz, 1.0, v);
  Kex.upload(v, s);
  has_dmi = (p.D_int != 0.0);
  if (has_dmi) {
    SPX_CHECK(p.n_int != nullptr, "interfacial DMI needs the interface normal field");
    HostBoundary bhost;
    const HostBoundary* bh = nullptr;
    if (dm) bh = &dm->bd.host;
    else { build_boundary(X, N, tets, E, bhost); bh = &bhost; }
    std::vector<double> b9;
    assemble_dmi_interfacial(X, tets, E, *fem, *bh, p.n_int, b9);
    for (int64_t i = 0; i < N; ++i) {
      const double sc = -2.0 * p.D_int / (mu0 * p.Ms) / 1e-9 / fem->vol[i];
      for (int64_t k = fem->rowptr[i]; k < fem->rowptr[i + 1]; ++k) {
        for (int q = 0; q < 9; ++q) b9[9 * k + q] *= sc;
        if (fem->col[k] == i)
          for (int c = 0; c < 3; ++c) diag[3 * i + c] += b9[9 * k + 4 * c];
      }
    }
    sell_values<T>(*hs, b9.data(), 9, true, nnz, 1.0, v);
    Kd.upload(v, s);
  }
  // anisotropy (per-node prefactor allowed)
  has_ani = false;
  if (p.n_ani && (p.Ku != 0.0 || p.Ku_nodes)) {
    has_ani = true;
    std::vector<T> nn(3 * N);
    for (int64_t i = 0; i < N; ++i) {
      double a = p.n_ani[3 * i], b = p.n_ani[3 * i + 1], c = p.n_ani[3 * i + 2];
      const double r = std::max(std::sqrt(a * a + b * b + c * c), 1e-300);
      nn[3 * i] = static_cast<T>(a / r);
      nn[3 * i + 1] = static_cast<T>(b / r);
      nn[3 * i + 2] = static_cast<T>(c / r);
      const double pr = 2.0 * (p.Ku_nodes ? p.Ku_nodes[i] : p.Ku) / (mu0 * p.Ms);
      for (int q = 0; q < 3; ++q) diag[3 * i + q] += pr * (a / r) * (a / r) * (q == 0) + pr * (b / r) * (b / r) * (q == 1) +
                                                     pr * (c / r) * (c / r) * (q == 2);
    }
    ani_n.upload(nn, s);
    ani_p0 = 2.0 * p.Ku / (mu0 * p.Ms);
    if (p.Ku_nodes) {
      std::vector<T> pp(N);
      for (int64_t i = 0; i < N; ++i) pp[i] = static_cast<T>(2.0 * p.Ku_nodes[i] / (mu0 * p.Ms));
      ani_p.upload(pp, s);
    }
  }
  std::vector<T> dg(diag.begin(), diag.end());
  diagK.upload(dg, s);
  if (p.H0_nodes) {
    std::vector<T> h(p.H0_nodes, p.H0_nodes + 3 * N);
    H0.upload(h, s);
  }
  h0[0] = p.H0_uniform[0];
  h0[1] = p.H0_uniform[1];
  h0[2] = p.H0_uniform[2];
  use_demag = (dm != nullptr) && p.use_demag;
  m.alloc(3 * N); ms0.alloc(3 * N); ms1.alloc(3 * N); acc.alloc(3 * N); tmp.alloc(3 * N); tmp2.alloc(3 * N);
  Mstate.alloc(3 * N); Hm.alloc(3 * N); pcinv.alloc(9 * N);
  red.alloc(2);
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class T>
StageArgs<T> LLGCtx<T>::args(const T* min, T* out, int mode, bool with_demag) const {
  StageArgs<T> a{};
  a.n = N;
  a.nslices = P.nslices;
  a.sp = P.slice_ptr.p;
  a.col = P.col.p;
  a.L = P.len;
  a.Kex = Kex.p;
  a.Kd = has_dmi ? Kd.p : nullptr;
  a.Gv = with_demag ? demag->Gv.p : nullptr;
  a.phi = with_demag ? demag->phi.p : nullptr;
  a.ani_n = has_ani ? ani_n.p : nullptr;
  a.ani_p = (has_ani && ani_p.n) ? ani_p.p : nullptr;
  a.ani_p0 = static_cast<T>(ani_p0);
  a.H0 = H0.n ? H0.p : nullptr;
  a.h0x = static_cast<T>(h0[0]);
  a.h0y = static_cast<T>(h0[1]);
  a.h0z = static_cast<T>(h0[2]);
  a.m = min;
  a.out = out;
  a.pref = static_cast<T>(pref);
  a.alpha = static_cast<T>(prm.alpha);
  a.precess = static_cast<T>(prm.do_precess);
  a.stab = static_cast<T>(stab);
  a.mode = mode;
  return a;
}

template <class T>
void LLGCtx<T>::launch_stage(const StageArgs<T>& a, bool with_demag, cudaStream_t s) const {
  const unsigned g = grid_for(a.nslices * 32, 256);
  const bool d = has_dmi, an = has_ani;
#define SPX_STAGE(DM, DE, AN) k_stage<T, DM, DE, AN><<<g, 256, 0, s>>>(a)
  if (d && with_demag && an) SPX_STAGE(true, true, true);
  else if (d && with_demag) SPX_STAGE(true, true, false);
  else if (d && an) SPX_STAGE(true, false, true);
  else if (d) SPX_STAGE(true, false, false);
  else if (with_demag && an) SPX_STAGE(false, true, true);
  else if (with_demag) SPX_STAGE(false, true, false);
  else if (an) SPX_STAGE(false, false, true);
  else SPX_STAGE(false, false, false);
#undef SPX_STAGE
  SPX_LAUNCH_CHECK();
  ++launches;
}

template <class T>
void LLGCtx<T>::heff(const T* min, T* Hout, bool with_demag, cudaStream_t s) {
  const bool dm = with_demag && use_demag;
  if (dm) demag->potential(min, s, true);
  launch_stage(args(min, Hout, 0, dm), dm, s);
}

template <class T>
void LLGCtx<T>::rhs(const T* min, T* out, cudaStream_t s) {
  if (use_demag) demag->potential(min, s, true);
  launch_stage(args(min, out, 1, use_demag), use_demag, s);
  ++rhs_evals;
}

template <class T>
void LLGCtx<T>::step_rk4(double dt, int64_t nsteps, cudaStream_t s) {
  const T h = static_cast<T>(dt);
  for (int64_t it = 0; it < nsteps; ++it) {
    const T* in[4] = {m.p, ms0.p, ms1.p, ms0.p};
    T* out[4] = {ms0.p, ms1.p, ms0.p, nullptr};
    const T cnext[4] = {T(0.5) * h, T(0.5) * h, h, T(0)};
    const T wacc[4] = {T(1), T(2), T(2), T(0)};
    for (int st = 0; st < 4; ++st) {
      if (use_demag) demag->potential(in[st], s, false);
      StageArgs<T> a = args(in[st], out[st], 2, use_demag);
      a.mn = m.p;
      a.acc = acc.p;
      a.stage = st;
      a.c_next = cnext[st];
      a.w_acc = wacc[st];
      a.dt6 = h / T(6);
      Profiler* pf = use_demag ? &demag->prof : nullptr;
      if (pf) pf->mark(PC_STAGE, s);
      launch_stage(a, use_demag, s);
      if (pf) {
        pf->mark(PC_STAGE, s);
        pf->launches[PC_STAGE] += 1;
      }
      ++rhs_evals;
    }
    ++steps;
  }
}

template <class T>
void LLGCtx<T>::update_jac_state(const T* min, cudaStream_t s) {
  SPX_CUDA(cudaMemcpyAsync(Mstate.p, min, 3 * N * sizeof(T), cudaMemcpyDeviceToDevice, s));
  launch_stage(args(Mstate.p, Hm.p, 0, false), false, s);
}

template <class T>
void LLGCtx<T>::jv(const T* v, T* out, cudaStream_t s) {
  StageArgs<T> a = args(Mstate.p, out, 0, false);
  const unsigned g = grid_for(a.nslices * 32, 256);
  const T gam = static_cast<T>(prm.gamma);
  if (has_dmi && has_ani) k_jv<T, true, true><<<g, 256, 0, s>>>(a, Mstate.p, Hm.p, v, out, gam);
  else if (has_dmi) k_jv<T, true, false><<<g, 256, 0, s>>>(a, Mstate.p, Hm.p, v, out, gam);
  else if (has_ani) k_jv<T, false, true><<<g, 256, 0, s>>>(a, Mstate.p, Hm.p, v, out, gam);
  else k_jv<T, false, false><<<g, 256, 0, s>>>(a, Mstate.p, Hm.p, v, out, gam);
  SPX_LAUNCH_CHECK();
}

template <class T>
void LLGCtx<T>::pc_build(double shift, int include_stab, int use_abs_kappa, cudaStream_t s) {
  k_pc_build<T><<<grid_for(N, 256), 256, 0, s>>>(N, Mstate.p, Hm.p, diagK.p, include_stab, use_abs_kappa, shift,
                                                 1e-14, 1e-30, c1, c2, stab, pcinv.p);
  SPX_LAUNCH_CHECK();
  pc_ready = true;
}

template <class T>
void LLGCtx<T>::pc_apply(const T* x, T* y, cudaStream_t s) {
  if (!pc_ready) {
    SPX_CUDA(cudaMemcpyAsync(y, x, 3 * N * sizeof(T), cudaMemcpyDeviceToDevice, s));
    return;
  }
  k_pc_apply<T><<<grid_for(N, 256), 256, 0, s>>>(N, pcinv.p, x, y);
  SPX_LAUNCH_CHECK();
}

template <class T>
double LLGCtx<T>::mdoth(const double* w, const T* a, const T* b, cudaStream_t s) {
  SPX_CUDA(cudaMemsetAsync(red.p, 0, sizeof(double), s));
  k_mdoth<T><<<std::min<unsigned>(grid_for(N, 256), 1184), 256, 0, s>>>(N, w, a, b, red.p);
  SPX_LAUNCH_CHECK();
  double h = 0.0;
  SPX_CUDA(cudaMemcpyAsync(&h, red.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  return h;
}

template struct LLGCtx<double>;
template struct LLGCtx<float>;

template <class T>
double demag_energy(DemagCtx<T>& d, const T* m, const T* H, cudaStream_t s) {
  DevBuf<double> r(1);
  r.zero(s);
  k_mdoth<T><<<std::min<unsigned>(grid_for(d.N, 256), 1184), 256, 0, s>>>(d.N, d.vol.p, m, H, r.p);
  SPX_LAUNCH_CHECK();
  double h = 0.0;
  SPX_CUDA(cudaMemcpyAsync(&h, r.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  return -0.5 * d.mu0 * d.Ms * h / 1e27;
}
template double demag_energy<double>(DemagCtx<double>&, const double*, const double*, cudaStream_t);
template double demag_energy<float>(DemagCtx<float>&, const float*, const float*, cudaStream_t);

}  // namespace spx
