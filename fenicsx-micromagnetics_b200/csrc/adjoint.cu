// Adjoint (vector-Jacobian) and tangent (Jacobian-vector) products of the demag map and of
// the LLG RK4 step.  The reference has no adjoint; these operators exist for gradients of
// trajectory losses with respect to the magnetisation, a nodal Ku(x) map and the uniform
// applied field.
//
// Demag map D: m -> H = Gv phi (fem.cu):
//   b = Div m ;  u1 = Pi A^+ Pi b ;  g = B u1|bnd ;  u_I = -A_II^-1 A_IB g ;
//   phi = u1 + [g ; u_I] ;  H = Gv phi
// so D^T w = Div^T Pi A^+ Pi (psi + E^T B^T (psi_B - A_BI A_II^-1 psi_I)),  psi = Gv^T w,
// with E the boundary restriction and Pi the projection that removes the constant.  Gv^T
// and Div^T are the forward value planes moved to the transposed positions of the
// (structurally symmetric) P1 pattern; B^T is a transposed dense GEMV or the transposed
// H-matrix (HMatrix::transposed); both Poisson systems are symmetric and reuse the forward
// solvers.
//
// LLG right-hand side f(m) = pref (p m x H + alpha m x (m x H)) + stab (1 - |m|^2) m with
// H = L m + H0 (L: exchange + DMI + anisotropy + demag, linear):
//   J^T w = T^T w + L^T u,   u = (df/dH)^T w = pref (p (w x m) + alpha (w x m) x m),
//   T^T w = pref (p H x w + alpha ((m x H) x w + H x (w x m))) + stab (1-|m|^2) w - 2 stab (m.w) m.
//   dL/dKu_i = 2/(mu0 Ms) (m_i.n_i)(n_i.u_i),   dL/dH0 = sum_i u_i.
// RK4 step backward (y1 = m, y2 = m + h/2 k1, y3 = m + h/2 k2, y4 = m + h k3):
//   a4 = J4^T (h/6 l), a3 = J3^T (h/3 l + h a4), a2 = J2^T (h/3 l + h/2 a3),
//   a1 = J1^T (h/6 l + h/2 a2),  l_n = l + a1 + a2 + a3 + a4.
#include <algorithm>
#include <cmath>

#include "llg.cuh"

namespace spx {

namespace {

#define ADJ_SELL_LOOP(nslices, ...)                                                    \
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

// out_j = sum_i sum_c P_c(j,i) w_(i,c)   (difference form plus row sums S)
template <class TV, class TM>
__global__ void k_planes3_to1(int64_t n, int64_t nslices, const int64_t* __restrict__ sp,
                              const int32_t* __restrict__ col, const TM* __restrict__ P, int64_t L,
                              const double* __restrict__ S, const TV* __restrict__ w, TV* __restrict__ out) {
  ADJ_SELL_LOOP(nslices, {
    if (row < n) {
      const TV wx = w[3 * row], wy = w[3 * row + 1], wz = w[3 * row + 2];
      TV acc = 0;
      for (int k = 0; k < width; ++k) {
        const int64_t idx = base_ + ((int64_t)k << 5) + lane_;
        const int64_t j = col[idx];
        acc += static_cast<TV>(P[idx]) * (w[3 * j] - wx) + static_cast<TV>(P[L + idx]) * (w[3 * j + 1] - wy) +
               static_cast<TV>(P[2 * L + idx]) * (w[3 * j + 2] - wz);
      }
      acc += static_cast<TV>(S[row]) * wx + static_cast<TV>(S[n + row]) * wy + static_cast<TV>(S[2 * n + row]) * wz;
      out[row] = acc;
    }
  })
}

// out_(j,c) (+)= sum_i P_c(j,i) (y_i - y_j)   (rows of P_c sum to zero)
template <class TV, class TM>
__global__ void k_planes1_to3(int64_t n, int64_t nslices, const int64_t* __restrict__ sp,
                              const int32_t* __restrict__ col, const TM* __restrict__ P, int64_t L,
                              const TV* __restrict__ y, TV* __restrict__ out, int accumulate) {
  ADJ_SELL_LOOP(nslices, {
    if (row < n) {
      const TV yi = y[row];
      TV ox = 0, oy = 0, oz = 0;
      for (int k = 0; k < width; ++k) {
        const int64_t idx = base_ + ((int64_t)k << 5) + lane_;
        const TV d = y[col[idx]] - yi;
        ox += static_cast<TV>(P[idx]) * d;
        oy += static_cast<TV>(P[L + idx]) * d;
        oz += static_cast<TV>(P[2 * L + idx]) * d;
      }
      if (accumulate) {
        out[3 * row] += ox;
        out[3 * row + 1] += oy;
        out[3 * row + 2] += oz;
      } else {
        out[3 * row] = ox;
        out[3 * row + 1] = oy;
        out[3 * row + 2] = oz;
      }
    }
  })
}

template <class T>
__global__ void k_gather(int64_t n, const int32_t* __restrict__ idx, const T* __restrict__ src, T* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

template <class T>
__global__ void k_scatter_add(int64_t n, const int32_t* __restrict__ idx, const T* __restrict__ src, T* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[idx[i]] += src[i];
}

// gbar_b = psi[bverts[b]] - sum_i A_bi xI_i  (boundary rows, interior columns)
template <class TV>
__global__ void k_bnd_adj(int64_t nb, int64_t nslices, const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                          const double* __restrict__ v, const TV* __restrict__ xI, const TV* __restrict__ psi,
                          const int32_t* __restrict__ bverts, TV* __restrict__ gbar) {
  ADJ_SELL_LOOP(nslices, {
    if (row < nb) {
      double acc = 0.0;
      for (int k = 0; k < width; ++k) {
        const int64_t idx = base_ + ((int64_t)k << 5) + lane_;
        acc += v[idx] * static_cast<double>(xI[col[idx]]);
      }
      gbar[row] = static_cast<TV>(static_cast<double>(psi[bverts[row]]) - acc);
    }
  })
}

// partial[r][j] = sum over rows i of chunk r of B_ij x_i  (B row-major Nb x Nb, FP64)
template <class TV>
__global__ void k_dense_gemv_t(int64_t Nb, const double* __restrict__ B, const TV* __restrict__ x, int64_t chunk,
                               double* __restrict__ part) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= Nb) return;
  const int64_t i0 = blockIdx.y * chunk, i1 = std::min<int64_t>(Nb, i0 + chunk);
  double acc = 0.0;
  for (int64_t i = i0; i < i1; ++i) acc += B[i * Nb + j] * static_cast<double>(x[i]);
  part[blockIdx.y * Nb + j] = acc;
}

template <class TV>
__global__ void k_sum_parts(int64_t Nb, int R, const double* __restrict__ part, TV* __restrict__ y) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= Nb) return;
  double acc = 0.0;
  for (int r = 0; r < R; ++r) acc += part[r * Nb + j];
  y[j] = static_cast<TV>(acc);
}

// ---------------------------------------------------------------- LLG kernels
template <class TV>
struct LocalPrm {
  const TV* ani_n;
  const TV* ani_p;
  TV ani_p0;
  TV pref, alpha, precess, stab;
  double kuscale;  // 2 / (mu0 Ms)
};

template <class TV>
__device__ __forceinline__ void cross3(TV ax, TV ay, TV az, TV bx, TV by, TV bz, TV& cx, TV& cy, TV& cz) {
  cx = ay * bz - az * by;
  cy = az * bx - ax * bz;
  cz = ax * by - ay * bx;
}

// a = T^T w (overwrite), u = (df/dH)^T w, gKu_i += kuscale (m.n)(n.u)
template <class TV>
__global__ void k_vjp_local(int64_t n, const TV* __restrict__ m, const TV* __restrict__ H, const TV* __restrict__ w,
                            LocalPrm<TV> q, TV* __restrict__ a, TV* __restrict__ u, double* __restrict__ gKu) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TV mx = m[3 * i], my = m[3 * i + 1], mz = m[3 * i + 2];
  const TV hx = H[3 * i], hy = H[3 * i + 1], hz = H[3 * i + 2];
  const TV wx = w[3 * i], wy = w[3 * i + 1], wz = w[3 * i + 2];
  TV hwx, hwy, hwz, mhx, mhy, mhz, mhwx, mhwy, mhwz, wmx, wmy, wmz, hwmx, hwmy, hwmz, wmmx, wmmy, wmmz;
  cross3(hx, hy, hz, wx, wy, wz, hwx, hwy, hwz);
  cross3(mx, my, mz, hx, hy, hz, mhx, mhy, mhz);
  cross3(mhx, mhy, mhz, wx, wy, wz, mhwx, mhwy, mhwz);
  cross3(wx, wy, wz, mx, my, mz, wmx, wmy, wmz);
  cross3(hx, hy, hz, wmx, wmy, wmz, hwmx, hwmy, hwmz);
  cross3(wmx, wmy, wmz, mx, my, mz, wmmx, wmmy, wmmz);
  const TV mm = mx * mx + my * my + mz * mz, mw = mx * wx + my * wy + mz * wz;
  const TV s0 = q.stab * (TV(1) - mm), s1 = TV(2) * q.stab * mw;
  a[3 * i] = q.pref * (q.precess * hwx + q.alpha * (mhwx + hwmx)) + s0 * wx - s1 * mx;
  a[3 * i + 1] = q.pref * (q.precess * hwy + q.alpha * (mhwy + hwmy)) + s0 * wy - s1 * my;
  a[3 * i + 2] = q.pref * (q.precess * hwz + q.alpha * (mhwz + hwmz)) + s0 * wz - s1 * mz;
  const TV ux = q.pref * (q.precess * wmx + q.alpha * wmmx);
  const TV uy = q.pref * (q.precess * wmy + q.alpha * wmmy);
  const TV uz = q.pref * (q.precess * wmz + q.alpha * wmmz);
  u[3 * i] = ux;
  u[3 * i + 1] = uy;
  u[3 * i + 2] = uz;
  if (gKu && q.ani_n) {
    const TV nx = q.ani_n[3 * i], ny = q.ani_n[3 * i + 1], nz = q.ani_n[3 * i + 2];
    gKu[i] += q.kuscale * static_cast<double>(mx * nx + my * ny + mz * nz) *
              static_cast<double>(nx * ux + ny * uy + nz * uz);
  }
}

// a_i += (L_lin^T u)_i : transposed exchange and DMI (explicit planes + row sums), anisotropy
template <class TV, class TM, bool DMI, bool ANI>
__global__ void k_lin_t(int64_t n, int64_t nslices, const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                        int64_t L, const TM* __restrict__ KexT, const double* __restrict__ KexTsum,
                        const TM* __restrict__ KdT, const double* __restrict__ KdTsum, LocalPrm<TV> q,
                        const TV* __restrict__ u, TV* __restrict__ a) {
  ADJ_SELL_LOOP(nslices, {
    if (row < n) {
      const int64_t i = row;
      const TV ux = u[3 * i], uy = u[3 * i + 1], uz = u[3 * i + 2];
      TV hx = 0, hy = 0, hz = 0;
      for (int k = 0; k < width; ++k) {
        const int64_t idx = base_ + ((int64_t)k << 5) + lane_;
        const int64_t j = col[idx];
        const TV dx = u[3 * j] - ux, dy = u[3 * j + 1] - uy, dz = u[3 * j + 2] - uz;
        const TV e = static_cast<TV>(KexT[idx]);
        hx += e * dx;
        hy += e * dy;
        hz += e * dz;
        if (DMI) {
          const TM* K = KdT + idx;
          hx += static_cast<TV>(K[0]) * dx + static_cast<TV>(K[L]) * dy + static_cast<TV>(K[2 * L]) * dz;
          hy += static_cast<TV>(K[3 * L]) * dx + static_cast<TV>(K[4 * L]) * dy + static_cast<TV>(K[5 * L]) * dz;
          hz += static_cast<TV>(K[6 * L]) * dx + static_cast<TV>(K[7 * L]) * dy + static_cast<TV>(K[8 * L]) * dz;
        }
      }
      const TV es = static_cast<TV>(KexTsum[i]);
      hx += es * ux;
      hy += es * uy;
      hz += es * uz;
      if (DMI) {
        const double* S = KdTsum;
        hx += static_cast<TV>(S[i]) * ux + static_cast<TV>(S[n + i]) * uy + static_cast<TV>(S[2 * n + i]) * uz;
        hy += static_cast<TV>(S[3 * n + i]) * ux + static_cast<TV>(S[4 * n + i]) * uy + static_cast<TV>(S[5 * n + i]) * uz;
        hz += static_cast<TV>(S[6 * n + i]) * ux + static_cast<TV>(S[7 * n + i]) * uy + static_cast<TV>(S[8 * n + i]) * uz;
      }
      if (ANI) {
        const TV nx = q.ani_n[3 * i], ny = q.ani_n[3 * i + 1], nz = q.ani_n[3 * i + 2];
        const TV c = (q.ani_p ? q.ani_p[i] : q.ani_p0) * (ux * nx + uy * ny + uz * nz);
        hx += c * nx;
        hy += c * ny;
        hz += c * nz;
      }
      a[3 * i] += hx;
      a[3 * i + 1] += hy;
      a[3 * i + 2] += hz;
    }
  })
}

// per-CTA partial sums of the three components of u (fixed grid, deterministic order)
constexpr int SUM3_GRID = 148;
template <class TV>
__global__ void k_sum3_part(int64_t n, const TV* __restrict__ u, double* __restrict__ part) {
  __shared__ double sh[32];
  double s[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int c = 0; c < 3; ++c) s[c] += static_cast<double>(u[3 * i + c]);
  for (int c = 0; c < 3; ++c) {
    const double t = block_sum(s[c], sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x + c] = t;
  }
}

__global__ void k_sum3_final(int nparts, const double* __restrict__ part, double* __restrict__ g) {
  const int c = threadIdx.x;
  if (c >= 3) return;
  double acc = 0.0;
  for (int b = 0; b < nparts; ++b) acc += part[3 * b + c];
  g[c] += acc;
}

// Y_next = mn + c f(Y, H)
template <class TV>
__global__ void k_fwd_next(int64_t n, const TV* __restrict__ mn, const TV* __restrict__ Y, const TV* __restrict__ H,
                           TV c, LocalPrm<TV> q, TV* __restrict__ Yn) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TV mx = Y[3 * i], my = Y[3 * i + 1], mz = Y[3 * i + 2];
  const TV hx = H[3 * i], hy = H[3 * i + 1], hz = H[3 * i + 2];
  TV cx, cy, cz, ccx, ccy, ccz;
  cross3(mx, my, mz, hx, hy, hz, cx, cy, cz);
  cross3(mx, my, mz, cx, cy, cz, ccx, ccy, ccz);
  const TV s = q.stab * (TV(1) - (mx * mx + my * my + mz * mz));
  Yn[3 * i] = mn[3 * i] + c * (q.pref * (q.precess * cx + q.alpha * ccx) + s * mx);
  Yn[3 * i + 1] = mn[3 * i + 1] + c * (q.pref * (q.precess * cy + q.alpha * ccy) + s * my);
  Yn[3 * i + 2] = mn[3 * i + 2] + c * (q.pref * (q.precess * cz + q.alpha * ccz) + s * mz);
}

// out = ca a + cb b (b may be null)
template <class TV>
__global__ void k_comb(int64_t n, TV* __restrict__ out, TV ca, const TV* __restrict__ a, TV cb, const TV* __restrict__ b) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = ca * a[i] + (b ? cb * b[i] : TV(0));
}

template <class TV>
__global__ void k_add(int64_t n, TV* __restrict__ out, const TV* __restrict__ a) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] += a[i];
}

// one RK4 stage of the primal and tangent systems:
//   k = f(Y, H), dk = T dY + df/dH (dH + dKu term + dH0),
//   stage < 3: Yn = mn + c k, dYn = dm + c dk, K/dK accumulate; stage 3: m_out, dm_out
template <class TV>
__global__ void k_tan_stage(int64_t n, const TV* __restrict__ mn, const TV* __restrict__ dm, const TV* __restrict__ Y,
                            const TV* __restrict__ H, const TV* __restrict__ dY, const TV* __restrict__ dH,
                            const double* __restrict__ dKu, TV d0x, TV d0y, TV d0z, LocalPrm<TV> q, int stage, TV c,
                            TV wacc, TV h6, TV* __restrict__ Yn, TV* __restrict__ dYn, TV* __restrict__ K,
                            TV* __restrict__ dK, TV* __restrict__ m_out, TV* __restrict__ dm_out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TV mx = Y[3 * i], my = Y[3 * i + 1], mz = Y[3 * i + 2];
  const TV hx = H[3 * i], hy = H[3 * i + 1], hz = H[3 * i + 2];
  const TV vx = dY[3 * i], vy = dY[3 * i + 1], vz = dY[3 * i + 2];
  TV gx = dH[3 * i] + d0x, gy = dH[3 * i + 1] + d0y, gz = dH[3 * i + 2] + d0z;
  if (dKu && q.ani_n) {
    const TV nx = q.ani_n[3 * i], ny = q.ani_n[3 * i + 1], nz = q.ani_n[3 * i + 2];
    const TV t = static_cast<TV>(q.kuscale * dKu[i]) * (mx * nx + my * ny + mz * nz);
    gx += t * nx;
    gy += t * ny;
    gz += t * nz;
  }
  TV cx, cy, cz, ccx, ccy, ccz;
  cross3(mx, my, mz, hx, hy, hz, cx, cy, cz);
  cross3(mx, my, mz, cx, cy, cz, ccx, ccy, ccz);
  const TV mm = mx * mx + my * my + mz * mz;
  const TV s = q.stab * (TV(1) - mm);
  const TV kx = q.pref * (q.precess * cx + q.alpha * ccx) + s * mx;
  const TV ky = q.pref * (q.precess * cy + q.alpha * ccy) + s * my;
  const TV kz = q.pref * (q.precess * cz + q.alpha * ccz) + s * mz;
  // T v = pref (p v x H + alpha (v x (m x H) + m x (v x H))) + stab (1-|m|^2) v - 2 stab (m.v) m
  TV a1x, a1y, a1z, a2x, a2y, a2z, vhx, vhy, vhz, a3x, a3y, a3z;
  cross3(vx, vy, vz, hx, hy, hz, vhx, vhy, vhz);
  cross3(vx, vy, vz, cx, cy, cz, a2x, a2y, a2z);
  cross3(mx, my, mz, vhx, vhy, vhz, a3x, a3y, a3z);
  // df/dH g = pref (p m x g + alpha m x (m x g))
  TV mgx, mgy, mgz, mmgx, mmgy, mmgz;
  cross3(mx, my, mz, gx, gy, gz, mgx, mgy, mgz);
  cross3(mx, my, mz, mgx, mgy, mgz, mmgx, mmgy, mmgz);
  const TV mv = mx * vx + my * vy + mz * vz;
  const TV s2 = TV(2) * q.stab * mv;
  a1x = q.pref * (q.precess * (vhx + mgx) + q.alpha * (a2x + a3x + mmgx)) + s * vx - s2 * mx;
  a1y = q.pref * (q.precess * (vhy + mgy) + q.alpha * (a2y + a3y + mmgy)) + s * vy - s2 * my;
  a1z = q.pref * (q.precess * (vhz + mgz) + q.alpha * (a2z + a3z + mmgz)) + s * vz - s2 * mz;
  TV* Kp = K + 3 * i;
  TV* dKp = dK + 3 * i;
  if (stage == 0) {
    Kp[0] = kx; Kp[1] = ky; Kp[2] = kz;
    dKp[0] = a1x; dKp[1] = a1y; dKp[2] = a1z;
  } else if (stage < 3) {
    Kp[0] += wacc * kx; Kp[1] += wacc * ky; Kp[2] += wacc * kz;
    dKp[0] += wacc * a1x; dKp[1] += wacc * a1y; dKp[2] += wacc * a1z;
  }
  if (stage < 3) {
    Yn[3 * i] = mn[3 * i] + c * kx;
    Yn[3 * i + 1] = mn[3 * i + 1] + c * ky;
    Yn[3 * i + 2] = mn[3 * i + 2] + c * kz;
    dYn[3 * i] = dm[3 * i] + c * a1x;
    dYn[3 * i + 1] = dm[3 * i + 1] + c * a1y;
    dYn[3 * i + 2] = dm[3 * i + 2] + c * a1z;
  } else {
    const TV ox = mn[3 * i] + h6 * (Kp[0] + kx), oy = mn[3 * i + 1] + h6 * (Kp[1] + ky),
             oz = mn[3 * i + 2] + h6 * (Kp[2] + kz);
    const TV px = dm[3 * i] + h6 * (dKp[0] + a1x), py = dm[3 * i + 1] + h6 * (dKp[1] + a1y),
             pz = dm[3 * i + 2] + h6 * (dKp[2] + a1z);
    m_out[3 * i] = ox; m_out[3 * i + 1] = oy; m_out[3 * i + 2] = oz;
    dm_out[3 * i] = px; dm_out[3 * i + 1] = py; dm_out[3 * i + 2] = pz;
  }
}

// CSR position of (j, i) for every entry (i, j) of a structurally symmetric pattern
std::vector<int64_t> transpose_positions(const std::vector<int64_t>& rowptr, const std::vector<int32_t>& col) {
  const int64_t N = static_cast<int64_t>(rowptr.size()) - 1;
  std::vector<int64_t> t(rowptr.back(), -1);
  for (int64_t i = 0; i < N; ++i)
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
      const int32_t j = col[k];
      const auto b = col.begin() + rowptr[j], e = col.begin() + rowptr[j + 1];
      const auto it = std::lower_bound(b, e, static_cast<int32_t>(i));
      SPX_CHECK(it != e && *it == i, "FEM pattern is not structurally symmetric");
      t[k] = static_cast<int64_t>(it - col.begin());
    }
  return t;
}

}  // namespace

// ================================================================ demag adjoint
template <class TV, class TM>
void DemagCtx<TV, TM>::apply_transpose(const TV* w, TV* out, bool accumulate, int slot, cudaStream_t s) {
  DemagAdjoint<TV, TM>& A = adj;
  const int64_t nnz = fem.rowptr[N];
  SPX_CHECK(opt.backend != 2, "the ensemble backend has no transposed boundary operator");
  if (!A.ready) {
    const std::vector<int64_t> tp = transpose_positions(fem.rowptr, fem.col);
    std::vector<double> gt(3 * nnz), dt(3 * nnz), gsum(3 * N, 0.0);
    for (int64_t j = 0; j < N; ++j)
      for (int64_t k = fem.rowptr[j]; k < fem.rowptr[j + 1]; ++k) {
        const int64_t kt = tp[k];  // entry (i, j) in row i = col[k]
        const int32_t i = fem.col[k];
        for (int c = 0; c < 3; ++c) {
          gt[3 * k + c] = fem.G[3 * kt + c] / fem.vol[i];
          dt[3 * k + c] = Ms * fem.Div[3 * kt + c];
          gsum[c * N + j] += gt[3 * k + c];
        }
      }
    std::vector<TM> v;
    sell_values<TM>(hsell, gt.data(), 3, true, nnz, 1.0, v);
    A.GvT.upload(v, s);
    sell_values<TM>(hsell, dt.data(), 3, true, nnz, 1.0, v);
    A.DivT.upload(v, s);
    A.GvTsum.upload(gsum, s);
    if (NI > 0) {
      std::vector<int32_t> imap(N, -1);
      std::vector<int32_t> inter(NI);
      SPX_CUDA(cudaMemcpy(inter.data(), interior.p, NI * sizeof(int32_t), cudaMemcpyDeviceToHost));
      for (int64_t q = 0; q < NI; ++q) imap[inter[q]] = static_cast<int32_t>(q);
      HostSell sBI;
      build_sell(fem.rowptr, fem.col, bd.host.bverts, &imap, sBI);
      std::vector<double> aBI;
      sell_values<double>(sBI, fem.A.data(), 1, true, nnz, 1.0, aBI);
      A.PBI.upload(sBI, s);
      A.ABI.upload(aBI, s);
    }
    A.psi.alloc(N); A.u1bar.alloc(N); A.bbar.alloc(N);
    A.gbar.alloc(Nb); A.yb.alloc(Nb);
    A.bIbar.alloc(std::max<int64_t>(NI, 1));
    A.xIbar.alloc(std::max<int64_t>(NI, 1));
    A.bbar.zero(s);
    A.xIbar.zero(s);
    if (opt.backend == 1) H.transposed(s);
    SPX_CUDA(cudaStreamSynchronize(s));
    A.ready = true;
  }
  ++epoch;
  // adjoint solves start from the extrapolation of earlier adjoint solutions of the same RK
  // stage (slots 4-7) when warm starts are on, from zero otherwise
  const int sl = (opt.warm_start != 0 && slot >= 0) ? slot : -1;
  const bool warm = sl >= 0;
  const unsigned gs = grid_for(P.nslices * 32, 256);
  // psi = Gv^T w
  k_planes3_to1<TV, TM><<<gs, 256, 0, s>>>(N, P.nslices, P.slice_ptr.p, P.col.p, A.GvT.p, P.len, A.GvTsum.p, w,
                                            A.psi.p);
  SPX_LAUNCH_CHECK();
  // gbar = psi_B - A_BI A_II^-1 psi_I
  if (NI > 0) {
    k_gather<TV><<<grid_for(NI, 256), 256, 0, s>>>(NI, interior.p, A.psi.p, A.bIbar.p);
    SPX_LAUNCH_CHECK();
    cg2.template solve<TV>(A.bIbar.p, A.xIbar.p, opt.rtol_u2, opt.atol, opt.maxit_u2, warm, false, sl, s, false, 1);
    k_bnd_adj<TV><<<grid_for(A.PBI.nslices * 32, 256), 256, 0, s>>>(Nb, A.PBI.nslices, A.PBI.slice_ptr.p,
                                                                     A.PBI.col.p, A.ABI.p, A.xIbar.p, A.psi.p,
                                                                     bverts.p, A.gbar.p);
    SPX_LAUNCH_CHECK();
  } else {
    k_gather<TV><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, bverts.p, A.psi.p, A.gbar.p);
    SPX_LAUNCH_CHECK();
  }
  // yb = B^T gbar
  if (opt.backend == 0) {
    const int R = static_cast<int>(std::min<int64_t>(32, std::max<int64_t>(1, Nb / 256)));
    const int64_t chunk = (Nb + R - 1) / R;
    if (A.part.n < static_cast<size_t>(R * Nb)) A.part.alloc(R * Nb);
    k_dense_gemv_t<TV><<<dim3(grid_for(Nb, 256), R), 256, 0, s>>>(Nb, Bdense.p, A.gbar.p, chunk, A.part.p);
    SPX_LAUNCH_CHECK();
    k_sum_parts<TV><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, R, A.part.p, A.yb.p);
    SPX_LAUNCH_CHECK();
  } else {
    H.transposed(s).template apply_gather<TV>(A.gbar.p, nullptr, A.yb.p, nullptr, nullptr, s);
  }
  // u1bar = psi + E^T yb ; bbar = Pi A^+ Pi u1bar ; out (+)= Div^T bbar
  SPX_CUDA(cudaMemcpyAsync(A.u1bar.p, A.psi.p, N * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  k_scatter_add<TV><<<grid_for(Nb, 256), 256, 0, s>>>(Nb, bverts.p, A.yb.p, A.u1bar.p);
  SPX_LAUNCH_CHECK();
  cg1.template solve<TV>(A.u1bar.p, A.bbar.p, opt.rtol_u1, opt.atol, opt.maxit_u1, warm, true, sl, s, false, 1);
  k_planes1_to3<TV, TM><<<gs, 256, 0, s>>>(N, P.nslices, P.slice_ptr.p, P.col.p, A.DivT.p, P.len, A.bbar.p, out,
                                            accumulate ? 1 : 0);
  SPX_LAUNCH_CHECK();
}

template void DemagCtx<double, double>::apply_transpose(const double*, double*, bool, int, cudaStream_t);
template void DemagCtx<float, float>::apply_transpose(const float*, float*, bool, int, cudaStream_t);
template void DemagCtx<double, float>::apply_transpose(const double*, double*, bool, int, cudaStream_t);

// ================================================================ LLG adjoint / tangent
template <class TV, class TM>
void LLGCtx<TV, TM>::adjoint_setup(cudaStream_t s) {
  LLGAdjoint<TV, TM>& A = adj;
  if (A.ready) return;
  SPX_CHECK(!has_stt && !has_sot, "adjoint and tangent products do not include spin torques");
  const HostFem& fem = demag ? demag->fem : own_fem;
  const HostSell& hs = demag ? demag->hsell : own_sell;
  const int64_t nnz = fem.rowptr[N];
  const double mu0 = 4e-7 * 3.141592653589793;
  const std::vector<int64_t> tp = transpose_positions(fem.rowptr, fem.col);
  {
    std::vector<double> kt(nnz, 0.0), ks(N, 0.0);
    for (int64_t j = 0; j < N; ++j)
      for (int64_t k = fem.rowptr[j]; k < fem.rowptr[j + 1]; ++k) {
        const int32_t i = fem.col[k];
        const double sc = (prm.Aex != 0.0) ? -2.0 * prm.Aex / (mu0 * prm.Ms) / fem.vol[i] / 1e-18 : 0.0;
        kt[k] = sc * fem.A[tp[k]];
        ks[j] += kt[k];
      }
    std::vector<TM> v;
    sell_values<TM>(hs, kt.data(), 1, true, nnz, 1.0, v);
    A.KexT.upload(v, s);
    A.KexTsum.upload(ks, s);
  }
  if (has_dmi) {
    HostBoundary bhost;
    const HostBoundary* bh = nullptr;
    if (demag) bh = &demag->bd.host;
    else { build_boundary(X_host.data(), N, tets_host.data(), static_cast<int64_t>(tets_host.size() / 4), bhost); bh = &bhost; }
    std::vector<double> b9;
    dmi_blocks_scaled(X_host.data(), tets_host.data(), static_cast<int64_t>(tets_host.size() / 4), fem, *bh,
                      prm.Ms, prm.D_int, n_int_host.empty() ? nullptr : n_int_host.data(), prm.D_bulk, b9);
    std::vector<double> bt(9 * nnz), ks(9 * N, 0.0);
    for (int64_t j = 0; j < N; ++j)
      for (int64_t k = fem.rowptr[j]; k < fem.rowptr[j + 1]; ++k) {
        const int64_t kt = tp[k];
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            const double v = b9[9 * kt + 3 * r + c];  // block (i, j)[r][c] -> (j, i)[c][r]
            bt[9 * k + 3 * c + r] = v;
            ks[(3 * c + r) * N + j] += v;
          }
      }
    std::vector<TM> v;
    sell_values<TM>(hs, bt.data(), 9, true, nnz, 1.0, v);
    A.KdT.upload(v, s);
    A.KdTsum.upload(ks, s);
  }
  for (int k = 0; k < 4; ++k) {
    A.Y[k].alloc(3 * N);
    A.Hs[k].alloc(3 * N);
  }
  A.dY[0].alloc(3 * N); A.dY[1].alloc(3 * N);
  A.u.alloc(3 * N); A.w.alloc(3 * N); A.a.alloc(3 * N); A.ap.alloc(3 * N); A.lam.alloc(3 * N);
  A.acc.alloc(3 * N); A.K.alloc(3 * N); A.dK.alloc(3 * N); A.dH.alloc(3 * N);
  A.part.alloc(3 * SUM3_GRID);
  SPX_CUDA(cudaStreamSynchronize(s));
  A.ready = true;
}

namespace {
template <class TV, class TM>
LocalPrm<TV> local_prm(const LLGCtx<TV, TM>& c) {
  LocalPrm<TV> q{};
  q.ani_n = c.has_ani ? c.ani_n.p : nullptr;
  q.ani_p = (c.has_ani && c.ani_p.n) ? c.ani_p.p : nullptr;
  q.ani_p0 = static_cast<TV>(c.ani_p0);
  q.pref = static_cast<TV>(c.pref);
  q.alpha = static_cast<TV>(c.prm.alpha);
  q.precess = static_cast<TV>(c.prm.do_precess);
  q.stab = static_cast<TV>(c.stab);
  q.kuscale = 2.0 / (4e-7 * 3.141592653589793 * c.prm.Ms);
  return q;
}
}  // namespace

template <class TV, class TM>
void LLGCtx<TV, TM>::rhs_vjp(const TV* min, const TV* H, const TV* w, TV* out, double* gKu, double* gH0, int slot,
                             cudaStream_t s) {
  adjoint_setup(s);
  LLGAdjoint<TV, TM>& A = adj;
  const LocalPrm<TV> q = local_prm(*this);
  k_vjp_local<TV><<<grid_for(N, 256), 256, 0, s>>>(N, min, H, w, q, out, A.u.p, gKu);
  SPX_LAUNCH_CHECK();
  const unsigned g = grid_for(P.nslices * 32, 256);
#define SPX_LINT(DM, AN)                                                                                   \
  k_lin_t<TV, TM, DM, AN><<<g, 256, 0, s>>>(N, P.nslices, P.slice_ptr.p, P.col.p, P.len, A.KexT.p, A.KexTsum.p, \
                                            has_dmi ? A.KdT.p : nullptr, has_dmi ? A.KdTsum.p : nullptr, q, A.u.p, out)
  if (has_dmi && has_ani) SPX_LINT(true, true);
  else if (has_dmi) SPX_LINT(true, false);
  else if (has_ani) SPX_LINT(false, true);
  else SPX_LINT(false, false);
#undef SPX_LINT
  SPX_LAUNCH_CHECK();
  if (use_demag) demag->apply_transpose(A.u.p, out, true, slot, s);
  if (gH0) {
    k_sum3_part<TV><<<SUM3_GRID, 256, 0, s>>>(N, A.u.p, A.part.p);
    SPX_LAUNCH_CHECK();
    k_sum3_final<<<1, 32, 0, s>>>(SUM3_GRID, A.part.p, gH0);
    SPX_LAUNCH_CHECK();
  }
}

template <class TV, class TM>
void LLGCtx<TV, TM>::step_vjp(const TV* mn, double dt, const TV* lam_in, TV* lam_out, double* gKu, double* gH0,
                              cudaStream_t s) {
  adjoint_setup(s);
  LLGAdjoint<TV, TM>& A = adj;
  const int64_t n3 = 3 * N;
  const LocalPrm<TV> q = local_prm(*this);
  const TV h = static_cast<TV>(dt);
  const unsigned ge = grid_for(N, 256), g3 = grid_for(n3, 256);
  // primal stages: Y_s and H(Y_s)
  SPX_CUDA(cudaMemcpyAsync(A.Y[0].p, mn, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  SPX_CUDA(cudaMemcpyAsync(A.lam.p, lam_in, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  const TV cn[3] = {TV(0.5) * h, TV(0.5) * h, h};
  for (int st = 0; st < 4; ++st) {
    if (use_demag) demag->potential(A.Y[st].p, s, false, st);
    launch_stage(args(A.Y[st].p, A.Hs[st].p, 0, use_demag), use_demag, s);
    if (st < 3) {
      k_fwd_next<TV><<<ge, 256, 0, s>>>(N, mn, A.Y[st].p, A.Hs[st].p, cn[st], q, A.Y[st + 1].p);
      SPX_LAUNCH_CHECK();
    }
  }
  // reverse sweep
  SPX_CUDA(cudaMemcpyAsync(A.acc.p, A.lam.p, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  const TV cl[4] = {h / TV(6), h / TV(3), h / TV(3), h / TV(6)};  // weight of lambda in w_s
  const TV ca[4] = {TV(0.5) * h, TV(0.5) * h, h, TV(0)};         // weight of a_(s+1) in w_s
  for (int st = 3; st >= 0; --st) {
    k_comb<TV><<<g3, 256, 0, s>>>(n3, A.w.p, cl[st], A.lam.p, ca[st], st < 3 ? A.ap.p : nullptr);
    SPX_LAUNCH_CHECK();
    rhs_vjp(A.Y[st].p, A.Hs[st].p, A.w.p, A.a.p, gKu, gH0, 4 + st, s);
    k_add<TV><<<g3, 256, 0, s>>>(n3, A.acc.p, A.a.p);
    SPX_LAUNCH_CHECK();
    std::swap(A.a, A.ap);
  }
  SPX_CUDA(cudaMemcpyAsync(lam_out, A.acc.p, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
}

template <class TV, class TM>
void LLGCtx<TV, TM>::step_jvp(const TV* mn, const TV* dm, const double* dKu, const double dH0[3], double dt, TV* m_out,
                              TV* dm_out, cudaStream_t s) {
  adjoint_setup(s);
  LLGAdjoint<TV, TM>& A = adj;
  const int64_t n3 = 3 * N;
  const LocalPrm<TV> q = local_prm(*this);
  const TV h = static_cast<TV>(dt);
  const unsigned ge = grid_for(N, 256);
  SPX_CUDA(cudaMemcpyAsync(A.Y[0].p, mn, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  SPX_CUDA(cudaMemcpyAsync(A.dY[0].p, dm, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  // the stage inputs are copies, so m_out / dm_out may alias mn / dm
  SPX_CUDA(cudaMemcpyAsync(A.Y[3].p, mn, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  SPX_CUDA(cudaMemcpyAsync(A.lam.p, dm, n3 * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  const TV* mn0 = A.Y[3].p;
  const TV* dm0 = A.lam.p;
  const TV cn[4] = {TV(0.5) * h, TV(0.5) * h, h, TV(0)};
  const TV wa[4] = {TV(1), TV(2), TV(2), TV(0)};
  int cur = 0;
  for (int st = 0; st < 4; ++st) {
    TV* Y = A.Y[cur].p;
    TV* dY = A.dY[cur].p;
    if (use_demag) demag->potential(Y, s, false, st);
    launch_stage(args(Y, A.Hs[0].p, 0, use_demag), use_demag, s);
    if (use_demag) demag->potential(dY, s, false, 8 + st);
    StageArgs<TV, TM> la = args(dY, A.dH.p, 0, use_demag);
    la.H0 = nullptr;
    la.h0x = la.h0y = la.h0z = TV(0);
    launch_stage(la, use_demag, s);
    const int nxt = cur ^ 1;
    k_tan_stage<TV><<<ge, 256, 0, s>>>(N, mn0, dm0, Y, A.Hs[0].p, dY, A.dH.p, dKu,
                                       static_cast<TV>(dH0 ? dH0[0] : 0.0), static_cast<TV>(dH0 ? dH0[1] : 0.0),
                                       static_cast<TV>(dH0 ? dH0[2] : 0.0), q, st, cn[st], wa[st], h / TV(6),
                                       A.Y[nxt].p, A.dY[nxt].p, A.K.p, A.dK.p, m_out, dm_out);
    SPX_LAUNCH_CHECK();
    cur = nxt;
  }
}

template <class TV, class TM>
void LLGCtx<TV, TM>::set_ku_map(const double* Ku_nodes, cudaStream_t s) {
  SPX_CHECK(has_ani, "a Ku map needs the anisotropy axis given at creation");
  const double mu0 = 4e-7 * 3.141592653589793;
  std::vector<TV> pp(N), nn(3 * N);
  std::vector<double> dg = diag_lin_host;
  SPX_CUDA(cudaMemcpy(nn.data(), ani_n.p, 3 * N * sizeof(TV), cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < N; ++i) {
    const double pr = 2.0 * Ku_nodes[i] / (mu0 * prm.Ms);
    pp[i] = static_cast<TV>(pr);
    for (int c = 0; c < 3; ++c) dg[3 * i + c] += pr * static_cast<double>(nn[3 * i + c]) * nn[3 * i + c];
  }
  ani_p.upload(pp, s);
  std::vector<TV> d(dg.begin(), dg.end());
  diagK.upload(d, s);
  SPX_CUDA(cudaStreamSynchronize(s));
}

#define SPX_ADJ_INST(TV, TM)                                                                                    \
  template void LLGCtx<TV, TM>::adjoint_setup(cudaStream_t);                                                    \
  template void LLGCtx<TV, TM>::rhs_vjp(const TV*, const TV*, const TV*, TV*, double*, double*, int, cudaStream_t); \
  template void LLGCtx<TV, TM>::step_vjp(const TV*, double, const TV*, TV*, double*, double*, cudaStream_t);       \
  template void LLGCtx<TV, TM>::step_jvp(const TV*, const TV*, const double*, const double*, double, TV*, TV*,     \
                                         cudaStream_t);                                                          \
  template void LLGCtx<TV, TM>::set_ku_map(const double*, cudaStream_t);
SPX_ADJ_INST(double, double)
SPX_ADJ_INST(float, float)
SPX_ADJ_INST(double, float)
#undef SPX_ADJ_INST

}  // namespace spx
