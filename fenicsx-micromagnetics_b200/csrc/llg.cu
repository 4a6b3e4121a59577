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
// k_stage fuses, per node and in one pass over the shared SELL pattern: the exchange and
// DMI SpMVs on m and the demag gradient G phi / V_i (all in difference form, see fem.cuh),
// anisotropy, Zeeman, the LLG RHS and the RK4 stage combination.  The only other per-stage
// work is the demag potential (Div SpMV, two CG solves, boundary operator).
#include <algorithm>
#include <cmath>

#include "llg.cuh"

namespace spx {


template <class TV, class TM, bool DMI, bool DEMAG, bool ANI>
__global__ void __launch_bounds__(256) k_stage(StageArgs<TV, TM> a) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t sl = gw; sl < a.nslices; sl += nw) {
    const int64_t i = sl * 32 + lane;
    if (i >= a.n) continue;
    const int64_t base = a.sp[sl];
    const int width = static_cast<int>((a.sp[sl + 1] - base) >> 5);
    const TV mx = a.m[3 * i], my = a.m[3 * i + 1], mz = a.m[3 * i + 2];
    const TV pi = DEMAG ? a.phi[i] : TV(0);
    TV hx = 0, hy = 0, hz = 0;
    TV zx = 0, zy = 0, zz = 0;  // Zhang-Li (J . grad) m / V_i
    for (int k = 0; k < width; ++k) {
      const int64_t idx = base + ((int64_t)k << 5) + lane;
      const int64_t j = a.col[idx];
      const TV dx = a.m[3 * j] - mx, dy = a.m[3 * j + 1] - my, dz = a.m[3 * j + 2] - mz;
      const TV e = static_cast<TV>(a.Kex[idx]);
      hx += e * dx;
      hy += e * dy;
      hz += e * dz;
      if (a.Kz) {
        const TV kz = static_cast<TV>(a.Kz[idx]);
        zx += kz * dx;
        zy += kz * dy;
        zz += kz * dz;
      }
      if (DMI) {
        const TM* K = a.Kd + idx;
        const int64_t L = a.L;
        hx += static_cast<TV>(K[0]) * dx + static_cast<TV>(K[L]) * dy + static_cast<TV>(K[2 * L]) * dz;
        hy += static_cast<TV>(K[3 * L]) * dx + static_cast<TV>(K[4 * L]) * dy + static_cast<TV>(K[5 * L]) * dz;
        hz += static_cast<TV>(K[6 * L]) * dx + static_cast<TV>(K[7 * L]) * dy + static_cast<TV>(K[8 * L]) * dz;
      }
      if (DEMAG) {
        const TV p = a.phi[j] - pi;
        hx += static_cast<TV>(a.Gv[idx]) * p;
        hy += static_cast<TV>(a.Gv[a.L + idx]) * p;
        hz += static_cast<TV>(a.Gv[2 * a.L + idx]) * p;
      }
    }
    if (DMI) {
      const double* S = a.Ksum;
      const int64_t n = a.n;
      hx += static_cast<TV>(S[i]) * mx + static_cast<TV>(S[n + i]) * my + static_cast<TV>(S[2 * n + i]) * mz;
      hy += static_cast<TV>(S[3 * n + i]) * mx + static_cast<TV>(S[4 * n + i]) * my + static_cast<TV>(S[5 * n + i]) * mz;
      hz += static_cast<TV>(S[6 * n + i]) * mx + static_cast<TV>(S[7 * n + i]) * my + static_cast<TV>(S[8 * n + i]) * mz;
    }
    if (ANI) {
      const TV nx = a.ani_n[3 * i], ny = a.ani_n[3 * i + 1], nz = a.ani_n[3 * i + 2];
      const TV c = (a.ani_p ? a.ani_p[i] : a.ani_p0) * (mx * nx + my * ny + mz * nz);
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
    if (a.Ht) {
      hx += a.Ht[3 * i];
      hy += a.Ht[3 * i + 1];
      hz += a.Ht[3 * i + 2];
    }
    hx += a.htx;
    hy += a.hty;
    hz += a.htz;
    if (a.mode == 0) {
      a.out[3 * i] = hx;
      a.out[3 * i + 1] = hy;
      a.out[3 * i + 2] = hz;
      if (a.zout) {
        a.zout[3 * i] = zx;
        a.zout[3 * i + 1] = zy;
        a.zout[3 * i + 2] = zz;
      }
      continue;
    }
    const TV cx = my * hz - mz * hy, cy = mz * hx - mx * hz, cz = mx * hy - my * hx;
    const TV ccx = my * cz - mz * cy, ccy = mz * cx - mx * cz, ccz = mx * cy - my * cx;
    const TV s = a.stab * (TV(1) - (mx * mx + my * my + mz * mz));
    TV rx = a.pref * (a.precess * cx + a.alpha * ccx) + s * mx;
    TV ry = a.pref * (a.precess * cy + a.alpha * ccy) + s * my;
    TV rz = a.pref * (a.precess * cz + a.alpha * ccz) + s * mz;
    if (a.Kz) {  // - prefZ (stt_a m x z + stt_b m x (m x z))   (llg_stt_module_GPU.py:101-139)
      const TV qx = my * zz - mz * zy, qy = mz * zx - mx * zz, qz = mx * zy - my * zx;
      const TV qqx = my * qz - mz * qy, qqy = mz * qx - mx * qz, qqz = mx * qy - my * qx;
      rx -= a.prefZ * (a.stt_a * qx + a.stt_b * qqx);
      ry -= a.prefZ * (a.stt_a * qy + a.stt_b * qqy);
      rz -= a.prefZ * (a.stt_a * qz + a.stt_b * qqz);
    }
    if (a.sot_p) {  // + c_fl m x p + c_dl m x (m x p)   (llg_SOT_module_GPU.py:170-205)
      const TV px = a.sot_p[3 * i], py = a.sot_p[3 * i + 1], pz = a.sot_p[3 * i + 2];
      const TV qx = my * pz - mz * py, qy = mz * px - mx * pz, qz = mx * py - my * px;
      const TV qqx = my * qz - mz * qy, qqy = mz * qx - mx * qz, qqz = mx * qy - my * qx;
      rx += a.c_fl * qx + a.c_dl * qqx;
      ry += a.c_fl * qy + a.c_dl * qqy;
      rz += a.c_fl * qz + a.c_dl * qqz;
    }
    if (a.mode == 1) {
      a.out[3 * i] = rx;
      a.out[3 * i + 1] = ry;
      a.out[3 * i + 2] = rz;
      continue;
    }
    // RK4 stage update
    TV* A = a.acc + 3 * i;
    TV* M = a.mn + 3 * i;
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
template <class TV, class TM, bool DMI, bool ANI>
__global__ void __launch_bounds__(256) k_jv(StageArgs<TV, TM> a, const TV* __restrict__ Ms,
                                            const TV* __restrict__ Hm, const TV* __restrict__ v,
                                            TV* __restrict__ out, TV gamma, const TV* __restrict__ Zm) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t sl = gw; sl < a.nslices; sl += nw) {
    const int64_t i = sl * 32 + lane;
    if (i >= a.n) continue;
    const int64_t base = a.sp[sl];
    const int width = static_cast<int>((a.sp[sl + 1] - base) >> 5);
    const TV vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
    TV hvx = 0, hvy = 0, hvz = 0;
    TV jvx = 0, jvy = 0, jvz = 0;  // Z(v)
    for (int k = 0; k < width; ++k) {
      const int64_t idx = base + ((int64_t)k << 5) + lane;
      const int64_t j = a.col[idx];
      const TV x = v[3 * j] - vx, y = v[3 * j + 1] - vy, z = v[3 * j + 2] - vz;
      const TV e = static_cast<TV>(a.Kex[idx]);
      hvx += e * x; hvy += e * y; hvz += e * z;
      if (a.Kz) {
        const TV kz = static_cast<TV>(a.Kz[idx]);
        jvx += kz * x; jvy += kz * y; jvz += kz * z;
      }
      if (DMI) {
        const TM* K = a.Kd + idx;
        const int64_t L = a.L;
        hvx += static_cast<TV>(K[0]) * x + static_cast<TV>(K[L]) * y + static_cast<TV>(K[2 * L]) * z;
        hvy += static_cast<TV>(K[3 * L]) * x + static_cast<TV>(K[4 * L]) * y + static_cast<TV>(K[5 * L]) * z;
        hvz += static_cast<TV>(K[6 * L]) * x + static_cast<TV>(K[7 * L]) * y + static_cast<TV>(K[8 * L]) * z;
      }
    }
    if (DMI) {
      const double* S = a.Ksum;
      const int64_t n = a.n;
      hvx += static_cast<TV>(S[i]) * vx + static_cast<TV>(S[n + i]) * vy + static_cast<TV>(S[2 * n + i]) * vz;
      hvy += static_cast<TV>(S[3 * n + i]) * vx + static_cast<TV>(S[4 * n + i]) * vy + static_cast<TV>(S[5 * n + i]) * vz;
      hvz += static_cast<TV>(S[6 * n + i]) * vx + static_cast<TV>(S[7 * n + i]) * vy + static_cast<TV>(S[8 * n + i]) * vz;
    }
    if (ANI) {
      const TV nx = a.ani_n[3 * i], ny = a.ani_n[3 * i + 1], nz = a.ani_n[3 * i + 2];
      const TV c = (a.ani_p ? a.ani_p[i] : a.ani_p0) * (vx * nx + vy * ny + vz * nz);
      hvx += c * nx; hvy += c * ny; hvz += c * nz;
    }
    const TV mx = Ms[3 * i], my = Ms[3 * i + 1], mz = Ms[3 * i + 2];
    const TV hx = Hm[3 * i], hy = Hm[3 * i + 1], hz = Hm[3 * i + 2];
    const TV cvx = vy * hz - vz * hy, cvy = vz * hx - vx * hz, cvz = vx * hy - vy * hx;
    const TV cmx = my * hvz - mz * hvy, cmy = mz * hvx - mx * hvz, cmz = mx * hvy - my * hvx;
    const TV mdHm = mx * hx + my * hy + mz * hz;
    const TV mdHv = mx * hvx + my * hvy + mz * hvz;
    const TV vdHm = vx * hx + vy * hy + vz * hz;
    const TV mdv = mx * vx + my * vy + mz * vz;
    const TV mdmm = mx * mx + my * my + mz * mz;
    const TV common = vdHm + mdHv;
    const TV dampx = vx * mdHm - TV(2) * hx * mdv + mx * common - hvx * mdmm;
    const TV dampy = vy * mdHm - TV(2) * hy * mdv + my * common - hvy * mdmm;
    const TV dampz = vz * mdHm - TV(2) * hz * mdv + mz * common - hvz * mdmm;
    const TV coef = -gamma / (TV(1) + a.alpha * a.alpha);
    const TV sc = a.stab * (TV(1) - mdmm);
    TV ox = coef * (a.precess * (cvx + cmx) + a.alpha * dampx) + sc * vx - TV(2) * a.stab * mx * mdv;
    TV oy = coef * (a.precess * (cvy + cmy) + a.alpha * dampy) + sc * vy - TV(2) * a.stab * my * mdv;
    TV oz = coef * (a.precess * (cvz + cmz) + a.alpha * dampz) + sc * vz - TV(2) * a.stab * mz * mdv;
    if (a.Kz) {  // _JAC_VEC_STT_KERNEL (llg_stt_module_GPU.py:142-215), jm = Z(m_state), jv = Z(v)
      const TV jmx = Zm[3 * i], jmy = Zm[3 * i + 1], jmz = Zm[3 * i + 2];
      const TV mjx = my * jvz - mz * jvy, mjy = mz * jvx - mx * jvz, mjz = mx * jvy - my * jvx;
      const TV vjx = vy * jmz - vz * jmy, vjy = vz * jmx - vx * jmz, vjz = vx * jmy - vy * jmx;
      const TV MjV = mx * jvx + my * jvy + mz * jvz, VjM = vx * jmx + vy * jmy + vz * jmz;
      const TV MjM = mx * jmx + my * jmy + mz * jmz;
      const TV pa = -a.stt_a * a.prefZ, pb = -a.stt_b * a.prefZ;
      ox += pa * (mjx + vjx) + pb * (vx * MjM + mx * VjM + mx * MjV - jvx * mdmm - TV(2) * jmx * mdv);
      oy += pa * (mjy + vjy) + pb * (vy * MjM + my * VjM + my * MjV - jvy * mdmm - TV(2) * jmy * mdv);
      oz += pa * (mjz + vjz) + pb * (vz * MjM + mz * VjM + mz * MjV - jvz * mdmm - TV(2) * jmz * mdv);
    }
    if (a.sot_p) {  // _JAC_VEC_SOT_KERNEL (llg_SOT_module_GPU.py:208-275)
      const TV px = a.sot_p[3 * i], py = a.sot_p[3 * i + 1], pz = a.sot_p[3 * i + 2];
      const TV qx = my * pz - mz * py, qy = mz * px - mx * pz, qz = mx * py - my * px;
      const TV dx = vy * pz - vz * py, dy = vz * px - vx * pz, dz = vx * py - vy * px;
      ox += a.c_fl * dx + a.c_dl * ((vy * qz - vz * qy) + (my * dz - mz * dy));
      oy += a.c_fl * dy + a.c_dl * ((vz * qx - vx * qz) + (mz * dx - mx * dz));
      oz += a.c_fl * dz + a.c_dl * ((vx * qy - vy * qx) + (mx * dy - my * dx));
    }
    out[3 * i] = ox;
    out[3 * i + 1] = oy;
    out[3 * i + 2] = oz;
  }
}

// spin torques of the 3x3 block preconditioner: STT (G = Z(m_state), c3, c4:
// _PC_BUILD_INV3_STT_KERNEL, llg_stt_module_GPU.py:218-393) or SOT (column-wise local
// Jacobian with per-component diagonal, _PC_BUILD_INV3_SOT_KERNEL, llg_SOT_module_GPU.py:278-437)
struct PcTorque {
  const void* G;  // TV [3n] or null
  double c3, c4;
  const void* P;  // TV [3n] (SOT polarisation) or null
  double pref, alpha, precess, c_fl, c_dl;
};

// column c of the local SOT Jacobian: Jv_SOT with v = e_c and H_v = k e_c
__device__ __forceinline__ void sot_column(const double m[3], const double h[3], const double p[3], int c, double k,
                                           const PcTorque& t, double Stab, double out[3]) {
  double v[3] = {0.0, 0.0, 0.0}, hv[3] = {0.0, 0.0, 0.0};
  v[c] = 1.0;
  hv[c] = k;
  auto cross = [](const double a[3], const double b[3], double r[3]) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
  };
  double cv[3], cm[3], q[3], dq[3], vq[3], mdq[3];
  cross(v, h, cv);
  cross(m, hv, cm);
  const double mdH = m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
  const double mdHv = m[0] * hv[0] + m[1] * hv[1] + m[2] * hv[2];
  const double vdH = v[0] * h[0] + v[1] * h[1] + v[2] * h[2];
  const double mdv = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
  const double mdm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
  const double common = vdH + mdHv;
  cross(m, p, q);
  cross(v, p, dq);
  cross(v, q, vq);
  cross(m, dq, mdq);
  const double sc = Stab * (1.0 - mdm);
  for (int r = 0; r < 3; ++r) {
    const double damp = v[r] * mdH - 2.0 * h[r] * mdv + m[r] * common - hv[r] * mdm;
    out[r] = t.pref * (t.precess * (cv[r] + cm[r]) + t.alpha * damp) + t.c_fl * dq[r] + t.c_dl * (vq[r] + mdq[r]) +
             sc * v[r] - 2.0 * Stab * m[r] * mdv;
  }
}

template <class TV>
__global__ void k_pc_build(int64_t n, const TV* __restrict__ M, const TV* __restrict__ H, const TV* __restrict__ D,
                           int include_stab, int use_abs_kappa, double shift, double eps_reg, double det_eps,
                           double c1, double c2, double Stab, PcTorque tq, TV* __restrict__ inv) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double mx = M[3 * i], my = M[3 * i + 1], mz = M[3 * i + 2];
  const double hx = H[3 * i], hy = H[3 * i + 1], hz = H[3 * i + 2];
  const double dex = D[3 * i], dey = D[3 * i + 1], dez = D[3 * i + 2];
  if (tq.P) {  // SOT: columns of the local Jacobian, then the same inverse with its own det guard
    const TV* Pp = static_cast<const TV*>(tq.P);
    const double m3[3] = {mx, my, mz}, h3[3] = {hx, hy, hz};
    const double p3[3] = {static_cast<double>(Pp[3 * i]), static_cast<double>(Pp[3 * i + 1]),
                          static_cast<double>(Pp[3 * i + 2])};
    const double kd[3] = {use_abs_kappa ? fabs(dex) : dex, use_abs_kappa ? fabs(dey) : dey,
                          use_abs_kappa ? fabs(dez) : dez};
    double Jc[3][3];
    for (int c = 0; c < 3; ++c) sot_column(m3, h3, p3, c, kd[c], tq, Stab, Jc[c]);
    const double s = shift + eps_reg;
    double A[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) A[r][c] = (r == c ? s : 0.0) - Jc[c][r];
    double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                 A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    if (fabs(det) < det_eps) det += (det >= 0.0 ? 1.0 : -1.0) * det_eps;
    const double id = 1.0 / det;
    TV* o = inv + 9 * i;
    o[0] = static_cast<TV>((A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id);
    o[1] = static_cast<TV>(-(A[0][1] * A[2][2] - A[0][2] * A[2][1]) * id);
    o[2] = static_cast<TV>((A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id);
    o[3] = static_cast<TV>(-(A[1][0] * A[2][2] - A[1][2] * A[2][0]) * id);
    o[4] = static_cast<TV>((A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id);
    o[5] = static_cast<TV>(-(A[0][0] * A[1][2] - A[0][2] * A[1][0]) * id);
    o[6] = static_cast<TV>((A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id);
    o[7] = static_cast<TV>(-(A[0][0] * A[2][1] - A[0][1] * A[2][0]) * id);
    o[8] = static_cast<TV>((A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id);
    return;
  }
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
  if (tq.G) {  // STT: c3 [g]x-like terms and c4 B(g)
    const TV* Gp = static_cast<const TV*>(tq.G);
    const double gx = Gp[3 * i], gy = Gp[3 * i + 1], gz = Gp[3 * i + 2];
    const double mdG = mx * gx + my * gy + mz * gz;
    J[0][1] += tq.c3 * (-gz);
    J[0][2] += tq.c3 * gy;
    J[1][0] += tq.c3 * gz;
    J[1][2] += tq.c3 * (-gx);
    J[2][0] += tq.c3 * (-gy);
    J[2][1] += tq.c3 * gx;
    J[0][0] += tq.c4 * (mdG - gx * mx);
    J[1][1] += tq.c4 * (mdG - gy * my);
    J[2][2] += tq.c4 * (mdG - gz * mz);
    J[0][1] += tq.c4 * (mx * gy - 2.0 * gx * my);
    J[0][2] += tq.c4 * (mx * gz - 2.0 * gx * mz);
    J[1][0] += tq.c4 * (my * gx - 2.0 * gy * mx);
    J[1][2] += tq.c4 * (my * gz - 2.0 * gy * mz);
    J[2][0] += tq.c4 * (mz * gx - 2.0 * gz * mx);
    J[2][1] += tq.c4 * (mz * gy - 2.0 * gz * my);
  }
  const double s = shift + eps_reg;
  double A[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[r][c] = (r == c ? s : 0.0) - J[r][c];
  double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
               A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (fabs(det) < det_eps) det += ((det + det_eps) > 0.0 ? 1.0 : -1.0) * det_eps;
  const double id = 1.0 / det;
  TV* o = inv + 9 * i;
  o[0] = static_cast<TV>((A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id);
  o[1] = static_cast<TV>(-(A[0][1] * A[2][2] - A[0][2] * A[2][1]) * id);
  o[2] = static_cast<TV>((A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id);
  o[3] = static_cast<TV>(-(A[1][0] * A[2][2] - A[1][2] * A[2][0]) * id);
  o[4] = static_cast<TV>((A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id);
  o[5] = static_cast<TV>(-(A[0][0] * A[1][2] - A[0][2] * A[1][0]) * id);
  o[6] = static_cast<TV>((A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id);
  o[7] = static_cast<TV>(-(A[0][0] * A[2][1] - A[0][1] * A[2][0]) * id);
  o[8] = static_cast<TV>((A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id);
}

template <class TV>
__global__ void k_pc_apply(int64_t n, const TV* __restrict__ inv, const TV* __restrict__ x, TV* __restrict__ y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TV* o = inv + 9 * i;
  const TV a = x[3 * i], b = x[3 * i + 1], c = x[3 * i + 2];
  y[3 * i] = o[0] * a + o[1] * b + o[2] * c;
  y[3 * i + 1] = o[3] * a + o[4] * b + o[5] * c;
  y[3 * i + 2] = o[6] * a + o[7] * b + o[8] * c;
}

// sum_i w_i m_i . H_i  (w = nodal volume)
template <class TV>
__global__ void k_mdoth(int64_t n, const double* __restrict__ w, const TV* __restrict__ m, const TV* __restrict__ H,
                        double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += w[i] * (static_cast<double>(m[3 * i]) * H[3 * i] + static_cast<double>(m[3 * i + 1]) * H[3 * i + 1] +
                 static_cast<double>(m[3 * i + 2]) * H[3 * i + 2]);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = s;  // one partial per CTA, summed in a fixed order
}

// out[0] = sum of part[0..n) in a fixed order (one CTA), so the energy is run-to-run exact
__global__ void k_sum_parts(int n, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) out[0] = s;
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
template <class TV, class TM>
void LLGCtx<TV, TM>::create(DemagCtx<TV, TM>* dm, const double* X, int64_t N_, const int32_t* tets, int64_t E,
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
  std::vector<TM> v;
  sell_values<TM>(*hs, kex.data(), 1, true, nnz, 1.0, v);
  Kex.upload(v, s);
  has_dmi = (p.D_int != 0.0) || (p.D_bulk != 0.0);
  if (has_dmi) {
    SPX_CHECK(p.D_int == 0.0 || p.n_int != nullptr, "interfacial DMI needs the interface normal field");
    HostBoundary bhost;
    const HostBoundary* bh = nullptr;
    if (dm) bh = &dm->bd.host;
    else { build_boundary(X, N, tets, E, bhost); bh = &bhost; }
    std::vector<double> b9;
    dmi_blocks_scaled(X, tets, E, *fem, *bh, p.Ms, p.D_int, p.n_int, p.D_bulk, b9);
    std::vector<double> ks(9 * N, 0.0);
    for (int64_t i = 0; i < N; ++i) {
      for (int64_t k = fem->rowptr[i]; k < fem->rowptr[i + 1]; ++k) {
        for (int q = 0; q < 9; ++q) ks[q * N + i] += b9[9 * k + q];
        if (fem->col[k] == i)
          for (int c = 0; c < 3; ++c) diag[3 * i + c] += b9[9 * k + 4 * c];
      }
    }
    sell_values<TM>(*hs, b9.data(), 9, true, nnz, 1.0, v);
    Kd.upload(v, s);
    Ksum.upload(ks, s);
  }
  diag_lin_host = diag;
  if (has_dmi) {
    X_host.assign(X, X + 3 * N);
    tets_host.assign(tets, tets + 4 * E);
    if (p.n_int) n_int_host.assign(p.n_int, p.n_int + 3 * N);
  }
  has_ani = false;
  if (p.n_ani && (p.Ku != 0.0 || p.Ku_nodes)) {
    has_ani = true;
    std::vector<TV> nn(3 * N);
    for (int64_t i = 0; i < N; ++i) {
      const double a = p.n_ani[3 * i], b = p.n_ani[3 * i + 1], c = p.n_ani[3 * i + 2];
      const double r = std::max(std::sqrt(a * a + b * b + c * c), 1e-300);
      const double u[3] = {a / r, b / r, c / r};
      const double pr = 2.0 * (p.Ku_nodes ? p.Ku_nodes[i] : p.Ku) / (mu0 * p.Ms);
      for (int q = 0; q < 3; ++q) {
        nn[3 * i + q] = static_cast<TV>(u[q]);
        diag[3 * i + q] += pr * u[q] * u[q];
      }
    }
    ani_n.upload(nn, s);
    ani_p0 = 2.0 * p.Ku / (mu0 * p.Ms);
    if (p.Ku_nodes) {
      std::vector<TV> pp(N);
      for (int64_t i = 0; i < N; ++i) pp[i] = static_cast<TV>(2.0 * p.Ku_nodes[i] / (mu0 * p.Ms));
      ani_p.upload(pp, s);
    }
  }
  std::vector<TV> dg(diag.begin(), diag.end());
  diagK.upload(dg, s);
  if (p.H0_nodes) {
    std::vector<TV> h(p.H0_nodes, p.H0_nodes + 3 * N);
    H0.upload(h, s);
  }
  h0[0] = p.H0_uniform[0];
  h0[1] = p.H0_uniform[1];
  h0[2] = p.H0_uniform[2];
  has_stt = p.stt_dir != nullptr;
  has_sot = p.sot_p != nullptr;
  SPX_CHECK(!(has_stt && has_sot), "STT and SOT together are not supported (separate solvers in the reference)");
  if (has_stt) {
    // prefZhang = J P muB / (e Ms (1 + beta^2)) / (1 + alpha^2) / 1e-9 (llg_stt_module_GPU.py:571-578)
    const double e = 1.6021766e-19, muB = 9.27400915e-24;
    prefZ = p.stt_J * p.stt_P * muB / (e * p.Ms * (1.0 + p.stt_beta * p.stt_beta)) / (1.0 + p.alpha * p.alpha) / 1e-9;
    stt_a = p.stt_beta - p.alpha;
    stt_b = 1.0 + p.alpha * p.stt_beta;
    c3 = (p.stt_beta - p.alpha) * prefZ;
    c4 = -(1.0 + p.alpha * p.stt_beta) * prefZ;
    std::vector<double> kz;
    assemble_zhang_li(X, tets, E, *fem, p.stt_dir, kz);
    for (int64_t i = 0; i < N; ++i)
      for (int64_t k = fem->rowptr[i]; k < fem->rowptr[i + 1]; ++k) kz[k] /= fem->vol[i];
    sell_values<TM>(*hs, kz.data(), 1, true, nnz, 1.0, v);
    Kz.upload(v, s);
    Zm.alloc(3 * N);
    Zm.zero(s);
  }
  if (has_sot) set_sot(p.sot_Hdl, p.sot_Hfl, p.sot_p, s);
  use_demag = (dm != nullptr) && p.use_demag;
  m.alloc(3 * N); ms0.alloc(3 * N); ms1.alloc(3 * N); acc.alloc(3 * N);
  Mstate.alloc(3 * N); Hm.alloc(3 * N); pcinv.alloc(9 * N);
  red.alloc(2);
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class TV, class TM>
StageArgs<TV, TM> LLGCtx<TV, TM>::args(const TV* min, TV* out, int mode, bool with_demag) const {
  StageArgs<TV, TM> a{};
  a.n = N;
  a.nslices = P.nslices;
  a.sp = P.slice_ptr.p;
  a.col = P.col.p;
  a.L = P.len;
  a.Kex = Kex.p;
  a.Kd = has_dmi ? Kd.p : nullptr;
  a.Ksum = has_dmi ? Ksum.p : nullptr;
  a.Gv = with_demag ? demag->Gv.p : nullptr;
  a.phi = with_demag ? demag->phi.p : nullptr;
  a.ani_n = has_ani ? ani_n.p : nullptr;
  a.ani_p = (has_ani && ani_p.n) ? ani_p.p : nullptr;
  a.ani_p0 = static_cast<TV>(ani_p0);
  a.H0 = H0.n ? H0.p : nullptr;
  a.h0x = static_cast<TV>(h0[0]);
  a.h0y = static_cast<TV>(h0[1]);
  a.h0z = static_cast<TV>(h0[2]);
  a.Ht = ht_nodes.n ? ht_nodes.p : nullptr;
  a.htx = static_cast<TV>(ht[0]);
  a.hty = static_cast<TV>(ht[1]);
  a.htz = static_cast<TV>(ht[2]);
  a.m = min;
  a.out = out;
  a.pref = static_cast<TV>(pref);
  a.alpha = static_cast<TV>(prm.alpha);
  a.precess = static_cast<TV>(prm.do_precess);
  a.stab = static_cast<TV>(stab);
  a.mode = mode;
  a.Kz = has_stt ? Kz.p : nullptr;
  a.zout = nullptr;
  a.prefZ = static_cast<TV>(prefZ);
  a.stt_a = static_cast<TV>(stt_a);
  a.stt_b = static_cast<TV>(stt_b);
  a.sot_p = has_sot ? sotp.p : nullptr;
  a.c_fl = static_cast<TV>(c_fl);
  a.c_dl = static_cast<TV>(c_dl);
  return a;
}

template <class TV, class TM>
void LLGCtx<TV, TM>::launch_stage(const StageArgs<TV, TM>& a, bool with_demag, cudaStream_t s) const {
  const unsigned g = grid_for(a.nslices * 32, 256);
  const bool d = has_dmi, an = has_ani;
#define SPX_STAGE(DM, DE, AN) k_stage<TV, TM, DM, DE, AN><<<g, 256, 0, s>>>(a)
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

template <class TV, class TM>
void LLGCtx<TV, TM>::heff(const TV* min, TV* Hout, bool with_demag, cudaStream_t s) {
  const bool dm = with_demag && use_demag;
  if (dm) demag->potential(min, s, true);
  launch_stage(args(min, Hout, 0, dm), dm, s);
}

template <class TV, class TM>
void LLGCtx<TV, TM>::rhs(const TV* min, TV* out, cudaStream_t s) {
  if (use_demag) demag->potential(min, s, true);
  launch_stage(args(min, out, 1, use_demag), use_demag, s);
  ++rhs_evals;
}

template <class TV, class TM>
LLGCtx<TV, TM>::~LLGCtx() {
  graph_reset();
  if (gstream) cudaStreamDestroy(gstream);
}

template <class TV, class TM>
void LLGCtx<TV, TM>::graph_reset() {
  for (auto& g : gexec)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  graph_ok = false;
}

template <class TV, class TM>
void LLGCtx<TV, TM>::step_rk4(double dt, int64_t nsteps, cudaStream_t s) {
  const bool profiling = use_demag && demag->prof.on;
  for (int64_t it = 0; it < nsteps; ++it) {
    if (!graph_on || profiling) {
      step_once(dt, s);
      continue;
    }
    const int64_t ep = use_demag ? demag->epoch : 0;
    if (graph_ok && (dt != gdt || ep != gepoch)) graph_reset();
    if (!graph_ok) {
      if (gwarm < CG_HIST) {  // fill the extrapolation rings (and every lazily allocated buffer) first
        step_once(dt, s);
        ++gwarm;
        continue;
      }
      if (!gstream) SPX_CUDA(cudaStreamCreateWithFlags(&gstream, cudaStreamNonBlocking));
      const int64_t st0 = steps, re0 = rhs_evals, la0 = launches;
      try {
        for (int p = 0; p < CG_HIST; ++p) {
          cudaGraph_t g = nullptr;
          SPX_CUDA(cudaStreamBeginCapture(gstream, cudaStreamCaptureModeThreadLocal));
          try {
            step_once(dt, gstream);
          } catch (...) {
            cudaStreamEndCapture(gstream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
          }
          SPX_CUDA(cudaStreamEndCapture(gstream, &g));
          const cudaError_t e = cudaGraphInstantiate(&gexec[p], g, 0);
          cudaGraphDestroy(g);
          SPX_CUDA(e);
        }
      } catch (const Error& e) {
        // capture not possible here: keep stepping without graphs
        graph_reset();
        graph_on = false;
        graph_error = e.what();
        cudaGetLastError();
        steps = st0; rhs_evals = re0; launches = la0;
        step_once(dt, s);
        continue;
      }
      // the CG_HIST captures advanced the rings by one period: back to the same phase
      launches = la0;
      steps = st0;
      rhs_evals = re0;
      graph_ok = true;
      gdt = dt;
      gphase = 0;
      gepoch = use_demag ? demag->epoch : 0;
    }
    SPX_CUDA(cudaGraphLaunch(gexec[gphase], s));
    gphase = (gphase + 1) % CG_HIST;
    if (use_demag) demag->replay_step_advance();
    ++graph_replays;
    ++steps;
    rhs_evals += 4;
    launches += 4;
  }
}

template <class TV, class TM>
void LLGCtx<TV, TM>::step_once(double dt, cudaStream_t s, const double* htu, const TV* htn) {
  const TV h = static_cast<TV>(dt);
  for (int64_t it = 0; it < 1; ++it) {
    const TV* in[4] = {m.p, ms0.p, ms1.p, ms0.p};
    TV* out[4] = {ms0.p, ms1.p, ms0.p, nullptr};
    const TV cnext[4] = {TV(0.5) * h, TV(0.5) * h, h, TV(0)};
    const TV wacc[4] = {TV(1), TV(2), TV(2), TV(0)};
    for (int st = 0; st < 4; ++st) {
      if (use_demag) demag->potential(in[st], s, false, st);
      StageArgs<TV, TM> a = args(in[st], out[st], 2, use_demag);
      a.mn = m.p;
      a.acc = acc.p;
      a.stage = st;
      a.c_next = cnext[st];
      a.w_acc = wacc[st];
      a.dt6 = h / TV(6);
      if (htu || htn) {  // per-stage time field replaces the current-time one
        a.htx = htu ? static_cast<TV>(htu[3 * st]) : TV(0);
        a.hty = htu ? static_cast<TV>(htu[3 * st + 1]) : TV(0);
        a.htz = htu ? static_cast<TV>(htu[3 * st + 2]) : TV(0);
        a.Ht = htn ? htn + 3 * N * st : nullptr;
      }
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

template <class TV, class TM>
void LLGCtx<TV, TM>::update_jac_state(const TV* min, cudaStream_t s) {
  SPX_CUDA(cudaMemcpyAsync(Mstate.p, min, 3 * N * sizeof(TV), cudaMemcpyDeviceToDevice, s));
  StageArgs<TV, TM> a = args(Mstate.p, Hm.p, 0, false);
  if (has_stt) a.zout = Zm.p;
  launch_stage(a, false, s);
}

template <class TV, class TM>
void LLGCtx<TV, TM>::jv(const TV* v, TV* out, cudaStream_t s) {
  StageArgs<TV, TM> a = args(Mstate.p, out, 0, false);
  const unsigned g = grid_for(a.nslices * 32, 256);
  const TV gam = static_cast<TV>(prm.gamma);
  const TV* zm = has_stt ? Zm.p : nullptr;
  if (has_dmi && has_ani) k_jv<TV, TM, true, true><<<g, 256, 0, s>>>(a, Mstate.p, Hm.p, v, out, gam, zm);
  else if (has_dmi) k_jv<TV, TM, true, false><<<g, 256, 0, s>>>(a, Mstate.p, Hm.p, v, out, gam, zm);
  else if (has_ani) k_jv<TV, TM, false, true><<<g, 256, 0, s>>>(a, Mstate.p, Hm.p, v, out, gam, zm);
  else k_jv<TV, TM, false, false><<<g, 256, 0, s>>>(a, Mstate.p, Hm.p, v, out, gam, zm);
  SPX_LAUNCH_CHECK();
}

template <class TV, class TM>
void LLGCtx<TV, TM>::pc_build(double shift, int include_stab, int use_abs_kappa, cudaStream_t s) {
  PcTorque tq{};
  if (has_stt) {
    tq.G = Zm.p;
    tq.c3 = c3;
    tq.c4 = c4;
  }
  if (has_sot) {
    tq.P = sotp.p;
    tq.pref = pref;
    tq.alpha = prm.alpha;
    tq.precess = prm.do_precess;
    tq.c_fl = c_fl;
    tq.c_dl = c_dl;
  }
  k_pc_build<TV><<<grid_for(N, 256), 256, 0, s>>>(N, Mstate.p, Hm.p, diagK.p, include_stab, use_abs_kappa, shift,
                                                  1e-14, 1e-30, c1, c2, stab, tq, pcinv.p);
  SPX_LAUNCH_CHECK();
  pc_ready = true;
}

template <class TV, class TM>
void LLGCtx<TV, TM>::zhang_li(const TV* min, TV* out, cudaStream_t s) {
  SPX_CHECK(has_stt, "no spin-transfer torque configured");
  DevBuf<TV> tmp(3 * N);
  StageArgs<TV, TM> a = args(min, tmp.p, 0, false);
  a.zout = out;
  launch_stage(a, false, s);
  SPX_CUDA(cudaStreamSynchronize(s));
}

template <class TV, class TM>
void LLGCtx<TV, TM>::set_sot(double Hdl, double Hfl, const double* p_nodes, cudaStream_t s) {
  // c_fl = -gamma (H_fl - alpha H_dl) / (1 + alpha^2), c_dl = -gamma (H_dl + alpha H_fl) / (1 + alpha^2)
  // (llg_SOT_module_GPU.py:814-817)
  prm.sot_Hdl = Hdl;
  prm.sot_Hfl = Hfl;
  const double den = 1.0 + prm.alpha * prm.alpha;
  c_fl = -prm.gamma * (Hfl - prm.alpha * Hdl) / den;
  c_dl = -prm.gamma * (Hdl + prm.alpha * Hfl) / den;
  if (p_nodes) {
    std::vector<TV> pp(3 * N);
    for (int64_t i = 0; i < N; ++i) {
      const double a = p_nodes[3 * i], b = p_nodes[3 * i + 1], c = p_nodes[3 * i + 2];
      const double r = std::sqrt(a * a + b * b + c * c);
      const double sc = r > 0.0 ? 1.0 / r : 1.0;
      pp[3 * i] = static_cast<TV>(a * sc);
      pp[3 * i + 1] = static_cast<TV>(b * sc);
      pp[3 * i + 2] = static_cast<TV>(c * sc);
    }
    sotp.upload(pp, s);
    has_sot = true;
  }
  SPX_CHECK(has_sot, "SOT needs a polarisation field");
}

template <class TV, class TM>
void LLGCtx<TV, TM>::pc_apply(const TV* x, TV* y, cudaStream_t s) {
  if (!pc_ready) {
    SPX_CUDA(cudaMemcpyAsync(y, x, 3 * N * sizeof(TV), cudaMemcpyDeviceToDevice, s));
    return;
  }
  k_pc_apply<TV><<<grid_for(N, 256), 256, 0, s>>>(N, pcinv.p, x, y);
  SPX_LAUNCH_CHECK();
}

template struct LLGCtx<double, double>;
template struct LLGCtx<float, float>;
template struct LLGCtx<double, float>;

template <class TV, class TM>
double demag_energy(DemagCtx<TV, TM>& d, const TV* m, const TV* H, cudaStream_t s) {
  const unsigned grid = std::max(1u, std::min<unsigned>(grid_for(d.N, 256), 1184));
  DevBuf<double> r(grid + 1);
  k_mdoth<TV><<<grid, 256, 0, s>>>(d.N, d.vol.p, m, H, r.p);
  SPX_LAUNCH_CHECK();
  k_sum_parts<<<1, 256, 0, s>>>(static_cast<int>(grid), r.p, r.p + grid);
  SPX_LAUNCH_CHECK();
  double h = 0.0;
  SPX_CUDA(cudaMemcpyAsync(&h, r.p + grid, sizeof(double), cudaMemcpyDeviceToHost, s));
  SPX_CUDA(cudaStreamSynchronize(s));
  return -0.5 * d.mu0 * d.Ms * h / 1e27;
}
template double demag_energy<double, double>(DemagCtx<double, double>&, const double*, const double*, cudaStream_t);
template double demag_energy<float, float>(DemagCtx<float, float>&, const float*, const float*, cudaStream_t);
template double demag_energy<double, float>(DemagCtx<double, float>&, const double*, const double*, cudaStream_t);

}  // namespace spx
