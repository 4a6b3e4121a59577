// Host-side (native) set-up: boundary extraction, P1 FEM assembly, SELL-32
// conversion and the cluster tree.  These run once per mesh; the reference does
// the same work with DOLFINx on the host (gpu/fields/Demag_Lindholm_GPU.py:188-281,
// 554-567) and in Python (gpu/fields/Demag_Lindholm.py:177-285, tree.py:41-96).
#include <algorithm>
#include <array>
#include <cmath>
#include <numeric>

#include "spx_internal.cuh"

namespace spx {

namespace {

inline void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double norm3(const double* a) { return std::sqrt(dot3(a, a)); }

// Lindholm_kernel.py:30-48 (solid angle of (p0,p1,p2) seen from x0)
double solid_angle(const double* x0, const double* p0, const double* p1, const double* p2) {
  const double tiny = 1e-300;
  double r0[3], r1[3], r2[3];
  for (int k = 0; k < 3; ++k) {
    r0[k] = p0[k] - x0[k];
    r1[k] = p1[k] - x0[k];
    r2[k] = p2[k] - x0[k];
  }
  const double n0 = norm3(r0) + tiny, n1 = norm3(r1) + tiny, n2 = norm3(r2) + tiny;
  const double det = r0[0] * (r1[1] * r2[2] - r1[2] * r2[1]) - r0[1] * (r1[0] * r2[2] - r1[2] * r2[0]) +
                     r0[2] * (r1[0] * r2[1] - r1[1] * r2[0]);
  const double d01 = dot3(r0, r1), d12 = dot3(r1, r2), d20 = dot3(r2, r0);
  const double denom = n0 * n1 * n2 + d01 * n2 + d12 * n0 + d20 * n1;
  return 2.0 * std::atan2(det, denom);
}

// barycentric gradients g[4][3] and volume of a tet
void tet_grads(const double* X, const int32_t* t, double g[4][3], double* vol) {
  const double* x0 = X + 3 * (int64_t)t[0];
  double M[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) M[r][c] = X[3 * (int64_t)t[r + 1] + c] - x0[c];
  const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                     M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                     M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
  double inv[3][3];
  inv[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
  inv[0][1] = -(M[0][1] * M[2][2] - M[0][2] * M[2][1]) / det;
  inv[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
  inv[1][0] = -(M[1][0] * M[2][2] - M[1][2] * M[2][0]) / det;
  inv[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
  inv[1][2] = -(M[0][0] * M[1][2] - M[0][2] * M[1][0]) / det;
  inv[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det;
  inv[2][1] = -(M[0][0] * M[2][1] - M[0][1] * M[2][0]) / det;
  inv[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
  // grad lambda_k (k=1..3), component c = inv[c][k-1]
  for (int k = 1; k < 4; ++k)
    for (int c = 0; c < 3; ++c) g[k][c] = inv[c][k - 1];
  for (int c = 0; c < 3; ++c) g[0][c] = -(g[1][c] + g[2][c] + g[3][c]);
  *vol = std::fabs(det) / 6.0;
}

}  // namespace

void build_boundary(const double* X, int64_t N, const int32_t* tets, int64_t E, HostBoundary& out) {
  static const int FL[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  struct Face {
    int32_t v[3];
    int64_t cell;
  };
  std::vector<Face> faces(static_cast<size_t>(4 * E));
  for (int64_t e = 0; e < E; ++e) {
    for (int f = 0; f < 4; ++f) {
      Face& F = faces[4 * e + f];
      int32_t a = tets[4 * e + FL[f][0]], b = tets[4 * e + FL[f][1]], c = tets[4 * e + FL[f][2]];
      if (a > b) std::swap(a, b);
      if (b > c) std::swap(b, c);
      if (a > b) std::swap(a, b);
      F.v[0] = a; F.v[1] = b; F.v[2] = c;
      F.cell = e;
    }
  }
  std::sort(faces.begin(), faces.end(), [](const Face& x, const Face& y) {
    if (x.v[0] != y.v[0]) return x.v[0] < y.v[0];
    if (x.v[1] != y.v[1]) return x.v[1] < y.v[1];
    if (x.v[2] != y.v[2]) return x.v[2] < y.v[2];
    return x.cell < y.cell;
  });
  std::vector<std::array<int32_t, 3>> tris;
  std::vector<std::array<double, 3>> normals;
  const size_t F = faces.size();
  for (size_t i = 0; i < F;) {
    size_t j = i + 1;
    while (j < F && faces[j].v[0] == faces[i].v[0] && faces[j].v[1] == faces[i].v[1] &&
           faces[j].v[2] == faces[i].v[2])
      ++j;
    if (j - i == 1) {
      int32_t v0 = faces[i].v[0], v1 = faces[i].v[1], v2 = faces[i].v[2];
      const double *p0 = X + 3 * (int64_t)v0, *p1 = X + 3 * (int64_t)v1, *p2 = X + 3 * (int64_t)v2;
      double e1[3], e2[3], n[3];
      for (int k = 0; k < 3; ++k) { e1[k] = p1[k] - p0[k]; e2[k] = p2[k] - p0[k]; }
      cross3(e1, e2, n);
      const double nn = norm3(n);
      if (nn != 0.0) {
        for (int k = 0; k < 3; ++k) n[k] /= nn;
        const int64_t cell = faces[i].cell;
        double cc[3] = {0, 0, 0}, fc[3];
        for (int q = 0; q < 4; ++q)
          for (int k = 0; k < 3; ++k) cc[k] += X[3 * (int64_t)tets[4 * cell + q] + k];
        for (int k = 0; k < 3; ++k) {
          cc[k] /= 4.0;
          fc[k] = (p0[k] + p1[k] + p2[k]) / 3.0;
        }
        double d[3] = {fc[0] - cc[0], fc[1] - cc[1], fc[2] - cc[2]};
        if (dot3(d, n) < 0.0) {
          std::swap(v1, v2);
          const double *q1 = X + 3 * (int64_t)v1, *q2 = X + 3 * (int64_t)v2;
          for (int k = 0; k < 3; ++k) { e1[k] = q1[k] - p0[k]; e2[k] = q2[k] - p0[k]; }
          cross3(e1, e2, n);
          const double nn2 = norm3(n) + 1e-30;
          for (int k = 0; k < 3; ++k) n[k] /= nn2;
        }
        tris.push_back({v0, v1, v2});
        normals.push_back({n[0], n[1], n[2]});
      }
    }
    i = j;
  }
  const int64_t Nt = static_cast<int64_t>(tris.size());
  std::vector<int32_t> bmap(static_cast<size_t>(N), -1);
  std::vector<char> isb(static_cast<size_t>(N), 0);
  for (auto& t : tris)
    for (int k = 0; k < 3; ++k) isb[t[k]] = 1;
  out.bverts.clear();
  for (int64_t v = 0; v < N; ++v)
    if (isb[v]) { bmap[v] = static_cast<int32_t>(out.bverts.size()); out.bverts.push_back(static_cast<int32_t>(v)); }
  const int64_t Nb = static_cast<int64_t>(out.bverts.size());
  out.N = N; out.Nb = Nb; out.Nt = Nt;
  out.Xb.resize(3 * Nb);
  for (int64_t i = 0; i < Nb; ++i)
    for (int k = 0; k < 3; ++k) out.Xb[3 * i + k] = X[3 * (int64_t)out.bverts[i] + k];
  out.tris.resize(3 * Nt); out.tri_lid.resize(3 * Nt); out.tri_pts.resize(9 * Nt);
  out.ntri.resize(3 * Nt); out.area.resize(Nt); out.s_edge.resize(3 * Nt);
  out.eta.resize(9 * Nt); out.gamma.resize(9 * Nt);
  for (int64_t t = 0; t < Nt; ++t) {
    double P[3][3];
    for (int a = 0; a < 3; ++a) {
      out.tris[3 * t + a] = tris[t][a];
      out.tri_lid[3 * t + a] = bmap[tris[t][a]];
      for (int k = 0; k < 3; ++k) { P[a][k] = X[3 * (int64_t)tris[t][a] + k]; out.tri_pts[9 * t + 3 * a + k] = P[a][k]; }
    }
    for (int k = 0; k < 3; ++k) out.ntri[3 * t + k] = normals[t][k];
    double e[3][3], c[3];
    for (int k = 0; k < 3; ++k) {
      e[0][k] = P[1][k] - P[0][k];
      e[1][k] = P[2][k] - P[1][k];
      e[2][k] = P[0][k] - P[2][k];
    }
    double d20[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
    cross3(e[0], d20, c);
    out.area[t] = 0.5 * norm3(c);
    double xi[3][3];
    for (int a = 0; a < 3; ++a) {
      const double s = norm3(e[a]) + 1e-30;
      out.s_edge[3 * t + a] = s;
      for (int k = 0; k < 3; ++k) xi[a][k] = e[a][k] / s;
    }
    for (int a = 0; a < 3; ++a) {
      double et[3];
      cross3(normals[t].data(), xi[a], et);
      for (int k = 0; k < 3; ++k) out.eta[9 * t + 3 * a + k] = et[k];
    }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out.gamma[9 * t + 3 * i + j] = dot3(xi[(i + 1) % 3], xi[j]);
  }
  // omega_sum (Demag_Lindholm.py:265-283)
  out.omega_sum.assign(Nb, 0.0);
  for (int64_t e = 0; e < E; ++e) {
    const int32_t* vs = tets + 4 * e;
    for (int j = 0; j < 4; ++j) {
      const int32_t lid = bmap[vs[j]];
      if (lid < 0) continue;
      out.omega_sum[lid] += std::fabs(solid_angle(X + 3 * (int64_t)vs[j], X + 3 * (int64_t)vs[(j + 1) % 4],
                                                  X + 3 * (int64_t)vs[(j + 2) % 4], X + 3 * (int64_t)vs[(j + 3) % 4]));
    }
  }
}

void assemble_fem(const double* X, int64_t N, const int32_t* tets, int64_t E, HostFem& out) {
  out.N = N; out.E = E;
  // node -> tets adjacency
  std::vector<int64_t> nptr(N + 1, 0);
  for (int64_t e = 0; e < 4 * E; ++e) nptr[tets[e] + 1]++;
  for (int64_t i = 0; i < N; ++i) nptr[i + 1] += nptr[i];
  std::vector<int64_t> ntet(nptr[N]);
  {
    std::vector<int64_t> cur(nptr.begin(), nptr.end() - 1);
    for (int64_t e = 0; e < E; ++e)
      for (int q = 0; q < 4; ++q) ntet[cur[tets[4 * e + q]]++] = e;
  }
  out.rowptr.assign(N + 1, 0);
  std::vector<std::vector<int32_t>> rows(static_cast<size_t>(N));
  std::vector<int32_t> buf;
  for (int64_t i = 0; i < N; ++i) {
    buf.clear();
    for (int64_t k = nptr[i]; k < nptr[i + 1]; ++k)
      for (int q = 0; q < 4; ++q) buf.push_back(tets[4 * ntet[k] + q]);
    std::sort(buf.begin(), buf.end());
    buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
    rows[i] = buf;
    out.rowptr[i + 1] = out.rowptr[i] + static_cast<int64_t>(buf.size());
  }
  const int64_t nnz = out.rowptr[N];
  out.col.resize(nnz);
  for (int64_t i = 0; i < N; ++i) std::copy(rows[i].begin(), rows[i].end(), out.col.begin() + out.rowptr[i]);
  rows.clear();
  rows.shrink_to_fit();
  out.A.assign(nnz, 0.0);
  out.Div.assign(3 * nnz, 0.0);
  out.G.assign(3 * nnz, 0.0);
  out.vol.assign(N, 0.0);
  auto find = [&](int32_t i, int32_t j) -> int64_t {
    const int32_t* b = out.col.data() + out.rowptr[i];
    const int32_t* e = out.col.data() + out.rowptr[i + 1];
    return out.rowptr[i] + (std::lower_bound(b, e, j) - b);
  };
  for (int64_t e = 0; e < E; ++e) {
    const int32_t* t = tets + 4 * e;
    double g[4][3], vol;
    tet_grads(X, t, g, &vol);
    for (int a = 0; a < 4; ++a) {
      out.vol[t[a]] += vol / 4.0;
      for (int b = 0; b < 4; ++b) {
        const int64_t k = find(t[a], t[b]);
        out.A[k] += vol * (g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2]);
        for (int c = 0; c < 3; ++c) {
          out.Div[3 * k + c] += vol / 4.0 * g[a][c];   // row node a, column node b, component c
          out.G[3 * k + c] -= vol / 4.0 * g[b][c];     // row node a (component c), column node b
        }
      }
    }
  }
}

// Zhang-Li advection operator (gpu/solvers/llg_stt_module_GPU.py:402-429): the P1 form
// int (J . grad u) v dx with the nodal (P1) current-direction field J, on the node pattern,
// unscaled.  Per tetrahedron grad(phi_b) is constant and int phi_a phi_k = vol/20 (1 + d_ak).
void assemble_zhang_li(const double* X, const int32_t* tets, int64_t E, const HostFem& fem, const double* J,
                       std::vector<double>& K) {
  const int64_t nnz = fem.rowptr[fem.N];
  K.assign(nnz, 0.0);
  auto find = [&](int32_t i, int32_t j) -> int64_t {
    const int32_t* b = fem.col.data() + fem.rowptr[i];
    const int32_t* e = fem.col.data() + fem.rowptr[i + 1];
    return fem.rowptr[i] + (std::lower_bound(b, e, j) - b);
  };
  for (int64_t e = 0; e < E; ++e) {
    const int32_t* t = tets + 4 * e;
    double g[4][3], vol;
    tet_grads(X, t, g, &vol);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        double sum = 0.0;
        for (int k = 0; k < 4; ++k) {
          const double* Jk = J + 3 * static_cast<int64_t>(t[k]);
          sum += vol / 20.0 * (a == k ? 2.0 : 1.0) * (Jk[0] * g[b][0] + Jk[1] * g[b][1] + Jk[2] * g[b][2]);
        }
        K[find(t[a], t[b])] += sum;
      }
  }
}

void assemble_dmi_interfacial(const double* X, const int32_t* tets, int64_t E, const HostFem& fem,
                              const HostBoundary& bd, const double* nN, std::vector<double>& B9) {
  const int64_t nnz = fem.rowptr[fem.N];
  B9.assign(9 * nnz, 0.0);
  auto find = [&](int32_t i, int32_t j) -> int64_t {
    const int32_t* b = fem.col.data() + fem.rowptr[i];
    const int32_t* e = fem.col.data() + fem.rowptr[i + 1];
    const int32_t* p = std::lower_bound(b, e, j);
    if (p == e || *p != j) throw Error(ERR_INTERNAL, "DMI entry outside the P1 pattern");
    return fem.rowptr[i] + (p - b);
  };
  for (int64_t e = 0; e < E; ++e) {
    const int32_t* t = tets + 4 * e;
    double g[4][3], vol;
    tet_grads(X, t, g, &vol);
    double M[4][4];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) M[a][b] = vol / 20.0 * (a == b ? 2.0 : 1.0);
    double Mn[4][3] = {};
    for (int a = 0; a < 4; ++a)
      for (int k = 0; k < 4; ++k)
        for (int c = 0; c < 3; ++c) Mn[a][c] += M[a][k] * nN[3 * (int64_t)t[k] + c];
    double dn[3][3] = {};  // d_c n_d
    for (int k = 0; k < 4; ++k)
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) dn[c][d] += nN[3 * (int64_t)t[k] + d] * g[k][c];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        const int64_t k = find(t[a], t[b]);
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d)
            B9[9 * k + 3 * c + d] += g[b][d] * Mn[a][c] - dn[c][d] * M[a][b] - g[b][c] * Mn[a][d];
      }
  }
  // 0.5 int_ds ((n x nu) x u) . v = 0.5 int phi_a phi_b (nu_c n_d - n_c nu_d)
  for (int64_t f = 0; f < bd.Nt; ++f) {
    const int32_t* tv = bd.tris.data() + 3 * f;
    const double* nu = bd.ntri.data() + 3 * f;
    const double A = bd.area[f];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double nab[3] = {0, 0, 0};
        for (int q = 0; q < 3; ++q) {
          int cnt[3] = {0, 0, 0};
          cnt[a]++; cnt[b]++; cnt[q]++;
          auto fac = [](int x) { return x == 3 ? 6.0 : (x == 2 ? 2.0 : 1.0); };
          const double w = 2.0 * A * fac(cnt[0]) * fac(cnt[1]) * fac(cnt[2]) / 120.0;
          for (int d = 0; d < 3; ++d) nab[d] += w * nN[3 * (int64_t)tv[q] + d];
        }
        const int64_t k = find(tv[a], tv[b]);
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) B9[9 * k + 3 * c + d] += 0.5 * (nu[c] * nab[d] - nab[c] * nu[d]);
      }
  }
}

// Bulk DMI operator restating gpu/fields/DMI_Bulk_GPU.py:52-66 (unscaled):
//   K u . v = - int curl(u) . v dx + 0.5 int_ds (nu x u) . v,
// as 3x3 blocks [c][d] (row component c of phi_a, column component d of phi_b) on the scalar
// pattern: volume part - sum_k eps_{c k d} int phi_a d_k phi_b, boundary part
// 0.5 sum_k eps_{c k d} nu_k int_F phi_a phi_b.
void assemble_dmi_bulk(const double* X, const int32_t* tets, int64_t E, const HostFem& fem, const HostBoundary& bd,
                       std::vector<double>& B9) {
  const int64_t nnz = fem.rowptr[fem.N];
  B9.assign(9 * nnz, 0.0);
  auto find = [&](int32_t i, int32_t j) -> int64_t {
    const int32_t* b = fem.col.data() + fem.rowptr[i];
    const int32_t* e = fem.col.data() + fem.rowptr[i + 1];
    const int32_t* p = std::lower_bound(b, e, j);
    if (p == e || *p != j) throw Error(ERR_INTERNAL, "DMI entry outside the P1 pattern");
    return fem.rowptr[i] + (p - b);
  };
  // eps_{c k d} w_k as a 3x3 matrix [c][d] (the cross product e_c . (w x e_d))
  auto cross_mat = [](const double w[3], double C[3][3]) {
    C[0][0] = 0.0;   C[0][1] = -w[2]; C[0][2] = w[1];
    C[1][0] = w[2];  C[1][1] = 0.0;   C[1][2] = -w[0];
    C[2][0] = -w[1]; C[2][1] = w[0];  C[2][2] = 0.0;
  };
  for (int64_t e = 0; e < E; ++e) {
    const int32_t* t = tets + 4 * e;
    double g[4][3], vol;
    tet_grads(X, t, g, &vol);
    for (int b = 0; b < 4; ++b) {
      double C[3][3];
      cross_mat(g[b], C);  // (curl(phi_b e_d))_c = eps_{c k d} d_k phi_b
      for (int a = 0; a < 4; ++a) {
        const int64_t k = find(t[a], t[b]);
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) B9[9 * k + 3 * c + d] -= (vol / 4.0) * C[c][d];
      }
    }
  }
  for (int64_t f = 0; f < bd.Nt; ++f) {
    const int32_t* tv = bd.tris.data() + 3 * f;
    double C[3][3];
    cross_mat(bd.ntri.data() + 3 * f, C);  // (nu x e_d)_c
    const double A = bd.area[f];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        const double mab = A / 12.0 * (a == b ? 2.0 : 1.0);  // int_F phi_a phi_b
        const int64_t k = find(tv[a], tv[b]);
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) B9[9 * k + 3 * c + d] += 0.5 * mab * C[c][d];
      }
  }
}

void dmi_blocks_scaled(const double* X, const int32_t* tets, int64_t E, const HostFem& fem, const HostBoundary& bd,
                       double Ms, double D_int, const double* n_int, double D_bulk, std::vector<double>& B9) {
  constexpr double mu0 = 4e-7 * 3.14159265358979323846;
  const int64_t nnz = fem.rowptr[fem.N];
  B9.assign(9 * nnz, 0.0);
  std::vector<double> part;
  if (D_int != 0.0) {
    SPX_CHECK(n_int != nullptr, "interfacial DMI needs the interface normal field");
    assemble_dmi_interfacial(X, tets, E, fem, bd, n_int, part);
    for (int64_t i = 0; i < fem.N; ++i) {
      const double sc = -2.0 * D_int / (mu0 * Ms) / 1e-9 / fem.vol[i];
      for (int64_t k = fem.rowptr[i]; k < fem.rowptr[i + 1]; ++k)
        for (int q = 0; q < 9; ++q) B9[9 * k + q] += sc * part[9 * k + q];
    }
  }
  if (D_bulk != 0.0) {
    assemble_dmi_bulk(X, tets, E, fem, bd, part);
    for (int64_t i = 0; i < fem.N; ++i) {
      const double sc = 2.0 * D_bulk / (mu0 * Ms) * 1e9 / fem.vol[i];
      for (int64_t k = fem.rowptr[i]; k < fem.rowptr[i + 1]; ++k)
        for (int q = 0; q < 9; ++q) B9[9 * k + q] += sc * part[9 * k + q];
    }
  }
}

// ------------------------------------------------------------------ SELL-32
void build_sell(const std::vector<int64_t>& rowptr, const std::vector<int32_t>& col,
                const std::vector<int32_t>& rows, const std::vector<int32_t>* col_map, HostSell& out) {
  const int64_t R = static_cast<int64_t>(rows.size());
  out.nrows = R;
  out.nslices = (R + SELL_C - 1) / SELL_C;
  out.slice_ptr.assign(out.nslices + 1, 0);
  auto row_len = [&](int64_t r) {
    const int32_t i = rows[r];
    if (!col_map) return rowptr[i + 1] - rowptr[i];
    int64_t n = 0;
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) n += ((*col_map)[col[k]] >= 0);
    return n;
  };
  for (int64_t s = 0; s < out.nslices; ++s) {
    int64_t w = 0;
    for (int64_t r = s * SELL_C; r < std::min(R, (s + 1) * SELL_C); ++r) w = std::max(w, row_len(r));
    out.slice_ptr[s + 1] = out.slice_ptr[s] + w * SELL_C;
  }
  out.col.assign(out.slice_ptr.back(), 0);
  out.map.assign(rowptr.back(), -1);
  for (int64_t r = 0; r < R; ++r) {
    const int64_t s = r / SELL_C, lane = r % SELL_C;
    const int64_t w = (out.slice_ptr[s + 1] - out.slice_ptr[s]) / SELL_C;
    const int32_t i = rows[r];
    int64_t q = 0;
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
      int32_t c = col[k];
      if (col_map) {
        c = (*col_map)[c];
        if (c < 0) continue;
      }
      const int64_t pos = out.slice_ptr[s] + q * SELL_C + lane;
      out.col[pos] = c;
      out.map[k] = pos;
      ++q;
    }
    // padding: point at a valid column with value 0
    const int32_t pad = col_map ? 0 : static_cast<int32_t>(r);
    for (; q < w; ++q) out.col[out.slice_ptr[s] + q * SELL_C + lane] = pad;
  }
  // unused lanes of the last slice
  for (int64_t r = R; r < out.nslices * SELL_C; ++r) {
    const int64_t s = r / SELL_C, lane = r % SELL_C;
    const int64_t w = (out.slice_ptr[s + 1] - out.slice_ptr[s]) / SELL_C;
    for (int64_t q = 0; q < w; ++q) out.col[out.slice_ptr[s] + q * SELL_C + lane] = 0;
  }
}

// ------------------------------------------------------------------ cluster tree
double TreeNode::diameter() const {
  const double d0 = bmax[0] - bmin[0], d1 = bmax[1] - bmin[1], d2 = bmax[2] - bmin[2];
  return std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}

void build_cluster_tree(const double* pts, int64_t n, int leaf_size, ClusterTree& out) {
  SPX_CHECK(n > 0, "cluster tree needs at least one point");
  SPX_CHECK(leaf_size >= 1, "leaf_size must be positive");
  out.perm.clear();
  out.perm.reserve(n);
  out.nodes.clear();
  std::vector<int32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::vector<int32_t> tmp(n);
  // explicit stack: (lo, hi, node index); children are visited left then right,
  // matching the reference's recursion order (ordered_indices appended at leaves)
  struct Frame { int64_t lo, hi; int32_t node; int stage; };
  out.nodes.push_back(TreeNode{});
  std::vector<Frame> st;
  st.push_back({0, n, 0, 0});
  while (!st.empty()) {
    Frame& f = st.back();
    TreeNode* nd = &out.nodes[f.node];
    if (f.stage == 0) {
      double mn[3] = {1e308, 1e308, 1e308}, mx[3] = {-1e308, -1e308, -1e308};
      for (int64_t k = f.lo; k < f.hi; ++k)
        for (int c = 0; c < 3; ++c) {
          const double v = pts[3 * (int64_t)idx[k] + c];
          mn[c] = std::min(mn[c], v);
          mx[c] = std::max(mx[c], v);
        }
      for (int c = 0; c < 3; ++c) { nd->bmin[c] = mn[c]; nd->bmax[c] = mx[c]; }
      if (f.hi - f.lo <= leaf_size) {
        nd->start = static_cast<int32_t>(out.perm.size());
        for (int64_t k = f.lo; k < f.hi; ++k) out.perm.push_back(idx[k]);
        nd->stop = static_cast<int32_t>(out.perm.size());
        st.pop_back();
        continue;
      }
      // argmax extent (first on ties), stable sort along that axis, mid = size//2
      int axis = 0;
      double best = mx[0] - mn[0];
      for (int c = 1; c < 3; ++c)
        if (mx[c] - mn[c] > best) { best = mx[c] - mn[c]; axis = c; }
      std::stable_sort(idx.begin() + f.lo, idx.begin() + f.hi, [&](int32_t a, int32_t b) {
        return pts[3 * (int64_t)a + axis] < pts[3 * (int64_t)b + axis];
      });
      int64_t mid = (f.hi - f.lo) / 2;
      if (mid == 0 || mid == f.hi - f.lo) mid = std::max<int64_t>(1, (f.hi - f.lo) / 2);
      const int32_t L = static_cast<int32_t>(out.nodes.size());
      out.nodes.push_back(TreeNode{});
      out.nodes.push_back(TreeNode{});
      nd = &out.nodes[f.node];
      nd->left = L;
      nd->right = L + 1;
      f.stage = 1;
      const int64_t lo = f.lo, hi = f.hi;
      st.push_back({lo + mid, hi, L + 1, 0});  // right processed after left
      st.push_back({lo, lo + mid, L, 0});
      continue;
    }
    st.pop_back();
  }
  // fill start/stop of internal nodes bottom-up (children always have larger index)
  for (int64_t k = static_cast<int64_t>(out.nodes.size()) - 1; k >= 0; --k) {
    TreeNode& nd = out.nodes[k];
    if (!nd.leaf()) {
      nd.start = out.nodes[nd.left].start;
      nd.stop = out.nodes[nd.right].stop;
    }
  }
}

bool admissible(const TreeNode& a, const TreeNode& b, double eta) {
  double s = 0.0;
  for (int c = 0; c < 3; ++c) {
    const double g = std::max(std::max(a.bmin[c] - b.bmax[c], b.bmin[c] - a.bmax[c]), 0.0);
    s += g * g;
  }
  const double dist = std::sqrt(s);
  if (dist <= 0.0) return false;
  return std::max(a.diameter(), b.diameter()) <= eta * dist;
}

}  // namespace spx
