// Host set-up of the smoothed-aggregation hierarchy (see amg.cuh for the method).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "amg.cuh"

namespace spx {
namespace {

double diag_of(const CsrHost& A, int64_t i) {
  for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
    if (A.ci[k] == i) return A.v[k];
  return 0.0;
}

// lambda_max(D^-1 A) by power iteration from a fixed pseudo-random start
double lambda_max_dinv_a(const CsrHost& A, const std::vector<double>& dinv, int iters) {
  const int64_t n = A.n;
  std::vector<double> x(n), y(n);
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (int64_t i = 0; i < n; ++i) {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    x[i] = 0.5 + static_cast<double>(s >> 11) * (1.0 / 9007199254740992.0);
  }
  double lam = 0.0;
  for (int it = 0; it < iters; ++it) {
    double nx = 0.0;
    for (int64_t i = 0; i < n; ++i) nx += x[i] * x[i];
    nx = std::sqrt(nx);
    if (!(nx > 0.0)) break;
    for (int64_t i = 0; i < n; ++i) x[i] /= nx;
    for (int64_t i = 0; i < n; ++i) {
      double a = 0.0;
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) a += A.v[k] * x[A.ci[k]];
      y[i] = dinv[i] * a;
    }
    double xy = 0.0;
    for (int64_t i = 0; i < n; ++i) xy += x[i] * y[i];
    lam = xy;
    x.swap(y);
  }
  return lam;
}

// aggregate id of every node (three passes), returns the number of aggregates
int64_t aggregate(const CsrHost& A, double theta, std::vector<int64_t>& agg) {
  const int64_t n = A.n;
  std::vector<double> d(n);
  for (int64_t i = 0; i < n; ++i) d[i] = std::fabs(diag_of(A, i));
  auto strong = [&](int64_t i, int64_t k) {
    const int64_t j = A.ci[k];
    if (j == i) return false;
    const double a = std::fabs(A.v[k]);
    return a > theta * std::sqrt(d[i] * d[j]) && a > 1e-14 * std::sqrt(d[i] * d[j]);
  };
  agg.assign(n, -1);
  int64_t na = 0;
  // pass 1: a node whose strong neighbours are all free roots a new aggregate
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    bool free = true, any = false;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1] && free; ++k)
      if (strong(i, k)) {
        any = true;
        if (agg[A.ci[k]] >= 0) free = false;
      }
    if (!free || !any) continue;
    agg[i] = na;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (strong(i, k)) agg[A.ci[k]] = na;
    ++na;
  }
  // pass 2: join the aggregate of the strongest aggregated neighbour (pass-1 labels only)
  std::vector<int64_t> agg1 = agg;
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    double best = -1.0;
    int64_t ba = -1;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (strong(i, k) && agg1[A.ci[k]] >= 0 && std::fabs(A.v[k]) > best) {
        best = std::fabs(A.v[k]);
        ba = agg1[A.ci[k]];
      }
    if (ba >= 0) agg[i] = ba;
  }
  // pass 3: the rest, with their free strong neighbours (isolated nodes alone)
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    agg[i] = na;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (strong(i, k) && agg[A.ci[k]] < 0) agg[A.ci[k]] = na;
    ++na;
  }
  return na;
}

// C = A * B (CSR, sorted columns), dense accumulator per row
void spgemm(const CsrHost& A, const CsrHost& B, CsrHost& C) {
  C.n = A.n;
  C.ncols = B.ncols;
  C.rp.assign(A.n + 1, 0);
  C.ci.clear();
  C.v.clear();
  std::vector<double> acc(B.ncols, 0.0);
  std::vector<int32_t> mark(B.ncols, -1), cols;
  for (int64_t i = 0; i < A.n; ++i) {
    cols.clear();
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const int64_t j = A.ci[k];
      const double a = A.v[k];
      for (int64_t q = B.rp[j]; q < B.rp[j + 1]; ++q) {
        const int32_t c = B.ci[q];
        if (mark[c] != static_cast<int32_t>(i)) {
          mark[c] = static_cast<int32_t>(i);
          acc[c] = 0.0;
          cols.push_back(c);
        }
        acc[c] += a * B.v[q];
      }
    }
    std::sort(cols.begin(), cols.end());
    for (int32_t c : cols) {
      C.ci.push_back(c);
      C.v.push_back(acc[c]);
    }
    C.rp[i + 1] = static_cast<int64_t>(C.ci.size());
  }
}

void transpose(const CsrHost& A, CsrHost& T) {
  T.n = A.ncols;
  T.ncols = A.n;
  T.rp.assign(T.n + 1, 0);
  for (int32_t c : A.ci) T.rp[c + 1]++;
  for (int64_t i = 0; i < T.n; ++i) T.rp[i + 1] += T.rp[i];
  T.ci.resize(A.ci.size());
  T.v.resize(A.v.size());
  std::vector<int64_t> pos(T.rp.begin(), T.rp.end() - 1);
  for (int64_t i = 0; i < A.n; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const int64_t p = pos[A.ci[k]]++;
      T.ci[p] = static_cast<int32_t>(i);
      T.v[p] = A.v[k];
    }
}

}  // namespace

void amg_build(const CsrHost& A0, const std::vector<double>& null0, bool singular, const AmgOptions& o,
               AmgHost& out) {
  out.lv.clear();
  CsrHost A = A0;
  std::vector<double> w = null0;
  for (int level = 0;; ++level) {
    AmgHostLevel L;
    L.A = A;
    L.dinv.resize(A.n);
    for (int64_t i = 0; i < A.n; ++i) {
      const double d = diag_of(A, i);
      SPX_CHECK(d > 0.0, "AMG level matrix has a non-positive diagonal");
      L.dinv[i] = 1.0 / d;
    }
    // the top level is always smoothed (at least one coarsening), unless it is tiny
    const bool last = (A.n <= o.coarse_max && (level > 0 || A.n <= 64)) || level + 1 >= o.max_levels;
    if (last) {
      out.lv.push_back(std::move(L));
      break;
    }
    L.lmax = lambda_max_dinv_a(A, L.dinv, o.power_iters);
    std::vector<int64_t> agg;
    const int64_t nc = aggregate(A, o.theta, agg);
    if (nc >= A.n || nc == 0 || static_cast<double>(nc) > 0.85 * static_cast<double>(A.n)) {
      out.lv.push_back(std::move(L));  // coarsening stalled: this level becomes the coarsest
      break;
    }
    // tentative prolongator
    std::vector<double> wn(nc, 0.0);
    for (int64_t i = 0; i < A.n; ++i) wn[agg[i]] += w[i] * w[i];
    for (auto& v : wn) v = std::sqrt(v);
    CsrHost P0;
    P0.n = A.n;
    P0.ncols = nc;
    P0.rp.resize(A.n + 1);
    P0.ci.resize(A.n);
    P0.v.resize(A.n);
    for (int64_t i = 0; i < A.n; ++i) {
      P0.rp[i] = i;
      P0.ci[i] = static_cast<int32_t>(agg[i]);
      P0.v[i] = wn[agg[i]] > 0.0 ? w[i] / wn[agg[i]] : 0.0;
    }
    P0.rp[A.n] = A.n;
    // smoothed prolongator P = P0 - omega D^-1 A P0
    const double omega = 4.0 / (3.0 * L.lmax);
    CsrHost AP0;
    spgemm(A, P0, AP0);
    CsrHost P;
    P.n = A.n;
    P.ncols = nc;
    P.rp.assign(A.n + 1, 0);
    for (int64_t i = 0; i < A.n; ++i) {
      // merge row i of P0 (one entry) with -omega dinv_i (A P0)_i
      const int32_t c0 = P0.ci[i];
      bool placed = false;
      for (int64_t k = AP0.rp[i]; k < AP0.rp[i + 1]; ++k) {
        const int32_t c = AP0.ci[k];
        double v = -omega * L.dinv[i] * AP0.v[k];
        if (c == c0) {
          v += P0.v[i];
          placed = true;
        }
        if (v != 0.0) {
          P.ci.push_back(c);
          P.v.push_back(v);
        }
      }
      if (!placed && P0.v[i] != 0.0) {  // keep columns sorted
        auto it = std::lower_bound(P.ci.begin() + P.rp[i], P.ci.end(), c0);
        const int64_t pos = it - P.ci.begin();
        P.ci.insert(it, c0);
        P.v.insert(P.v.begin() + pos, P0.v[i]);
      }
      P.rp[i + 1] = static_cast<int64_t>(P.ci.size());
    }
    CsrHost R, AP, Ac;
    transpose(P, R);
    spgemm(A, P, AP);
    spgemm(R, AP, Ac);
    // symmetrise the Galerkin product (removes rounding asymmetry)
    {
      CsrHost At;
      transpose(Ac, At);
      for (int64_t i = 0; i < Ac.n; ++i)
        for (int64_t k = Ac.rp[i], q = At.rp[i]; k < Ac.rp[i + 1]; ++k, ++q) Ac.v[k] = 0.5 * (Ac.v[k] + At.v[q]);
    }
    L.P = std::move(P);
    L.R = std::move(R);
    out.lv.push_back(std::move(L));
    A = std::move(Ac);
    w = std::move(wn);
  }
  // coarsest: dense A_c (+ rank-one term on the null vector when singular), inverted on the device
  const CsrHost& C = out.lv.back().A;
  const int64_t nc = C.n;
  SPX_CHECK(nc <= 8192, "AMG coarsest level is too large for a dense inverse");
  std::vector<double> M(nc * nc, 0.0);
  double dsum = 0.0;
  for (int64_t i = 0; i < nc; ++i)
    for (int64_t k = C.rp[i]; k < C.rp[i + 1]; ++k) {
      M[i * nc + C.ci[k]] = C.v[k];
      if (C.ci[k] == i) dsum += C.v[k];
    }
  if (singular) {
    // one null vector per connected component of the coarse graph (a disjoint union of
    // meshes, e.g. an ensemble of independent samples, has one constant per sample): add
    // tau w_c w_c^T for each component c
    std::vector<int64_t> comp(nc, -1), stack;
    int64_t ncomp = 0;
    for (int64_t r = 0; r < nc; ++r) {
      if (comp[r] >= 0) continue;
      comp[r] = ncomp;
      stack.assign(1, r);
      while (!stack.empty()) {
        const int64_t i = stack.back();
        stack.pop_back();
        for (int64_t k = C.rp[i]; k < C.rp[i + 1]; ++k)
          if (C.v[k] != 0.0 && comp[C.ci[k]] < 0) {
            comp[C.ci[k]] = ncomp;
            stack.push_back(C.ci[k]);
          }
      }
      ++ncomp;
    }
    std::vector<double> ww(ncomp, 0.0);
    for (int64_t i = 0; i < nc; ++i) ww[comp[i]] += w[i] * w[i];
    const double dmean = dsum / static_cast<double>(nc);
    for (int64_t i = 0; i < nc; ++i)
      for (int64_t j = 0; j < nc; ++j)
        if (comp[i] == comp[j]) M[i * nc + j] += dmean / std::max(ww[comp[i]], 1e-300) * w[i] * w[j];
  }
  out.coarse_dense = std::move(M);
}

}  // namespace spx
