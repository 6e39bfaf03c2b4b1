// Reference tetrahedron operators on the host in FP64: the mesh-independent half of NewDG3D
// (element/library/gonudg/startup3d.go:94-176) — nodes, Vandermonde, Dr/Ds/Dt, Fmask and LIFT.
// These Np x Np matrices are setup inputs of the hot path; they are bound to the runner like the
// reference binds GetRefMatrices() (tetnudg/tet_nudg_mesh.go:371-389).
//
// Dense linear algebra is self-contained: a partially pivoted LU inverse, and cyclic Jacobi rotations
// (Golub & Van Loan, "Matrix Computations", 8.5) for the symmetric tridiagonal Jacobi matrix whose
// eigen-decomposition gives Gauss-Jacobi nodes and weights (Golub & Welsch 1969).
#include "element.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace dgk {
namespace {

using Vec = std::vector<double>;

// Orthonormal Jacobi polynomial P_n^(alpha,beta) at every x (jacobip.go:30-98).
Vec jacobi_p(const Vec &x, double alpha, double beta, int n) {
  const double ab = alpha + beta, ab1 = ab + 1.0, a1 = alpha + 1.0, b1 = beta + 1.0;
  const double g0 = std::pow(2.0, ab1) / ab1 * std::tgamma(a1) * std::tgamma(b1) / std::tgamma(ab1);
  Vec p0(x.size(), 1.0 / std::sqrt(g0));
  if (n == 0) return p0;
  const double g1 = a1 * b1 / (ab + 3.0) * g0;
  Vec p1(x.size());
  for (size_t i = 0; i < x.size(); ++i) p1[i] = ((ab + 2.0) * x[i] / 2.0 + (alpha - beta) / 2.0) * (1.0 / std::sqrt(g1));
  if (n == 1) return p1;
  double aold = 2.0 / (2.0 + ab) * std::sqrt(a1 * b1 / (ab + 3.0));
  for (int k = 1; k < n; ++k) {
    const double fk = k, h1 = 2.0 * fk + ab;
    const double anew =
        2.0 / (h1 + 2.0) * std::sqrt((fk + 1.0) * (fk + ab1) * (fk + a1) * (fk + b1) / (h1 + 1.0) / (h1 + 3.0));
    const double bnew = -(alpha * alpha - beta * beta) / h1 / (h1 + 2.0);
    Vec p2(x.size());
    for (size_t i = 0; i < x.size(); ++i) p2[i] = 1.0 / anew * (-aold * p0[i] + (x[i] - bnew) * p1[i]);
    p0.swap(p1);
    p1.swap(p2);
    aold = anew;
  }
  return p1;
}

Vec grad_jacobi_p(const Vec &x, double alpha, double beta, int n) {
  if (n == 0) return Vec(x.size(), 0.0);
  Vec p = jacobi_p(x, alpha + 1.0, beta + 1.0, n - 1);
  const double f = std::sqrt(n * (n + alpha + beta + 1.0));
  for (double &v : p) v *= f;
  return p;
}

// Eigenvalues (ascending) and first eigenvector components of the symmetric tridiagonal matrix with
// diagonal d and off-diagonal e, by the cyclic Jacobi method: each rotation zeroes one off-diagonal entry
// A[p][q] with tan(phi) the smaller root of t^2 + 2 theta t - 1 = 0, theta = (A_qq - A_pp) / (2 A_pq);
// sweeps repeat until the off-diagonal mass vanishes (quadratic convergence, n <= 9 here).
void tridiag_eig(const Vec &d, const Vec &e, Vec &lambda, Vec &first) {
  const int n = (int)d.size();
  std::vector<Vec> A(n, Vec(n, 0.0)), Q(n, Vec(n, 0.0));
  for (int i = 0; i < n; ++i) {
    A[i][i] = d[i];
    Q[i][i] = 1.0;
    if (i + 1 < n) A[i][i + 1] = A[i + 1][i] = e[i];
  }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) (i == j ? diag : off) += A[i][j] * A[i][j];
    if (off <= 1e-34 * (diag + 1e-300)) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p][q];
        if (apq == 0.0) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
        const double tn = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(tn * tn + 1.0), s = tn * c;
        for (int k = 0; k < n; ++k) {  // A <- A J (columns p, q)
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // A <- J^T A (rows p, q)
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {  // Q <- Q J
          const double qkp = Q[k][p], qkq = Q[k][q];
          Q[k][p] = c * qkp - s * qkq;
          Q[k][q] = s * qkp + c * qkq;
        }
      }
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return A[a][a] < A[b][b]; });
  lambda.resize(n);
  first.resize(n);
  for (int i = 0; i < n; ++i) {
    lambda[i] = A[order[i]][order[i]];
    first[i] = Q[0][order[i]];
  }
}

double gamma0(double alpha, double beta) {
  const double ab1 = alpha + beta + 1.0;
  return std::tgamma(alpha + 1.0) * std::tgamma(beta + 1.0) * std::pow(2.0, ab1) / ab1 / std::tgamma(ab1);
}

// Gauss-Jacobi nodes and weights (jacobi_quadrature.go:39-101).
void jacobi_gq(double alpha, double beta, int n, Vec &x, Vec &w) {
  if (n == 0) {
    x = {-(alpha - beta) / (alpha + beta + 2.0)};
    w = {2.0};
    return;
  }
  Vec d0(n + 1), d1(n);
  for (int i = 0; i <= n; ++i) {
    const double h1 = 2.0 * i + alpha + beta;
    d0[i] = (alpha + beta < 1e-15 && i == 0) ? 0.0 : (beta * beta - alpha * alpha) / (h1 * (h1 + 2.0));
    if (i < n) {
      const double ip1 = i + 1.0;
      d1[i] = 2.0 / (h1 + 2.0) *
              std::sqrt(ip1 * (ip1 + alpha + beta) * (ip1 + alpha) * (ip1 + beta) / (h1 + 1.0) / (h1 + 3.0));
    }
  }
  Vec first;
  tridiag_eig(d0, d1, x, first);
  const double g = gamma0(alpha, beta);
  w.resize(x.size());
  for (size_t i = 0; i < x.size(); ++i) w[i] = first[i] * first[i] * g;
}

// Gauss-Lobatto nodes (jacobi_quadrature.go:16-37).
Vec jacobi_gl(double alpha, double beta, int n) {
  if (n == 0) return {0.0};
  if (n == 1) return {-1.0, 1.0};
  Vec xi, wi;
  jacobi_gq(alpha + 1.0, beta + 1.0, n - 2, xi, wi);
  Vec x(n + 1);
  x[0] = -1.0;
  std::copy(xi.begin(), xi.end(), x.begin() + 1);
  x[n] = 1.0;
  return x;
}

// Interpolated warp (nodes3d.go:290-324): the full Lagrange interpolant through the equidistant nodes of
// (gaussX - xeq), multiplied by (1 - x^2).  gaussX is the negated (so descending) Lobatto set.
Vec eval_warp(int p, const Vec &gauss_x, const Vec &xs) {
  Vec xeq(p + 1);
  for (int i = 0; i <= p; ++i) xeq[i] = -1.0 + 2.0 * i / p;
  Vec out(xs.size());
  for (size_t q = 0; q < xs.size(); ++q) {
    const double x = xs[q];
    double acc = 0.0;
    for (int j = 0; j <= p; ++j) {
      double l = 1.0;
      for (int k = 0; k <= p; ++k)
        if (k != j) l *= (x - xeq[k]) / (xeq[j] - xeq[k]);
      acc += l * (gauss_x[j] - xeq[j]);
    }
    out[q] = acc * (1.0 - x * x);
  }
  return out;
}

// Warp of one face in the equilateral triangle frame (nodes3d.go:221-287).
void eval_shift(int p, double pval, const Vec &l1, const Vec &l2, const Vec &l3, Vec &dx, Vec &dy) {
  Vec gx = jacobi_gl(0.0, 0.0, p);
  for (double &v : gx) v = -v;
  const size_t n = l1.size();
  Vec t1(n), t2(n), t3(n);
  for (size_t i = 0; i < n; ++i) {
    t1[i] = l3[i] - l2[i];
    t2[i] = l1[i] - l3[i];
    t3[i] = l2[i] - l1[i];
  }
  Vec w1 = eval_warp(p, gx, t1), w2 = eval_warp(p, gx, t2), w3 = eval_warp(p, gx, t3);
  const double c2 = std::cos(2.0 * M_PI / 3.0), c4 = std::cos(4.0 * M_PI / 3.0);
  const double s2 = std::sin(2.0 * M_PI / 3.0), s4 = std::sin(4.0 * M_PI / 3.0);
  dx.resize(n);
  dy.resize(n);
  for (size_t i = 0; i < n; ++i) {
    const double a = l2[i] * l3[i] * (4.0 * w1[i]) * (1.0 + pval * pval * l1[i] * l1[i]);
    const double b = l1[i] * l3[i] * (4.0 * w2[i]) * (1.0 + pval * pval * l2[i] * l2[i]);
    const double c = l1[i] * l2[i] * (4.0 * w3[i]) * (1.0 + pval * pval * l3[i] * l3[i]);
    dx[i] = a + c2 * b + c4 * c;
    dy[i] = s2 * b + s4 * c;
  }
}

struct V3 {
  double x, y, z;
};
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 mid(V3 a, V3 b) { return {0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z)}; }
V3 unit(V3 a) {
  const double n = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return {a.x / n, a.y / n, a.z / n};
}

const V3 kV1{-1.0, -1.0 / std::sqrt(3.0), -1.0 / std::sqrt(6.0)};
const V3 kV2{1.0, -1.0 / std::sqrt(3.0), -1.0 / std::sqrt(6.0)};
const V3 kV3{0.0, 2.0 / std::sqrt(3.0), -1.0 / std::sqrt(6.0)};
const V3 kV4{0.0, 0.0, 3.0 / std::sqrt(6.0)};

// Warp & blend nodes (nodes3d.go:17-174), returned directly in (r,s,t) via the affine map of
// xyztorst.go:8-69.
void warp_blend_nodes(int p, Vec &r, Vec &s, Vec &t) {
  static const double kAlpha[15] = {0.0,    0.0,    0.0,    0.1002, 1.1332, 1.5608, 1.3413, 1.2577,
                                    1.1603, 1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655};
  const double alpha = (p >= 0 && p < 15) ? kAlpha[p] : 1.0;
  const double tol = 1e-10;
  // equidistant lattice, r fastest (nodes3d.go:177-205)
  Vec er, es, et;
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= p - n; ++m)
      for (int l = 0; l <= p - n - m; ++l) {
        er.push_back(-1.0 + 2.0 * l / p);
        es.push_back(-1.0 + 2.0 * m / p);
        et.push_back(-1.0 + 2.0 * n / p);
      }
  const size_t np = er.size();
  Vec L1(np), L2(np), L3(np), L4(np);
  for (size_t i = 0; i < np; ++i) {
    L1[i] = (1.0 + et[i]) / 2.0;
    L2[i] = (1.0 + es[i]) / 2.0;
    L3[i] = -(1.0 + er[i] + es[i] + et[i]) / 2.0;
    L4[i] = (1.0 + er[i]) / 2.0;
  }
  const V3 tan1[4] = {unit(sub(kV2, kV1)), unit(sub(kV2, kV1)), unit(sub(kV3, kV2)), unit(sub(kV3, kV1))};
  const V3 tan2[4] = {unit(sub(kV3, mid(kV1, kV2))), unit(sub(kV4, mid(kV1, kV2))), unit(sub(kV4, mid(kV2, kV3))),
                      unit(sub(kV4, mid(kV1, kV3)))};
  Vec X(np), Y(np), Z(np), sx(np, 0.0), sy(np, 0.0), sz(np, 0.0);
  for (size_t i = 0; i < np; ++i) {
    X[i] = L3[i] * kV1.x + L4[i] * kV2.x + L2[i] * kV3.x + L1[i] * kV4.x;
    Y[i] = L3[i] * kV1.y + L4[i] * kV2.y + L2[i] * kV3.y + L1[i] * kV4.y;
    Z[i] = L3[i] * kV1.z + L4[i] * kV2.z + L2[i] * kV3.z + L1[i] * kV4.z;
  }
  const Vec *perm[4][4] = {{&L1, &L2, &L3, &L4}, {&L2, &L1, &L3, &L4}, {&L3, &L1, &L4, &L2}, {&L4, &L1, &L3, &L2}};
  for (int f = 0; f < 4; ++f) {
    const Vec &La = *perm[f][0], &Lb = *perm[f][1], &Lc = *perm[f][2], &Ld = *perm[f][3];
    Vec w1, w2;
    eval_shift(p, alpha, Lb, Lc, Ld, w1, w2);
    for (size_t i = 0; i < np; ++i) {
      double blend = Lb[i] * Lc[i] * Ld[i];
      const double den = (Lb[i] + 0.5 * La[i]) * (Lc[i] + 0.5 * La[i]) * (Ld[i] + 0.5 * La[i]);
      if (den > tol) blend = (1.0 + alpha * alpha * La[i] * La[i]) * blend / den;
      sx[i] += blend * w1[i] * tan1[f].x + blend * w2[i] * tan2[f].x;
      sy[i] += blend * w1[i] * tan1[f].y + blend * w2[i] * tan2[f].y;
      sz[i] += blend * w1[i] * tan1[f].z + blend * w2[i] * tan2[f].z;
      const int inside = (Lb[i] > tol) + (Lc[i] > tol) + (Ld[i] > tol);
      if (La[i] < tol && inside < 3) {  // on this face but not on all three of its edges
        sx[i] = w1[i] * tan1[f].x + w2[i] * tan2[f].x;
        sy[i] = w1[i] * tan1[f].y + w2[i] * tan2[f].y;
        sz[i] = w1[i] * tan1[f].z + w2[i] * tan2[f].z;
      }
    }
  }
  // (x,y,z) -> (r,s,t): invert A = 0.5 [v2-v1, v3-v1, v4-v1] about the offset 0.5 (v2+v3+v4-v1)
  const double A[3][3] = {{0.5 * (kV2.x - kV1.x), 0.5 * (kV3.x - kV1.x), 0.5 * (kV4.x - kV1.x)},
                          {0.5 * (kV2.y - kV1.y), 0.5 * (kV3.y - kV1.y), 0.5 * (kV4.y - kV1.y)},
                          {0.5 * (kV2.z - kV1.z), 0.5 * (kV3.z - kV1.z), 0.5 * (kV4.z - kV1.z)}};
  const double off[3] = {0.5 * (kV2.x + kV3.x + kV4.x - kV1.x), 0.5 * (kV2.y + kV3.y + kV4.y - kV1.y),
                         0.5 * (kV2.z + kV3.z + kV4.z - kV1.z)};
  const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  double inv[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      // cofactor C[j][i] / det
      const int a0 = (j + 1) % 3, a1 = (j + 2) % 3, b0 = (i + 1) % 3, b1 = (i + 2) % 3;
      inv[i][j] = (A[a0][b0] * A[a1][b1] - A[a0][b1] * A[a1][b0]) / det;
    }
  r.resize(np);
  s.resize(np);
  t.resize(np);
  for (size_t i = 0; i < np; ++i) {
    const double q[3] = {X[i] + sx[i] - off[0], Y[i] + sy[i] - off[1], Z[i] + sz[i] - off[2]};
    r[i] = inv[0][0] * q[0] + inv[0][1] * q[1] + inv[0][2] * q[2];
    s[i] = inv[1][0] * q[0] + inv[1][1] * q[1] + inv[1][2] * q[2];
    t[i] = inv[2][0] * q[0] + inv[2][1] * q[1] + inv[2][2] * q[2];
  }
}

// Collapsed coordinates with the reference's 1e-12 guards (rsttoabc.go:7-34).
void rst_to_abc(double r, double s, double t, double &a, double &b, double &c) {
  a = std::fabs(s + t) < 1e-12 ? -1.0 : 2.0 * (1.0 + r) / (-s - t) - 1.0;
  b = std::fabs(t - 1.0) < 1e-12 ? -1.0 : 2.0 * (1.0 + s) / (1.0 - t) - 1.0;
  c = t;
}

}  // namespace

// Dense row-major inverse by LU with partial pivoting.
std::vector<double> invert(const std::vector<double> &M, int n) {
  std::vector<double> a(M), inv((size_t)n * n, 0.0);
  std::vector<int> piv(n);
  for (int i = 0; i < n; ++i) piv[i] = i;
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(a[(size_t)i * n + k]) > std::fabs(a[(size_t)p * n + k])) p = i;
    if (a[(size_t)p * n + k] == 0.0) throw std::runtime_error("singular matrix");
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * n + j], a[(size_t)p * n + j]);
      std::swap(piv[k], piv[p]);
    }
    for (int i = k + 1; i < n; ++i) {
      const double f = a[(size_t)i * n + k] / a[(size_t)k * n + k];
      a[(size_t)i * n + k] = f;
      for (int j = k + 1; j < n; ++j) a[(size_t)i * n + j] -= f * a[(size_t)k * n + j];
    }
  }
  for (int c = 0; c < n; ++c) {  // solve L U x = P e_c
    std::vector<double> x(n);
    for (int i = 0; i < n; ++i) {
      double v = (piv[i] == c) ? 1.0 : 0.0;
      for (int j = 0; j < i; ++j) v -= a[(size_t)i * n + j] * x[j];
      x[i] = v;
    }
    for (int i = n - 1; i >= 0; --i) {
      double v = x[i];
      for (int j = i + 1; j < n; ++j) v -= a[(size_t)i * n + j] * x[j];
      x[i] = v / a[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + c] = x[i];
  }
  return inv;
}

std::vector<double> matmul(const std::vector<double> &A, const std::vector<double> &B, int m, int k, int n) {
  std::vector<double> C((size_t)m * n, 0.0);
  for (int i = 0; i < m; ++i)
    for (int l = 0; l < k; ++l) {
      const double a = A[(size_t)i * k + l];
      for (int j = 0; j < n; ++j) C[(size_t)i * n + j] += a * B[(size_t)l * n + j];
    }
  return C;
}

std::vector<double> transpose(const std::vector<double> &A, int m, int n) {
  std::vector<double> T((size_t)m * n);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) T[(size_t)j * m + i] = A[(size_t)i * n + j];
  return T;
}

RefElement::RefElement(int order) : N(order) {
  if (N < 1 || N > 8) throw std::invalid_argument("element order must be in 1..8");
  Np = (N + 1) * (N + 2) * (N + 3) / 6;
  Nfp = (N + 1) * (N + 2) / 2;
  warp_blend_nodes(N, r, s, t);

  // Vandermonde and its gradients, modes ordered i, j, k (vandermonde3d.go:15-73, simplex3dp.go:15-118)
  V.assign((size_t)Np * Np, 0.0);
  std::vector<double> Vr(V), Vs(V), Vt(V);
  Vec a(Np), b(Np), c(Np);
  for (int q = 0; q < Np; ++q) rst_to_abc(r[q], s[q], t[q], a[q], b[q], c[q]);
  int m = 0;
  for (int i = 0; i <= N; ++i)
    for (int j = 0; j <= N - i; ++j)
      for (int k = 0; k <= N - i - j; ++k, ++m) {
        const Vec fa = jacobi_p(a, 0, 0, i), gb = jacobi_p(b, 2 * i + 1, 0, j), hc = jacobi_p(c, 2 * (i + j) + 2, 0, k);
        const Vec dfa = grad_jacobi_p(a, 0, 0, i), dgb = grad_jacobi_p(b, 2 * i + 1, 0, j),
                  dhc = grad_jacobi_p(c, 2 * (i + j) + 2, 0, k);
        const double nrm = std::pow(2.0, 2.0 * i + j + 1.5);
        for (int q = 0; q < Np; ++q) {
          const double ob = 1.0 - b[q], oc = 1.0 - c[q];
          V[(size_t)q * Np + m] = (2.0 * std::sqrt(2.0) * fa[q] * gb[q]) * std::pow(ob, (double)i) *
                                  (hc[q] * std::pow(oc, (double)(i + j)));
          double dr = dfa[q] * gb[q] * hc[q];
          if (i > 0) dr *= std::pow(0.5 * ob, i - 1.0);
          if (i + j > 0) dr *= std::pow(0.5 * oc, i + j - 1.0);
          double tmp = dgb[q] * std::pow(0.5 * ob, (double)i);
          if (i > 0) tmp -= 0.5 * i * gb[q] * std::pow(0.5 * ob, i - 1.0);
          if (i + j > 0) tmp *= std::pow(0.5 * oc, i + j - 1.0);
          tmp = fa[q] * tmp * hc[q];
          const double ds = 0.5 * (1.0 + a[q]) * dr + tmp;
          double tmp2 = dhc[q] * std::pow(0.5 * oc, (double)(i + j));
          if (i + j > 0) tmp2 -= 0.5 * (i + j) * hc[q] * std::pow(0.5 * oc, i + j - 1.0);
          tmp2 = fa[q] * gb[q] * tmp2 * std::pow(0.5 * ob, (double)i);
          const double dt = 0.5 * (1.0 + a[q]) * dr + 0.5 * (1.0 + b[q]) * tmp + tmp2;
          Vr[(size_t)q * Np + m] = dr * nrm;
          Vs[(size_t)q * Np + m] = ds * nrm;
          Vt[(size_t)q * Np + m] = dt * nrm;
        }
      }
  Vinv = invert(V, Np);
  MassMatrix = matmul(transpose(Vinv, Np, Np), Vinv, Np, Np, Np);
  Dr = matmul(Vr, Vinv, Np, Np, Np);
  Ds = matmul(Vs, Vinv, Np, Np, Np);
  Dt = matmul(Vt, Vinv, Np, Np, Np);
  M = matmul(V, transpose(V, Np, Np), Np, Np, Np);  // GetNodalModal's "M" (tet_nudg_mesh.go:323-330)
  Minv = invert(M, Np);

  // Fmask: t = -1, s = -1, r+s+t = -1, r = -1 within NODETOL 1e-7 (startup3d.go:179-209)
  Fmask.clear();
  for (int f = 0; f < 4; ++f) {
    int cnt = 0;
    for (int q = 0; q < Np; ++q) {
      const double v = f == 0 ? t[q] : f == 1 ? s[q] : f == 2 ? r[q] + s[q] + t[q] : r[q];
      if (std::fabs(1.0 + v) < 1e-7) {
        Fmask.push_back(q);
        ++cnt;
      }
    }
    if (cnt != Nfp) throw std::runtime_error("face node count mismatch");
  }

  // LIFT = V (V^T Emat), Emat holding inv(VFace VFace^T) per face (lift3d.go:9-90)
  const int NF = 4 * Nfp;
  std::vector<double> Emat((size_t)Np * NF, 0.0);
  for (int f = 0; f < 4; ++f) {
    std::vector<double> vf((size_t)Nfp * Nfp);
    for (int q = 0; q < Nfp; ++q) {
      const int v = Fmask[f * Nfp + q];
      const double fr = (f <= 1) ? r[v] : s[v];
      const double fs = (f == 0) ? s[v] : t[v];
      const double aa = fs != 1.0 ? 2.0 * (1.0 + fr) / (1.0 - fs) - 1.0 : -1.0;  // vandermonde2D.go:58-72
      int col = 0;
      for (int i = 0; i <= N; ++i)
        for (int j = 0; j <= N - i; ++j, ++col) {
          const Vec h1 = jacobi_p(Vec{aa}, 0, 0, i), h2 = jacobi_p(Vec{fs}, 2 * i + 1, 0, j);
          double pw = 1.0;
          for (int k = 0; k < i; ++k) pw *= (1.0 - fs);
          vf[(size_t)q * Nfp + col] = (1.4142135623730951 * h1[0] * h2[0]) * pw;
        }
    }
    const std::vector<double> mf = invert(matmul(vf, transpose(vf, Nfp, Nfp), Nfp, Nfp, Nfp), Nfp);
    for (int q = 0; q < Nfp; ++q)
      for (int j = 0; j < Nfp; ++j) Emat[(size_t)Fmask[f * Nfp + q] * NF + f * Nfp + j] = mf[(size_t)q * Nfp + j];
  }
  LIFT = matmul(V, matmul(transpose(V, Np, Np), Emat, Np, Np, NF), Np, Np, NF);
}

}  // namespace dgk
