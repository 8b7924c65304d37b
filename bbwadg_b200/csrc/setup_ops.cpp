// Host-side construction of the reference-element operators (FP64), packed
// in the FP32 layouts the time-step kernels consume.
//
// Restates, with independent code:
//   Jacobi polynomials / Vandermonde   cpp/src/Basis.cpp:83-339
//   Bernstein bases                    cpp/src/Basis.cpp:505-620
//   Warp & Blend nodes                 tabulated in cpp/include/NodeData.h;
//                                      computed here by the published
//                                      Warburton (2006) warp & blend
//                                      construction
//   nodal Dr/Ds/Dt, Fmask, LIFT, Vq    cpp/src/StartUp3d.cpp:25-226
//   BB D, LIFT pieces (L0, EEL), slices cpp/src/StartUp3d.cpp:228-510
//   WADG Vq/Pq (nodal and BB)          cpp/src/WaveOKL3d.cpp:459-483, 894-897
//   curvilinear Vrq.., Prq.., Vfq, Pfq,  cpp/src/StartUp3d.cpp:98-156, 848-856,
//   VfqFace                            cpp/src/WaveOKL3d.cpp:238-242
//   sparse packing                     cpp/src/Basis.cpp:980-1007,
//                                      cpp/src/WaveOKL3d.cpp:1427-1526
// The volume and face cubature rules are inputs; when none is given a
// Stroud conical-product (collapsed Gauss-Jacobi) rule of degree 2N+1 is
// built.  The reference uses tabulated rules of the same degree
// (cpp/src/Basis.cpp:833-949); all operators except Vq/Pq are independent of
// the rule up to round-off.
#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <memory>

#include "bbwadg.h"
#include "internal.h"

namespace bbw {

// ------------------------------------------------------------ linear algebra
Mat matmul(const Mat &A, const Mat &B) {
  Mat C(A.m, B.n);
  for (int i = 0; i < A.m; ++i)
    for (int k = 0; k < A.n; ++k) {
      const double a = A(i, k);
      if (a == 0.0) continue;
      for (int j = 0; j < B.n; ++j) C(i, j) += a * B(k, j);
    }
  return C;
}

Mat transpose(const Mat &A) {
  Mat T(A.n, A.m);
  for (int i = 0; i < A.m; ++i)
    for (int j = 0; j < A.n; ++j) T(j, i) = A(i, j);
  return T;
}

double maxabs(const Mat &A) {
  double m = 0;
  for (double v : A.a) m = std::max(m, std::fabs(v));
  return m;
}

// Householder QR with column pivoting; solves min |A X - B| (A m x n, m >= n)
static Mat qr_solve(Mat A, Mat B) {
  const int m = A.m, n = A.n, nr = B.n;
  std::vector<int> perm(n);
  for (int j = 0; j < n; ++j) perm[j] = j;
  std::vector<double> cn(n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) cn[j] += A(i, j) * A(i, j);
  for (int k = 0; k < n; ++k) {
    int piv = k;
    for (int j = k + 1; j < n; ++j)
      if (cn[j] > cn[piv]) piv = j;
    if (piv != k) {
      for (int i = 0; i < m; ++i) std::swap(A(i, k), A(i, piv));
      std::swap(cn[k], cn[piv]);
      std::swap(perm[k], perm[piv]);
    }
    double nrm = 0;
    for (int i = k; i < m; ++i) nrm += A(i, k) * A(i, k);
    nrm = std::sqrt(nrm);
    if (nrm == 0.0) continue;
    const double alpha = A(k, k) > 0 ? -nrm : nrm;
    std::vector<double> v(m - k);
    for (int i = k; i < m; ++i) v[i - k] = A(i, k);
    v[0] -= alpha;
    double vn = 0;
    for (double x : v) vn += x * x;
    if (vn == 0.0) continue;
    for (int j = k; j < n; ++j) {
      double d = 0;
      for (int i = k; i < m; ++i) d += v[i - k] * A(i, j);
      d = 2 * d / vn;
      for (int i = k; i < m; ++i) A(i, j) -= d * v[i - k];
    }
    for (int j = 0; j < nr; ++j) {
      double d = 0;
      for (int i = k; i < m; ++i) d += v[i - k] * B(i, j);
      d = 2 * d / vn;
      for (int i = k; i < m; ++i) B(i, j) -= d * v[i - k];
    }
    for (int j = k + 1; j < n; ++j) {  // downdate column norms
      cn[j] = 0;
      for (int i = k + 1; i < m; ++i) cn[j] += A(i, j) * A(i, j);
    }
  }
  Mat X(n, nr);
  for (int c = 0; c < nr; ++c) {
    std::vector<double> y(n);
    for (int i = n - 1; i >= 0; --i) {
      double s = B(i, c);
      for (int j = i + 1; j < n; ++j) s -= A(i, j) * y[j];
      y[i] = s / A(i, i);
    }
    for (int i = 0; i < n; ++i) X(perm[i], c) = y[i];
  }
  return X;
}

static Mat lu_solve(Mat A, Mat B) {
  const int n = A.m, nr = B.n;
  for (int k = 0; k < n; ++k) {
    int piv = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A(i, k)) > std::fabs(A(piv, k))) piv = i;
    if (piv != k) {
      for (int j = 0; j < n; ++j) std::swap(A(k, j), A(piv, j));
      for (int j = 0; j < nr; ++j) std::swap(B(k, j), B(piv, j));
    }
    for (int i = k + 1; i < n; ++i) {
      const double l = A(i, k) / A(k, k);
      if (l == 0.0) continue;
      for (int j = k; j < n; ++j) A(i, j) -= l * A(k, j);
      for (int j = 0; j < nr; ++j) B(i, j) -= l * B(k, j);
    }
  }
  for (int c = 0; c < nr; ++c)
    for (int i = n - 1; i >= 0; --i) {
      double s = B(i, c);
      for (int j = i + 1; j < n; ++j) s -= A(i, j) * B(j, c);
      B(i, c) = s / A(i, i);
    }
  return B;
}

Mat inverse(const Mat &A) {
  Mat I(A.m, A.m);
  for (int i = 0; i < A.m; ++i) I(i, i) = 1.0;
  return lu_solve(A, I);
}

Mat mldivide(const Mat &A, const Mat &B) {
  return A.m == A.n ? lu_solve(A, B) : qr_solve(A, B);
}

Mat mrdivide(const Mat &A, const Mat &B) { return transpose(mldivide(transpose(B), transpose(A))); }

// ------------------------------------------------------------ polynomials

static double factorial(int n) {
  double f = 1;
  for (int i = 2; i <= n; ++i) f *= i;
  return f;
}

// orthonormal Jacobi polynomial of degree d w.r.t. (1-x)^a (1+x)^b on [-1,1]
Vec jacobiP(const Vec &x, double a, double b, int d) {
  const size_t nx = x.size();
  const double g0 = std::pow(2.0, a + b + 1) / (a + b + 1) * std::tgamma(a + 1) *
                    std::tgamma(b + 1) / std::tgamma(a + b + 1);
  Vec p0(nx, 1.0 / std::sqrt(g0));
  if (d == 0) return p0;
  const double g1 = (a + 1) * (b + 1) / (a + b + 3) * g0;
  Vec p1(nx);
  for (size_t i = 0; i < nx; ++i) p1[i] = ((a + b + 2) * x[i] / 2 + (a - b) / 2) / std::sqrt(g1);
  if (d == 1) return p1;
  double aold = 2 / (2 + a + b) * std::sqrt((a + 1) * (b + 1) / (a + b + 3));
  for (int i = 1; i <= d - 1; ++i) {
    const double h1 = 2 * i + a + b;
    const double anew = 2 / (h1 + 2) *
                        std::sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b) /
                                  (h1 + 1) / (h1 + 3));
    const double bnew = -(a * a - b * b) / h1 / (h1 + 2);
    Vec p2(nx);
    for (size_t j = 0; j < nx; ++j) p2[j] = (-aold * p0[j] + (x[j] - bnew) * p1[j]) / anew;
    p0.swap(p1);
    p1.swap(p2);
    aold = anew;
  }
  return p1;
}

static Vec gradJacobiP(const Vec &x, double a, double b, int d) {
  if (d == 0) return Vec(x.size(), 0.0);
  Vec p = jacobiP(x, a + 1, b + 1, d - 1);
  const double c = std::sqrt(d * (d + a + b + 1));
  for (double &v : p) v *= c;
  return p;
}

// Gauss-Jacobi rule with n+1 points: Newton with deflation on the
// orthonormal polynomial, weights from the Christoffel function.
static void jacobiGQ(double a, double b, int n, Vec &x, Vec &w) {
  const int q = n + 1;
  x.assign(q, 0.0);
  w.assign(q, 0.0);
  for (int k = 0; k < q; ++k) {
    double r = -std::cos((2.0 * k + 1) * M_PI / (2.0 * q));
    if (k > 0) r = 0.5 * (r + x[k - 1]);
    for (int it = 0; it < 200; ++it) {
      Vec xr(1, r);
      const double f = jacobiP(xr, a, b, q)[0];
      const double df = gradJacobiP(xr, a, b, q)[0];
      double s = 0;
      for (int j = 0; j < k; ++j) s += 1.0 / (r - x[j]);
      const double dx = f / (df - f * s);
      r -= dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    x[k] = r;
  }
  std::sort(x.begin(), x.end());
  for (int i = 0; i < q; ++i) {
    double s = 0;
    Vec xi(1, x[i]);
    for (int k = 0; k < q; ++k) {
      const double p = jacobiP(xi, a, b, k)[0];
      s += p * p;
    }
    w[i] = 1.0 / s;
  }
}

// Gauss-Lobatto points (n+1 of them)
static Vec jacobiGL(double a, double b, int n) {
  Vec x(n + 1);
  x[0] = -1.0;
  x[n] = 1.0;
  if (n >= 2) {
    Vec xi, wi;
    jacobiGQ(a + 1, b + 1, n - 2, xi, wi);
    for (int i = 0; i < n - 1; ++i) x[i + 1] = xi[i];
  }
  return x;
}

// ------------------------------------------------------------ nodes
static Vec evalwarp(int p, const Vec &xnodes, const Vec &xout) {
  Vec warp(xout.size(), 0.0), xeq(p + 1);
  for (int i = 0; i <= p; ++i) xeq[i] = -1.0 + 2.0 * (p - i) / p;
  for (int i = 0; i <= p; ++i) {
    for (size_t o = 0; o < xout.size(); ++o) {
      double d = xnodes[i] - xeq[i];
      for (int j = 1; j < p; ++j)
        if (i != j) d *= (xout[o] - xeq[j]) / (xeq[i] - xeq[j]);
      if (i != 0) d = -d / (xeq[i] - xeq[0]);
      if (i != p) d = d / (xeq[i] - xeq[p]);
      warp[o] += d;
    }
  }
  return warp;
}

static void evalshift(int p, double pval, const Vec &L1, const Vec &L2, const Vec &L3, Vec &dx,
                      Vec &dy) {
  // xnodes = -JacobiGL(0,0,p): Gauss-Lobatto nodes in descending order,
  // paired with the descending equispaced nodes of evalwarp
  Vec neg = jacobiGL(0, 0, p);
  for (double &v : neg) v = -v;
  const size_t n = L1.size();
  Vec a(n), b(n), c(n);
  for (size_t i = 0; i < n; ++i) a[i] = L3[i] - L2[i], b[i] = L1[i] - L3[i], c[i] = L2[i] - L1[i];
  Vec w1 = evalwarp(p, neg, a), w2 = evalwarp(p, neg, b), w3 = evalwarp(p, neg, c);
  dx.assign(n, 0.0);
  dy.assign(n, 0.0);
  for (size_t i = 0; i < n; ++i) {
    const double b1 = L2[i] * L3[i], b2 = L1[i] * L3[i], b3 = L1[i] * L2[i];
    const double warp1 = b1 * 4 * w1[i] * (1 + (pval * L1[i]) * (pval * L1[i]));
    const double warp2 = b2 * 4 * w2[i] * (1 + (pval * L2[i]) * (pval * L2[i]));
    const double warp3 = b3 * 4 * w3[i] * (1 + (pval * L3[i]) * (pval * L3[i]));
    dx[i] = warp1 + std::cos(2 * M_PI / 3) * warp2 + std::cos(4 * M_PI / 3) * warp3;
    dy[i] = std::sin(2 * M_PI / 3) * warp2 + std::sin(4 * M_PI / 3) * warp3;
  }
}

// Warp & Blend nodes on the reference tetrahedron (Warburton 2006)
void nodes3d(int N, Vec &r, Vec &s, Vec &t) {
  static const double alpopt[15] = {0, 0, 0, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577,
                                    1.1603, 1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655};
  const double alpha = N <= 15 ? alpopt[N - 1] : 1.0;
  const double tol = 1e-10;
  r.clear(), s.clear(), t.clear();
  for (int n = 0; n <= N; ++n)
    for (int m = 0; m <= N - n; ++m)
      for (int q = 0; q <= N - n - m; ++q) {
        r.push_back(-1.0 + 2.0 * q / N);
        s.push_back(-1.0 + 2.0 * m / N);
        t.push_back(-1.0 + 2.0 * n / N);
      }
  const size_t np = r.size();
  Vec L1(np), L2(np), L3(np), L4(np);
  for (size_t i = 0; i < np; ++i) {
    L1[i] = (1 + t[i]) / 2, L2[i] = (1 + s[i]) / 2;
    L3[i] = -(1 + r[i] + s[i] + t[i]) / 2, L4[i] = (1 + r[i]) / 2;
  }
  const double s3 = std::sqrt(3.0), s6 = std::sqrt(6.0);
  const double v1[3] = {-1, -1 / s3, -1 / s6}, v2[3] = {1, -1 / s3, -1 / s6},
               v3[3] = {0, 2 / s3, -1 / s6}, v4[3] = {0, 0, 3 / s6};
  double t1[4][3], t2[4][3];
  for (int d = 0; d < 3; ++d) {
    t1[0][d] = v2[d] - v1[d], t1[1][d] = v2[d] - v1[d];
    t1[2][d] = v3[d] - v2[d], t1[3][d] = v3[d] - v1[d];
    t2[0][d] = v3[d] - 0.5 * (v1[d] + v2[d]), t2[1][d] = v4[d] - 0.5 * (v1[d] + v2[d]);
    t2[2][d] = v4[d] - 0.5 * (v2[d] + v3[d]), t2[3][d] = v4[d] - 0.5 * (v1[d] + v3[d]);
  }
  for (int f = 0; f < 4; ++f) {
    double n1 = 0, n2 = 0;
    for (int d = 0; d < 3; ++d) n1 += t1[f][d] * t1[f][d], n2 += t2[f][d] * t2[f][d];
    for (int d = 0; d < 3; ++d) t1[f][d] /= std::sqrt(n1), t2[f][d] /= std::sqrt(n2);
  }
  std::vector<std::array<double, 3>> X(np), shift(np, {0, 0, 0});
  for (size_t i = 0; i < np; ++i)
    for (int d = 0; d < 3; ++d)
      X[i][d] = L3[i] * v1[d] + L4[i] * v2[d] + L2[i] * v3[d] + L1[i] * v4[d];
  for (int face = 0; face < 4; ++face) {
    const Vec *La, *Lb, *Lc, *Ld;
    if (face == 0) La = &L1, Lb = &L2, Lc = &L3, Ld = &L4;
    if (face == 1) La = &L2, Lb = &L1, Lc = &L3, Ld = &L4;
    if (face == 2) La = &L3, Lb = &L1, Lc = &L4, Ld = &L2;
    if (face == 3) La = &L4, Lb = &L1, Lc = &L3, Ld = &L2;
    Vec w1, w2;
    evalshift(N, alpha, *Lb, *Lc, *Ld, w1, w2);
    for (size_t i = 0; i < np; ++i) {
      double blend = (*Lb)[i] * (*Lc)[i] * (*Ld)[i];
      const double denom =
          ((*Lb)[i] + .5 * (*La)[i]) * ((*Lc)[i] + .5 * (*La)[i]) * ((*Ld)[i] + .5 * (*La)[i]);
      if (denom > tol)
        blend = (1 + (alpha * (*La)[i]) * (alpha * (*La)[i])) * blend / denom;
      for (int d = 0; d < 3; ++d) shift[i][d] += blend * w1[i] * t1[face][d] + blend * w2[i] * t2[face][d];
      const int cnt = ((*Lb)[i] > tol) + ((*Lc)[i] > tol) + ((*Ld)[i] > tol);
      if ((*La)[i] < tol && cnt < 3)
        for (int d = 0; d < 3; ++d) shift[i][d] = w1[i] * t1[face][d] + w2[i] * t2[face][d];
    }
  }
  // back to (r,s,t): X = 0.5*(v2+v3+v4-v1) + A [r;s;t]
  Mat A(3, 3), rhs(3, (int)np);
  for (int d = 0; d < 3; ++d) {
    A(d, 0) = 0.5 * (v2[d] - v1[d]), A(d, 1) = 0.5 * (v3[d] - v1[d]), A(d, 2) = 0.5 * (v4[d] - v1[d]);
    for (size_t i = 0; i < np; ++i)
      rhs(d, (int)i) = X[i][d] + shift[i][d] - 0.5 * (v2[d] + v3[d] + v4[d] - v1[d]);
  }
  Mat RST = mldivide(A, rhs);
  for (size_t i = 0; i < np; ++i) r[i] = RST(0, (int)i), s[i] = RST(1, (int)i), t[i] = RST(2, (int)i);
}

// ------------------------------------------------------------ bases
static void rsttoabc(const Vec &r, const Vec &s, const Vec &t, Vec &a, Vec &b, Vec &c) {
  const size_t n = r.size();
  a.resize(n), b.resize(n), c.resize(n);
  for (size_t i = 0; i < n; ++i) {
    a[i] = std::fabs(s[i] + t[i]) > 1e-8 ? 2 * (1 + r[i]) / (-s[i] - t[i]) - 1 : -1;
    b[i] = std::fabs(t[i] - 1) > 1e-8 ? 2 * (1 + s[i]) / (1 - t[i]) - 1 : -1;
    c[i] = t[i];
  }
}

Mat vandermonde3d(int N, const Vec &r, const Vec &s, const Vec &t) {
  Vec a, b, c;
  rsttoabc(r, s, t, a, b, c);
  Mat V((int)r.size(), np_of(N));
  int sk = 0;
  for (int i = 0; i <= N; ++i)
    for (int j = 0; j <= N - i; ++j)
      for (int k = 0; k <= N - i - j; ++k, ++sk) {
        Vec h1 = jacobiP(a, 0, 0, i), h2 = jacobiP(b, 2 * i + 1, 0, j),
            h3 = jacobiP(c, 2 * (i + j) + 2, 0, k);
        for (size_t p = 0; p < r.size(); ++p)
          V((int)p, sk) = 2 * std::sqrt(2.0) * h1[p] * h2[p] * std::pow(1 - b[p], i) * h3[p] *
                          std::pow(1 - c[p], i + j);
      }
  return V;
}

void gradVandermonde3d(int N, const Vec &r, const Vec &s, const Vec &t, Mat &Vr, Mat &Vs,
                              Mat &Vt) {
  Vec a, b, c;
  rsttoabc(r, s, t, a, b, c);
  const int np = (int)r.size();
  Vr = Mat(np, np_of(N)), Vs = Mat(np, np_of(N)), Vt = Mat(np, np_of(N));
  int sk = 0;
  for (int id = 0; id <= N; ++id)
    for (int jd = 0; jd <= N - id; ++jd)
      for (int kd = 0; kd <= N - id - jd; ++kd, ++sk) {
        Vec fa = jacobiP(a, 0, 0, id), dfa = gradJacobiP(a, 0, 0, id);
        Vec gb = jacobiP(b, 2 * id + 1, 0, jd), dgb = gradJacobiP(b, 2 * id + 1, 0, jd);
        Vec hc = jacobiP(c, 2 * (id + jd) + 2, 0, kd),
            dhc = gradJacobiP(c, 2 * (id + jd) + 2, 0, kd);
        const double scale = std::pow(2.0, 2 * id + jd + 1.5);
        for (int p = 0; p < np; ++p) {
          const double hb = 0.5 * (1 - b[p]), hcc = 0.5 * (1 - c[p]);
          double vr = dfa[p] * (gb[p] * hc[p]);
          if (id > 0) vr *= std::pow(hb, id - 1);
          if (id + jd > 0) vr *= std::pow(hcc, id + jd - 1);
          double tmp = dgb[p] * std::pow(hb, id);
          if (id > 0) tmp += (-0.5 * id) * (gb[p] * std::pow(hb, id - 1));
          if (id + jd > 0) tmp *= std::pow(hcc, id + jd - 1);
          tmp = fa[p] * (tmp * hc[p]);
          const double vs = 0.5 * (1 + a[p]) * vr + tmp;
          double vt = 0.5 * (1 + a[p]) * vr + 0.5 * (1 + b[p]) * tmp;
          double tmp2 = dhc[p] * std::pow(hcc, id + jd);
          if (id + jd > 0) tmp2 += -0.5 * (id + jd) * (hc[p] * std::pow(hcc, id + jd - 1));
          tmp2 = fa[p] * (gb[p] * tmp2);
          tmp2 *= std::pow(hb, id);
          vt += tmp2;
          Vr(p, sk) = vr * scale, Vs(p, sk) = vs * scale, Vt(p, sk) = vt * scale;
        }
      }
}

Mat vandermonde2d(int N, const Vec &r, const Vec &s) {
  const size_t n = r.size();
  Vec a(n), b(n);
  for (size_t i = 0; i < n; ++i) {
    a[i] = std::fabs(s[i] - 1) > 1e-8 ? 2 * (1 + r[i]) / (1 - s[i]) - 1 : -1;
    b[i] = s[i];
  }
  Mat V((int)n, nfp_of(N));
  int sk = 0;
  for (int i = 0; i <= N; ++i)
    for (int j = 0; j <= N - i; ++j, ++sk) {
      Vec h1 = jacobiP(a, 0, 0, i), h2 = jacobiP(b, 2 * i + 1, 0, j);
      for (size_t p = 0; p < n; ++p)
        V((int)p, sk) = std::sqrt(2.0) * h1[p] * h2[p] * std::pow(1 - b[p], i);
    }
  return V;
}

static Mat bernTri(int N, const Vec &r, const Vec &s) {
  const size_t n = r.size();
  Mat V((int)n, nfp_of(N));
  int sk = 0;
  for (int k = 0; k <= N; ++k)
    for (int j = 0; j <= N - k; ++j, ++sk) {
      const int i = N - j - k;
      const double C = factorial(N) / (factorial(i) * factorial(j) * factorial(k));
      for (size_t p = 0; p < n; ++p) {
        const double L1 = -(r[p] + s[p]) / 2, L2 = (1 + r[p]) / 2, L3 = (1 + s[p]) / 2;
        V((int)p, sk) = C * std::pow(L1, i) * std::pow(L2, j) * std::pow(L3, k);
      }
    }
  return V;
}

static Mat bernTet(int N, const Vec &r, const Vec &s, const Vec &t, Mat *G = nullptr) {
  const size_t n = r.size();
  Mat V((int)n, np_of(N));
  if (G)
    for (int d = 0; d < 4; ++d) G[d] = Mat((int)n, np_of(N));
  int sk = 0;
  for (int l = 0; l <= N; ++l)
    for (int k = 0; k <= N - l; ++k)
      for (int j = 0; j <= N - l - k; ++j, ++sk) {
        const int i = N - j - k - l;
        const double C = factorial(N) / (factorial(i) * factorial(j) * factorial(k) * factorial(l));
        for (size_t p = 0; p < n; ++p) {
          const double L[4] = {-(1 + r[p] + s[p] + t[p]) / 2, (1 + r[p]) / 2, (1 + s[p]) / 2,
                               (1 + t[p]) / 2};
          const int e[4] = {i, j, k, l};
          V((int)p, sk) = C * std::pow(L[0], i) * std::pow(L[1], j) * std::pow(L[2], k) *
                          std::pow(L[3], l);
          if (G)
            for (int d = 0; d < 4; ++d) {  // d/dL_d of the Bernstein polynomial
              double v = 0;
              if (e[d] > 0) {
                v = C * e[d];
                for (int q = 0; q < 4; ++q) v *= std::pow(L[q], q == d ? e[q] - 1 : e[q]);
              }
              G[d]((int)p, sk) = v;
            }
        }
      }
  return V;
}

// fixed-bandwidth sparse form: column ids / values of entries above
// 1e-5 * max|A| per row, padded with (0, 0)
static void sparse_ids(const Mat &A, std::vector<std::vector<int>> &ids,
                       std::vector<std::vector<double>> &vals, int &width) {
  const double tol = 1e-5 * maxabs(A);
  ids.assign(A.m, {});
  vals.assign(A.m, {});
  width = 0;
  for (int i = 0; i < A.m; ++i) {
    for (int j = 0; j < A.n; ++j)
      if (std::fabs(A(i, j)) > tol) ids[i].push_back(j), vals[i].push_back(A(i, j));
    width = std::max(width, (int)ids[i].size());
  }
}

// Stroud conical product rules of degree 2q-1 (q points per direction)
static void stroud_tet(int q, Vec &r, Vec &s, Vec &t, Vec &w) {
  Vec a, wa, b, wb, c, wc;
  jacobiGQ(0, 0, q - 1, a, wa);
  jacobiGQ(1, 0, q - 1, b, wb);
  jacobiGQ(2, 0, q - 1, c, wc);
  r.clear(), s.clear(), t.clear(), w.clear();
  for (int k = 0; k < q; ++k)
    for (int j = 0; j < q; ++j)
      for (int i = 0; i < q; ++i) {
        r.push_back((1 + a[i]) * (1 - b[j]) * (1 - c[k]) / 4 - 1);
        s.push_back((1 + b[j]) * (1 - c[k]) / 2 - 1);
        t.push_back(c[k]);
        w.push_back(wa[i] * wb[j] * wc[k] / 8);
      }
}

static void stroud_tri(int q, Vec &r, Vec &s, Vec &w) {
  Vec a, wa, b, wb;
  jacobiGQ(0, 0, q - 1, a, wa);
  jacobiGQ(1, 0, q - 1, b, wb);
  r.clear(), s.clear(), w.clear();
  for (int j = 0; j < q; ++j)
    for (int i = 0; i < q; ++i) {
      r.push_back((1 + a[i]) * (1 - b[j]) / 2 - 1);
      s.push_back(b[j]);
      w.push_back(wa[i] * wb[j] / 2);
    }
}

// ------------------------------------------------------------ operator set
struct OpSet {
  std::map<std::string, std::vector<double>> f64;
  std::map<std::string, std::vector<float>> f32;
  std::map<std::string, std::vector<int>> i32;
};

static std::vector<double> colmajor(const Mat &A) {
  std::vector<double> v((size_t)A.m * A.n);
  for (int j = 0; j < A.n; ++j)
    for (int i = 0; i < A.m; ++i) v[(size_t)j * A.m + i] = A(i, j);
  return v;
}

static std::vector<float> to_f32(const std::vector<double> &v) {
  return std::vector<float>(v.begin(), v.end());
}

static int build(int N, const double *cub, int Nq_in, const double *tri, int Nfq_in, OpSet &o) {
  const int Np = np_of(N), Nfp = nfp_of(N);
  const double NODETOL = 1e-6;  // cpp/include/Mesh.h:13
  Vec r, s, t;
  nodes3d(N, r, s, t);
  Mat V = vandermonde3d(N, r, s, t);
  Mat Vr, Vs, Vt;
  gradVandermonde3d(N, r, s, t, Vr, Vs, Vt);
  Mat Dr = mrdivide(Vr, V), Ds = mrdivide(Vs, V), Dt = mrdivide(Vt, V);

  // Fmask, face-major (cpp/src/StartUp3d.cpp:41-56)
  std::vector<int> Fmask(4 * Nfp);
  int cnt[4] = {0, 0, 0, 0};
  for (int i = 0; i < Np; ++i) {
    const bool on[4] = {std::fabs(1 + t[i]) < NODETOL, std::fabs(1 + s[i]) < NODETOL,
                        std::fabs(1 + r[i] + s[i] + t[i]) < NODETOL, std::fabs(1 + r[i]) < NODETOL};
    for (int f = 0; f < 4; ++f)
      if (on[f]) {
        if (cnt[f] >= Nfp) return BBW_ERR_NUMERIC;
        Fmask[f * Nfp + cnt[f]++] = i;
      }
  }
  for (int f = 0; f < 4; ++f)
    if (cnt[f] != Nfp) return BBW_ERR_NUMERIC;

  // cubature rules
  Vec rq, sq, tq, wq, rt, st, wt;
  if (cub && Nq_in > 0) {
    rq.assign(cub, cub + Nq_in), sq.assign(cub + Nq_in, cub + 2 * Nq_in);
    tq.assign(cub + 2 * Nq_in, cub + 3 * Nq_in), wq.assign(cub + 3 * Nq_in, cub + 4 * Nq_in);
  } else {
    stroud_tet(N + 1, rq, sq, tq, wq);
  }
  if (tri && Nfq_in > 0) {
    rt.assign(tri, tri + Nfq_in), st.assign(tri + Nfq_in, tri + 2 * Nfq_in);
    wt.assign(tri + 2 * Nfq_in, tri + 3 * Nfq_in);
  } else {
    stroud_tri(N + 1, rt, st, wt);
  }
  const int Nq = (int)rq.size(), Nfq = (int)rt.size();

  // nodal LIFT (cpp/src/StartUp3d.cpp:188-202)
  Mat Emat(Np, 4 * Nfp);
  for (int f = 0; f < 4; ++f) {
    Vec rf(Nfp), sf(Nfp);
    for (int i = 0; i < Nfp; ++i) {
      const int v = Fmask[f * Nfp + i];
      if (f == 0) rf[i] = r[v], sf[i] = s[v];
      if (f == 1) rf[i] = r[v], sf[i] = t[v];
      if (f >= 2) rf[i] = s[v], sf[i] = t[v];
    }
    Mat Vf = vandermonde2d(N, rf, sf);
    Mat Mf = inverse(matmul(Vf, transpose(Vf)));
    for (int i = 0; i < Nfp; ++i)
      for (int j = 0; j < Nfp; ++j) Emat(Fmask[f * Nfp + i], j + f * Nfp) += Mf(i, j);
  }
  Mat invM = matmul(V, transpose(V));
  Mat LIFT = matmul(invM, Emat);

  // WADG interpolation / projection (cpp/src/WaveOKL3d.cpp:459-483, 894-897)
  Mat Vq = mrdivide(vandermonde3d(N, rq, sq, tq), V);
  Mat VqtW = transpose(Vq);
  for (int i = 0; i < Np; ++i)
    for (int q = 0; q < Nq; ++q) VqtW(i, q) *= wq[q];
  Mat Pq = matmul(invM, VqtW);
  Mat VBq = bernTet(N, rq, sq, tq);
  Mat VBqtW = transpose(VBq);
  for (int i = 0; i < Np; ++i)
    for (int q = 0; q < Nq; ++q) VBqtW(i, q) *= wq[q];
  Mat MB = matmul(VBqtW, VBq);
  Mat PqB = mldivide(MB, VBqtW);

  // curvilinear WADG operators (cpp/src/StartUp3d.cpp:98-156, 848-856;
  // cpp/src/WaveOKL3d.cpp:238-242): derivative interpolants at the volume
  // cubature, their weighted projections, interpolation to the face
  // cubature of all four faces and the face-node -> face-cubature map
  Mat Vrq, Vsq, Vtq;
  {
    Mat a, b, c;
    gradVandermonde3d(N, rq, sq, tq, a, b, c);
    Vrq = mrdivide(a, V), Vsq = mrdivide(b, V), Vtq = mrdivide(c, V);
  }
  auto weighted_proj = [&](const Mat &A, const Vec &w) {
    Mat T = transpose(A);
    for (int i = 0; i < T.m; ++i)
      for (int q = 0; q < T.n; ++q) T(i, q) *= w[q];
    return matmul(invM, T);
  };
  Mat Prq = weighted_proj(Vrq, wq), Psq = weighted_proj(Vsq, wq), Ptq = weighted_proj(Vtq, wq);
  Vec rfa(4 * Nfq), sfa(4 * Nfq), tfa(4 * Nfq), wfa(4 * Nfq);
  for (int q = 0; q < Nfq; ++q) {
    const double a = rt[q], b = st[q];
    const double pts[4][3] = {{a, b, -1.0}, {a, -1.0, b}, {-(1 + a + b), a, b}, {-1.0, a, b}};
    for (int f = 0; f < 4; ++f)
      rfa[f * Nfq + q] = pts[f][0], sfa[f * Nfq + q] = pts[f][1], tfa[f * Nfq + q] = pts[f][2],
                    wfa[f * Nfq + q] = wt[q];
  }
  Mat Vfq = mrdivide(vandermonde3d(N, rfa, sfa, tfa), V);
  Mat Pfq = weighted_proj(Vfq, wfa);
  Mat VfqFace;
  {
    Vec rf0(Nfp), sf0(Nfp);
    for (int i = 0; i < Nfp; ++i) rf0[i] = r[Fmask[i]], sf0[i] = s[Fmask[i]];
    VfqFace = mrdivide(vandermonde2d(N, rt, st), vandermonde2d(N, rf0, sf0));
  }

  // Bernstein derivative operators (cpp/src/StartUp3d.cpp:228-282)
  Mat G[4];
  Mat VB = bernTet(N, r, s, t, G);
  Mat invVB = inverse(VB);
  std::vector<std::vector<int>> Dids[4];
  std::vector<std::vector<double>> Dvals[4];
  for (int d = 0; d < 4; ++d) {
    int w;
    sparse_ids(mldivide(VB, G[d]), Dids[d], Dvals[d], w);
    if (w > 4) return BBW_ERR_NUMERIC;
  }
  // BB lift: L0 and the scaled degree-elevation EEL (:285-407)
  Mat VfB = bernTri(N, rt, st);
  Mat VfBtW = transpose(VfB);
  for (int i = 0; i < Nfp; ++i)
    for (int q = 0; q < Nfq; ++q) VfBtW(i, q) *= wt[q];
  Mat massFaceB = matmul(VfBtW, VfB);
  Mat EmatB(Np, 4 * Nfp);
  for (int f = 0; f < 4; ++f)
    for (int i = 0; i < Nfp; ++i)
      for (int j = 0; j < Nfp; ++j) EmatB(Fmask[f * Nfp + i], j + f * Nfp) += massFaceB(i, j);
  Mat LIFTB = mldivide(MB, EmatB);
  std::vector<double> cEL(N + 1);
  Mat EEL1(Np, Nfp);
  {
    int off = 0;
    for (int i = 0; i <= N; ++i) {
      const int NpElev = nfp_of(N - i);
      Mat Ei = mldivide(VfB, bernTri(N - i, rt, st));  // Nfp x NpElev
      cEL[i] = ((i % 2) ? -1.0 : 1.0) * (factorial(N) / (factorial(N - i) * factorial(i))) / (1 + i);
      for (int a = 0; a < NpElev; ++a)
        for (int b = 0; b < Nfp; ++b) EEL1(off + a, b) = cEL[i] * Ei(b, a);
      off += NpElev;
    }
  }
  const double maxL = maxabs(LIFTB);
  std::vector<int> rowperm((size_t)Np * 3);
  for (int f = 1; f < 4; ++f)
    for (int i = 0; i < Np; ++i) {
      int row = -1;
      for (int cand = 0; cand < Np && row < 0; ++cand) {
        double d = 0;
        for (int j = 0; j < Nfp; ++j)
          d = std::max(d, std::fabs(LIFTB(cand, j) - LIFTB(i, f * Nfp + j)));
        if (d < NODETOL * maxL) row = cand;
      }
      if (row < 0) return BBW_ERR_NUMERIC;
      rowperm[(size_t)i * 3 + f - 1] = row;
    }
  Mat EEL(Np, 4 * Nfp);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Nfp; ++j) {
      EEL(i, j) = EEL1(i, j);
      for (int f = 1; f < 4; ++f) EEL(i, f * Nfp + j) = EEL1(rowperm[(size_t)i * 3 + f - 1], j);
    }
  std::vector<std::vector<int>> Eids, Lids;
  std::vector<std::vector<double>> Evals, Lvals;
  int Ew, Lw;
  sparse_ids(EEL, Eids, Evals, Ew);
  Mat L0(Nfp, Nfp);
  for (int i = 0; i < Nfp; ++i)
    for (int j = 0; j < Nfp; ++j) L0(i, j) = LIFTB(i, j);
  sparse_ids(L0, Lids, Lvals, Lw);
  const int EEL_nnz = Nfp + 3, L0_nnz = std::min(Nfp, 7);

  // slice ids (cpp/src/StartUp3d.cpp:419-457)
  auto MAPJ = [](int NN, int JJ) { return (NN + 1) * JJ - JJ * (JJ + 1) / 2 + JJ; };
  auto MAPK = [](int NN, int KK) { return KK * (3 * NN * (NN - KK + 4) + KK * (KK - 6) + 11) / 6; };
  std::vector<int> slice_ids((size_t)Np * 4);
  {
    int sk = 0;
    for (int sl = 0; sl <= N; ++sl)
      for (int j = 0; j <= N - sl; ++j)
        for (int i = 0; i <= N - sl - j; ++i, ++sk) {
          slice_ids[4 * sk + 0] = i + MAPJ(N - sl, j) + MAPK(N, sl);
          slice_ids[4 * sk + 1] = i + MAPJ(N - j, sl) + MAPK(N, j);
          slice_ids[4 * sk + 2] = (N - sl - i - j) + MAPJ(N - j, i) + MAPK(N, j);
          slice_ids[4 * sk + 3] = sl + MAPJ(N - j, i) + MAPK(N, j);
        }
  }
  // slice-by-slice degree reductions (:460-509)
  std::vector<double> eel_val_vec;
  std::vector<int> eel_id_vec;
  for (int i = 0; i < N; ++i) {
    Mat Ei = mldivide(bernTri(N - i, rt, st), bernTri(N - i - 1, rt, st));
    std::vector<std::vector<int>> ids;
    std::vector<std::vector<double>> vals;
    int w;
    sparse_ids(transpose(Ei), ids, vals, w);
    const int rows = (int)ids.size(), wc = std::max(w, 3);
    for (int c = 0; c < wc; ++c)
      for (int q = 0; q < rows; ++q) {
        const bool has = c < (int)ids[q].size();
        eel_val_vec.push_back(has ? vals[q][c] : 0.0);
        eel_id_vec.push_back(has ? ids[q][c] : 0);
      }
  }

  // ---- pack (FP64 column-major for the oracle, FP32 in kernel layouts)
  o.f64["r"] = r, o.f64["s"] = s, o.f64["t"] = t;
  o.f64["rq"] = rq, o.f64["sq"] = sq, o.f64["tq"] = tq, o.f64["wq"] = wq;
  o.f64["rfq"] = rt, o.f64["sfq"] = st, o.f64["wfq"] = wt;
  o.f64["V"] = colmajor(V), o.f64["Dr"] = colmajor(Dr), o.f64["Ds"] = colmajor(Ds);
  o.f64["Dt"] = colmajor(Dt), o.f64["LIFT"] = colmajor(LIFT);
  o.f64["Vq_nodal"] = colmajor(Vq), o.f64["Pq_nodal"] = colmajor(Pq);
  o.f64["Vq_bb"] = colmajor(VBq), o.f64["Pq_bb"] = colmajor(PqB);
  o.f64["VB"] = colmajor(VB), o.f64["invVB"] = colmajor(invVB);
  o.f64["LIFTB"] = colmajor(LIFTB), o.f64["EEL"] = colmajor(EEL);
  o.f64["cEL"] = cEL;
  o.f64["EEL_val_vec"] = eel_val_vec;
  o.f64["Vrq"] = colmajor(Vrq), o.f64["Vsq"] = colmajor(Vsq), o.f64["Vtq"] = colmajor(Vtq);
  o.f64["Prq"] = colmajor(Prq), o.f64["Psq"] = colmajor(Psq), o.f64["Ptq"] = colmajor(Ptq);
  o.f64["Vfq"] = colmajor(Vfq), o.f64["Pfq"] = colmajor(Pfq), o.f64["VfqFace"] = colmajor(VfqFace);
  for (const char *k : {"Dr", "Ds", "Dt", "LIFT", "Vq_nodal", "Pq_nodal", "Vq_bb", "Pq_bb", "cEL",
                        "Vrq", "Vsq", "Vtq", "Prq", "Psq", "Ptq", "Vfq", "Pfq", "VfqFace"})
    o.f32[k] = to_f32(o.f64[k]);
  o.i32["Fmask"] = Fmask;
  o.i32["slice_ids"] = slice_ids;
  o.i32["EEL_id_vec"] = eel_id_vec;
  o.i32["faceVolPerm"] = rowperm;
  // D ids packed as in cpp/src/WaveOKL3d.cpp:1452-1476; values from D4
  for (int j = 0; j < 4; ++j) {
    std::vector<int> v((size_t)Np * 4, 0);
    for (int i = 0; i < Np; ++i)
      for (int m = 0; m < 4; ++m)
        v[4 * i + m] = j < (int)Dids[m][i].size() ? Dids[m][i][j] : 0;
    o.i32["D_ids" + std::to_string(j + 1)] = v;
  }
  {
    std::vector<float> v((size_t)Np * 4, 0.f);
    std::vector<double> v64((size_t)Np * 4, 0.0);
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < 4 && j < (int)Dvals[3][i].size(); ++j)
        v[4 * i + j] = (float)Dvals[3][i][j], v64[4 * i + j] = Dvals[3][i][j];
    o.f32["Dvals4"] = v;
    o.f64["Dvals4"] = v64;
  }
  {
    std::vector<int> ids((size_t)Np * EEL_nnz, 0);
    std::vector<double> vals((size_t)Np * EEL_nnz, 0.0);
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < EEL_nnz && j < (int)Eids[i].size(); ++j)
        ids[i + (size_t)j * Np] = Eids[i][j], vals[i + (size_t)j * Np] = Evals[i][j];
    o.i32["EEL_ids"] = ids;
    o.f64["EEL_vals"] = vals;
    o.f32["EEL_vals"] = to_f32(vals);
  }
  {
    std::vector<int> ids((size_t)Nfp * L0_nnz, 0);
    std::vector<double> vals((size_t)Nfp * L0_nnz, 0.0);
    for (int i = 0; i < Nfp; ++i)
      for (int j = 0; j < L0_nnz && j < (int)Lids[i].size(); ++j)
        ids[i + (size_t)j * Nfp] = Lids[i][j], vals[i + (size_t)j * Nfp] = Lvals[i][j];
    o.i32["L0_ids"] = ids;
    o.f64["L0_vals"] = vals;
    o.f32["L0_vals"] = to_f32(vals);
  }
  o.i32["sizes"] = {N, Np, Nfp, Nq, Nfq, EEL_nnz, L0_nnz, Ew, Lw};
  return BBW_OK;
}

}  // namespace bbw

struct bbw_ops {
  bbw::OpSet set;
};

extern "C" bbw_status bbw_ops_build(int N, const double *cub, int Nq, const double *tri, int Nfq,
                                    bbw_ops **out) {
  if (!out || N < 1 || N > BBW_MAX_N) return BBW_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<bbw_ops> o(new bbw_ops);
  int rc = bbw::build(N, cub, Nq, tri, Nfq, o->set);
  if (rc != BBW_OK) return (bbw_status)rc;
  *out = o.release();
  return BBW_OK;
}

extern "C" bbw_status bbw_ops_get(const bbw_ops *o, const char *name, int dtype, void *dst,
                                  long long *count) {
  if (!o || !name || !count) return BBW_ERR_ARG;
  const std::string k(name);
  const void *src = nullptr;
  size_t n = 0, esz = 0;
  if (dtype == 0) {
    auto it = o->set.f32.find(k);
    if (it == o->set.f32.end()) return BBW_ERR_ARG;
    src = it->second.data(), n = it->second.size(), esz = 4;
  } else if (dtype == 1) {
    auto it = o->set.f64.find(k);
    if (it == o->set.f64.end()) return BBW_ERR_ARG;
    src = it->second.data(), n = it->second.size(), esz = 8;
  } else if (dtype == 2) {
    auto it = o->set.i32.find(k);
    if (it == o->set.i32.end()) return BBW_ERR_ARG;
    src = it->second.data(), n = it->second.size(), esz = 4;
  } else {
    return BBW_ERR_ARG;
  }
  if (dst) {
    if (*count < (long long)n) return BBW_ERR_ARG;
    std::memcpy(dst, src, n * esz);
  }
  *count = (long long)n;
  return BBW_OK;
}

extern "C" void bbw_ops_free(bbw_ops *o) { delete o; }

extern "C" bbw_status bbw_basis_eval(int N, int variant, int npts, const double *r,
                                     const double *s, const double *t, double *out) {
  if (N < 1 || N > BBW_MAX_N || npts < 0 || (npts > 0 && (!r || !s || !t || !out)) ||
      (variant != BBW_NODAL && variant != BBW_BB))
    return BBW_ERR_ARG;
  if (npts == 0) return BBW_OK;
  bbw::Vec rr(r, r + npts), ss(s, s + npts), tt(t, t + npts);
  bbw::Mat B;
  if (variant == BBW_NODAL) {
    bbw::Vec rn, sn, tn;
    bbw::nodes3d(N, rn, sn, tn);
    B = bbw::mrdivide(bbw::vandermonde3d(N, rr, ss, tt), bbw::vandermonde3d(N, rn, sn, tn));
  } else {
    B = bbw::bernTet(N, rr, ss, tt);
  }
  const int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  for (int i = 0; i < npts; ++i)
    for (int n = 0; n < Np; ++n) out[(size_t)i * Np + n] = B(i, n);
  return BBW_OK;
}
