// Internal host-side helpers shared by the setup and runtime translation units.
#pragma once
#include <cmath>
#include <string>
#include <vector>

namespace bbw {

inline int np_of(int N) { return (N + 1) * (N + 2) * (N + 3) / 6; }
inline int nfp_of(int N) { return (N + 1) * (N + 2) / 2; }

// Dense row-major matrix for the FP64 operator construction.
struct Mat {
  int m = 0, n = 0;
  std::vector<double> a;
  Mat() {}
  Mat(int m_, int n_, double v = 0.0) : m(m_), n(n_), a((size_t)m_ * n_, v) {}
  double &operator()(int i, int j) { return a[(size_t)i * n + j]; }
  double operator()(int i, int j) const { return a[(size_t)i * n + j]; }
};

Mat matmul(const Mat &A, const Mat &B);
Mat transpose(const Mat &A);
Mat inverse(const Mat &A);                 // LU with partial pivoting
Mat mldivide(const Mat &A, const Mat &B);  // A\B: square solve or least squares
Mat mrdivide(const Mat &A, const Mat &B);  // A/B = (B'\A')'
double maxabs(const Mat &A);

typedef std::vector<double> Vec;
// orthonormal Jacobi polynomial of degree d for weight (1-x)^a (1+x)^b
Vec jacobiP(const Vec &x, double a, double b, int d);
// Warp & Blend nodes of the reference tetrahedron (vertices (-1,-1,-1),
// (1,-1,-1), (-1,1,-1), (-1,-1,1)) in the reference's node order
void nodes3d(int N, Vec &r, Vec &s, Vec &t);
// orthonormal simplex bases at the given points (rows) and their gradients
Mat vandermonde3d(int N, const Vec &r, const Vec &s, const Vec &t);
void gradVandermonde3d(int N, const Vec &r, const Vec &s, const Vec &t, Mat &Vr, Mat &Vs, Mat &Vt);
Mat vandermonde2d(int N, const Vec &r, const Vec &s);

}  // namespace bbw
