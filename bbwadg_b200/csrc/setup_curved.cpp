// Host-side setup of the curvilinear WADG path (FP64): Gordon-Hall curving
// of the elements that touch the unit sphere, and the geometric factors at
// the volume and face cubature points.
//
// Restates, with independent code:
//   GordonHallSphere                   cpp/src/WaveOKL3d.cpp:929-1231
//   hierarchical (vertex/edge/face)    cpp/src/Basis.cpp:343-416
//   basis of the blend
//   InitQuadratureArrays geofacs       cpp/src/StartUp3d.cpp:829-909,
//                                      cpp/src/Basis.cpp:625-723
//   vgeoq / fgeoq packing              cpp/src/WaveOKL3d.cpp:211-233
//
// The blend matrices (hierarchical functions at all nodes times the inverse
// of their values at the interior edge / face nodes) depend only on the span
// of the edge and face functions, so any basis of that span gives the same
// curving.  The face functions are the face bubble times all polynomials of
// degree N-3 in the two face coordinates (-L1+L2-L3, -L1-L2+L3) of the
// face's barycentrics.  The reference takes its second face coordinate from
// element 2 of a 2-vector (cpp/src/Basis.cpp:353-354); that value only
// matters for N >= 4, where the reference's curving is undefined, and is
// unused for N <= 3, where this code reproduces it.
#include <cmath>
#include <vector>

#include "bbwadg.h"
#include "internal.h"

namespace bbw {
namespace {

const double kGeoTol = 1e-6;  // cpp/src/WaveOKL3d.cpp:960

// edge e = (eA[e], eB[e]) and face f = (fA, fB, fC) vertex triples of the
// hierarchical basis (cpp/src/Basis.cpp:372-378, 396-400)
const int kHierEdges[6][2] = {{0, 3}, {1, 3}, {2, 3}, {0, 1}, {1, 2}, {2, 0}};
const int kHierFaces[4][3] = {{0, 1, 3}, {1, 2, 3}, {2, 0, 3}, {0, 1, 2}};

struct NodeSets {
  Vec r, s, t;
  std::vector<int> Fmask;                  // [4][Nfp]
  std::vector<std::vector<int>> edge;      // [6][N+1] nodes on each edge, index order
  std::vector<std::vector<int>> face_int;  // [4][(N-1)(N-2)/2] interior face nodes
};

int node_sets(int N, NodeSets &ns) {
  const int Np = np_of(N), Nfp = nfp_of(N);
  nodes3d(N, ns.r, ns.s, ns.t);
  const Vec &r = ns.r, &s = ns.s, &t = ns.t;
  ns.Fmask.assign(4 * Nfp, 0);
  int cnt[4] = {0, 0, 0, 0};
  for (int i = 0; i < Np; ++i) {
    const bool on[4] = {std::fabs(1 + t[i]) < kGeoTol, std::fabs(1 + s[i]) < kGeoTol,
                        std::fabs(1 + r[i] + s[i] + t[i]) < kGeoTol, std::fabs(1 + r[i]) < kGeoTol};
    for (int f = 0; f < 4; ++f)
      if (on[f]) {
        if (cnt[f] >= Nfp) return BBW_ERR_NUMERIC;
        ns.Fmask[f * Nfp + cnt[f]++] = i;
      }
  }
  // edges in the curving's order (cpp/src/WaveOKL3d.cpp:962-999)
  ns.edge.assign(6, {});
  for (int i = 0; i < Np; ++i) {
    const bool on[6] = {std::fabs(s[i] + 1) + std::fabs(t[i] + 1) < kGeoTol,
                        std::fabs(r[i] + s[i]) < kGeoTol,
                        std::fabs(r[i] + 1) + std::fabs(t[i] + 1) < kGeoTol,
                        std::fabs(r[i] + 1) + std::fabs(s[i] + 1) < kGeoTol,
                        std::fabs(r[i] + t[i]) < kGeoTol, std::fabs(s[i] + t[i]) < kGeoTol};
    for (int e = 0; e < 6; ++e)
      if (on[e]) ns.edge[e].push_back(i);
  }
  for (int e = 0; e < 6; ++e)
    if ((int)ns.edge[e].size() != N + 1) return BBW_ERR_NUMERIC;
  // interior face nodes by lattice index (cpp/src/WaveOKL3d.cpp:1001-1025)
  ns.face_int.assign(4, {});
  int sk = 0;
  for (int k = 0; k <= N; ++k)
    for (int j = 0; j <= N - k; ++j)
      for (int i = 0; i <= N - j - k; ++i, ++sk) {
        if (k == 0 && i > 0 && j > 0 && i + j < N) ns.face_int[0].push_back(sk);
        if (j == 0 && i > 0 && k > 0 && i + k < N) ns.face_int[1].push_back(sk);
        if (i + j + k == N && i > 0 && j > 0 && i + j < N) ns.face_int[2].push_back(sk);
        if (i == 0 && k > 0 && j > 0 && j + k < N) ns.face_int[3].push_back(sk);
      }
  return BBW_OK;
}

// hierarchical edge and face functions at the nodes (columns edge- / face-major)
void hier_functions(int N, const NodeSets &ns, Mat &edgeF, Mat &faceF) {
  const int Np = np_of(N);
  std::vector<Vec> L(4, Vec(Np));
  for (int i = 0; i < Np; ++i) {
    L[0][i] = -(1.0 + ns.r[i] + ns.s[i] + ns.t[i]) / 2.0;
    L[1][i] = (1.0 + ns.r[i]) / 2.0;
    L[2][i] = (1.0 + ns.s[i]) / 2.0;
    L[3][i] = (1.0 + ns.t[i]) / 2.0;
  }
  const int ne = std::max(N - 1, 0), nf = N >= 3 ? nfp_of(N - 3) : 0;
  edgeF = Mat(Np, 6 * ne), faceF = Mat(Np, 4 * nf);
  for (int e = 0; e < 6; ++e) {
    const Vec &a = L[kHierEdges[e][0]], &b = L[kHierEdges[e][1]];
    Vec d(Np);
    for (int i = 0; i < Np; ++i) d[i] = a[i] - b[i];
    for (int p = 0; p < ne; ++p) {
      Vec P = jacobiP(d, 0, 0, p);
      for (int i = 0; i < Np; ++i) edgeF(i, e * ne + p) = a[i] * b[i] * P[i];
    }
  }
  for (int f = 0; f < 4 && nf > 0; ++f) {
    const Vec &a = L[kHierFaces[f][0]], &b = L[kHierFaces[f][1]], &c = L[kHierFaces[f][2]];
    Vec fr(Np), fs(Np);
    for (int i = 0; i < Np; ++i) fr[i] = -a[i] + b[i] - c[i], fs[i] = -a[i] - b[i] + c[i];
    Mat V2 = vandermonde2d(N - 3, fr, fs);
    for (int p = 0; p < nf; ++p)
      for (int i = 0; i < Np; ++i) faceF(i, f * nf + p) = a[i] * b[i] * c[i] * V2(i, p);
  }
}

Mat rows_of(const Mat &A, const std::vector<int> &rows) {
  Mat B((int)rows.size(), A.n);
  for (int i = 0; i < B.m; ++i)
    for (int j = 0; j < A.n; ++j) B(i, j) = A(rows[i], j);
  return B;
}

// rx..tz, J at the points where Dr/Ds/Dt (rows) evaluate derivatives
// (cpp/src/Basis.cpp:625-662); out[c][p] with c = rx,sx,tx,ry,sy,ty,rz,sz,tz,J
void geofacs(const Mat &Dr, const Mat &Ds, const Mat &Dt, const double *x, const double *y,
             const double *z, std::vector<Vec> &out) {
  const int np = Dr.m, n = Dr.n;
  out.assign(10, Vec(np));
  for (int p = 0; p < np; ++p) {
    double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // d[coord][r,s,t]
    for (int m = 0; m < n; ++m) {
      const double a = Dr(p, m), b = Ds(p, m), c = Dt(p, m);
      d[0][0] += a * x[m], d[0][1] += b * x[m], d[0][2] += c * x[m];
      d[1][0] += a * y[m], d[1][1] += b * y[m], d[1][2] += c * y[m];
      d[2][0] += a * z[m], d[2][1] += b * z[m], d[2][2] += c * z[m];
    }
    const double xr = d[0][0], xs = d[0][1], xt = d[0][2];
    const double yr = d[1][0], ys = d[1][1], yt = d[1][2];
    const double zr = d[2][0], zs = d[2][1], zt = d[2][2];
    const double J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
    out[0][p] = (ys * zt - zs * yt) / J;    // rx
    out[3][p] = -(xs * zt - zs * xt) / J;   // ry
    out[6][p] = (xs * yt - ys * xt) / J;    // rz
    out[1][p] = -(yr * zt - zr * yt) / J;   // sx
    out[4][p] = (xr * zt - zr * xt) / J;    // sy
    out[7][p] = -(xr * yt - yr * xt) / J;   // sz
    out[2][p] = (yr * zs - zr * ys) / J;    // tx
    out[5][p] = -(xr * zs - zr * xs) / J;   // ty
    out[8][p] = (xr * ys - yr * xs) / J;    // tz
    out[9][p] = J;
  }
}

}  // namespace
}  // namespace bbw

using namespace bbw;

extern "C" bbw_status bbw_gordon_hall_sphere(int N, int K, const int *EToF, double *x, double *y,
                                             double *z, int *curved) {
  if (N < 1 || N > BBW_MAX_N || K < 1 || !EToF || !x || !y || !z || !curved) return BBW_ERR_ARG;
  NodeSets ns;
  int rc = node_sets(N, ns);
  if (rc != BBW_OK) return (bbw_status)rc;
  const int Np = np_of(N), Nfp = nfp_of(N), ne = N - 1;
  Mat edgeF, faceF;
  hier_functions(N, ns, edgeF, faceF);
  std::vector<int> eint, fint;
  for (int e = 0; e < 6; ++e)
    for (int i = 1; i < N; ++i) eint.push_back(ns.edge[e][i]);
  for (int f = 0; f < 4; ++f)
    for (int id : ns.face_int[f]) fint.push_back(id);
  Mat edgeBlend = ne > 0 ? mrdivide(edgeF, rows_of(edgeF, eint)) : Mat();
  Mat faceBlend = fint.empty() ? Mat() : mrdivide(faceF, rows_of(faceF, fint));
  double *X[3] = {x, y, z};
  auto radius = [&](size_t id) {
    return std::sqrt(x[id] * x[id] + y[id] * y[id] + z[id] * z[id]);
  };
  std::vector<double> xc[3];
  for (int k = 0; k < K; ++k) {
    const size_t o = (size_t)k * Np;
    bool edge_c = false, face_c = false;
    for (int c = 0; c < 3; ++c) xc[c].assign(X[c] + o, X[c] + o + Np);
    // snap the nodes of every edge whose end points lie on the sphere
    for (int e = 0; e < 6; ++e) {
      const int a = ns.edge[e][0], b = ns.edge[e][N];
      if (std::fabs(radius(o + a) - 1.0) < kGeoTol && std::fabs(radius(o + b) - 1.0) < kGeoTol) {
        edge_c = true;
        for (int id : ns.edge[e]) {
          const double rb = radius(o + id);
          for (int c = 0; c < 3; ++c) xc[c][id] = X[c][o + id] / rb;
        }
      }
    }
    if (edge_c && ne > 0) {  // blend the interior-edge displacements into the element
      Vec d[3];
      for (int c = 0; c < 3; ++c) {
        d[c].resize(eint.size());
        for (size_t i = 0; i < eint.size(); ++i) d[c][i] = xc[c][eint[i]] - X[c][o + eint[i]];
      }
      for (int n = 0; n < Np; ++n)
        for (int c = 0; c < 3; ++c) {
          double acc = 0;
          for (size_t i = 0; i < eint.size(); ++i) acc += edgeBlend(n, (int)i) * d[c][i];
          X[c][o + n] += acc;
        }
    }
    if (N > 2) {
      for (int c = 0; c < 3; ++c) xc[c].assign(X[c] + o, X[c] + o + Np);
      for (int f = 0; f < 4; ++f) {
        const int *Fm = &ns.Fmask[f * Nfp];
        const int v3[3] = {Fm[0], Fm[N], Fm[Nfp - 1]};
        bool on = true;
        for (int v : v3) on = on && std::fabs(radius(o + v) - 1.0) < kGeoTol;
        if (!on) continue;
        face_c = true;
        for (int i = 0; i < Nfp; ++i) {
          const double rb = radius(o + Fm[i]);
          for (int c = 0; c < 3; ++c) xc[c][Fm[i]] = X[c][o + Fm[i]] / rb;
        }
      }
      if (face_c) {
        Vec d[3];
        for (int c = 0; c < 3; ++c) d[c].assign(fint.size(), 0.0);
        size_t sk = 0;
        for (int f = 0; f < 4; ++f)
          for (int id : ns.face_int[f]) {
            if (EToF[4 * (size_t)k + f] == f)  // boundary faces only
              for (int c = 0; c < 3; ++c) d[c][sk] = xc[c][id] - X[c][o + id];
            ++sk;
          }
        for (int n = 0; n < Np; ++n)
          for (int c = 0; c < 3; ++c) {
            double acc = 0;
            for (size_t i = 0; i < fint.size(); ++i) acc += faceBlend(n, (int)i) * d[c][i];
            X[c][o + n] += acc;
          }
      }
    }
    curved[k] = (edge_c || face_c) ? 1 : 0;
  }
  return BBW_OK;
}

extern "C" bbw_status bbw_curved_geometry(int N, int K, const double *x, const double *y,
                                          const double *z, int Nq, const double *cub, int Nfq,
                                          const double *tri, double *vgeoq, double *Jq,
                                          double *fgeoq) {
  if (N < 1 || N > BBW_MAX_N || K < 1 || Nq < 1 || Nfq < 1 || !x || !y || !z || !cub || !tri ||
      !vgeoq || !Jq || !fgeoq)
    return BBW_ERR_ARG;
  const int Np = np_of(N);
  Vec r, s, t;
  nodes3d(N, r, s, t);
  Mat V = vandermonde3d(N, r, s, t);
  Vec rq(cub, cub + Nq), sq(cub + Nq, cub + 2 * Nq), tq(cub + 2 * Nq, cub + 3 * Nq);
  Mat a, b, c;
  gradVandermonde3d(N, rq, sq, tq, a, b, c);
  Mat Vrq = mrdivide(a, V), Vsq = mrdivide(b, V), Vtq = mrdivide(c, V);
  // face cubature on the four faces (cpp/src/StartUp3d.cpp:110-143)
  Vec rf(4 * Nfq), sf(4 * Nfq), tf(4 * Nfq);
  for (int q = 0; q < Nfq; ++q) {
    const double u = tri[q], v = tri[Nfq + q];
    const double pts[4][3] = {{u, v, -1.0}, {u, -1.0, v}, {-(1 + u + v), u, v}, {-1.0, u, v}};
    for (int f = 0; f < 4; ++f)
      rf[f * Nfq + q] = pts[f][0], sf[f * Nfq + q] = pts[f][1], tf[f * Nfq + q] = pts[f][2];
  }
  gradVandermonde3d(N, rf, sf, tf, a, b, c);
  Mat Vrf = mrdivide(a, V), Vsf = mrdivide(b, V), Vtf = mrdivide(c, V);
  std::vector<Vec> g;
  for (int k = 0; k < K; ++k) {
    const size_t o = (size_t)k * Np;
    geofacs(Vrq, Vsq, Vtq, x + o, y + o, z + o, g);
    for (int cc = 0; cc < 9; ++cc)
      for (int q = 0; q < Nq; ++q) vgeoq[((size_t)k * 9 + cc) * Nq + q] = g[cc][q];
    for (int q = 0; q < Nq; ++q) Jq[(size_t)k * Nq + q] = g[9][q];
    // outward normals and surface Jacobians (cpp/src/Basis.cpp:664-723)
    geofacs(Vrf, Vsf, Vtf, x + o, y + o, z + o, g);
    for (int f = 0; f < 4; ++f)
      for (int q = 0; q < Nfq; ++q) {
        const int p = f * Nfq + q;
        double n[3];
        for (int d = 0; d < 3; ++d) {
          const double rd = g[3 * d][p], sd = g[3 * d + 1][p], td = g[3 * d + 2][p];
          n[d] = f == 0 ? -td : f == 1 ? -sd : f == 2 ? rd + sd + td : -rd;
        }
        const double sJ = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        double *dst = fgeoq + ((size_t)k * 4 + f) * 4 * Nfq;
        dst[q] = n[0] / sJ, dst[Nfq + q] = n[1] / sJ, dst[2 * Nfq + q] = n[2] / sJ;
        dst[3 * Nfq + q] = sJ * g[9][p];
      }
  }
  return BBW_OK;
}
