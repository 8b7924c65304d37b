// Host-side mesh setup: connectivity, affine geometric factors and the
// packed arrays the time-step kernels consume.
//
// Restates, for affine tetrahedra:
//   FacePair3d          cpp/src/Mesh3d.cpp:335-410
//   GeometricFactors3d  cpp/src/Mesh3d.cpp:218-258
//   Normals3d           cpp/src/Mesh3d.cpp:260-287
//   node coordinates    cpp/src/StartUp3d.cpp:543-574
//   BuildMaps3d         cpp/src/StartUp3d.cpp:643-741
//   vgeo/fgeo/vmapP     cpp/src/WaveOKL3d.cpp:1530-1603, dt at :1677
//
// Face pairing sorts the full vertex triple (the reference compares only two
// of the three sorted vertices and skips the last sorted face); on meshes
// where the reference's pairing is correct both give identical EToE/EToF.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "bbwadg.h"
#include "internal.h"

namespace bbw {

// vertex triples of the four faces (cpp/src/Mesh3d.cpp:343)
static const int kFaceVerts[4][3] = {{0, 1, 2}, {0, 1, 3}, {1, 2, 3}, {0, 2, 3}};

struct Geo {
  double rx, ry, rz, sx, sy, sz, tx, ty, tz, J;
};

static Geo affine_geo(const double *X, const double *Y, const double *Z) {
  const double dxdr = (X[1] - X[0]) / 2, dxds = (X[2] - X[0]) / 2, dxdt = (X[3] - X[0]) / 2;
  const double dydr = (Y[1] - Y[0]) / 2, dyds = (Y[2] - Y[0]) / 2, dydt = (Y[3] - Y[0]) / 2;
  const double dzdr = (Z[1] - Z[0]) / 2, dzds = (Z[2] - Z[0]) / 2, dzdt = (Z[3] - Z[0]) / 2;
  Geo g;
  g.J = dxdr * (dyds * dzdt - dzds * dydt) - dydr * (dxds * dzdt - dzds * dxdt) +
        dzdr * (dxds * dydt - dyds * dxdt);
  g.rx = (dyds * dzdt - dzds * dydt) / g.J;
  g.ry = -(dxds * dzdt - dzds * dxdt) / g.J;
  g.rz = (dxds * dydt - dyds * dxdt) / g.J;
  g.sx = -(dydr * dzdt - dzdr * dydt) / g.J;
  g.sy = (dxdr * dzdt - dzdr * dxdt) / g.J;
  g.sz = -(dxdr * dydt - dydr * dxdt) / g.J;
  g.tx = (dydr * dzds - dzdr * dyds) / g.J;
  g.ty = -(dxdr * dzds - dzdr * dxds) / g.J;
  g.tz = (dxdr * dyds - dydr * dxds) / g.J;
  return g;
}

static void normals(const Geo &g, double nx[4], double ny[4], double nz[4], double sJ[4]) {
  nx[0] = -g.tx, nx[1] = -g.sx, nx[2] = g.rx + g.sx + g.tx, nx[3] = -g.rx;
  ny[0] = -g.ty, ny[1] = -g.sy, ny[2] = g.ry + g.sy + g.ty, ny[3] = -g.ry;
  nz[0] = -g.tz, nz[1] = -g.sz, nz[2] = g.rz + g.sz + g.tz, nz[3] = -g.rz;
  for (int f = 0; f < 4; ++f) {
    sJ[f] = std::sqrt(nx[f] * nx[f] + ny[f] * ny[f] + nz[f] * nz[f]);
    nx[f] /= sJ[f];
    ny[f] /= sJ[f];
    nz[f] /= sJ[f];
    sJ[f] *= g.J;
  }
}

}  // namespace bbw

using namespace bbw;

extern "C" bbw_status bbw_mesh_connect(int Nv, int K, const int *EToV, int *EToE, int *EToF) {
  if (Nv <= 0 || K <= 0 || !EToV || !EToE || !EToF) return BBW_ERR_ARG;
  if (Nv >= (1 << 21)) return BBW_ERR_UNSUPPORTED;
  struct FaceKey {
    uint64_t key;
    int elem, face;
  };
  std::vector<FaceKey> faces((size_t)K * 4);
  for (int k = 0; k < K; ++k) {
    for (int f = 0; f < 4; ++f) {
      int v[3];
      for (int i = 0; i < 3; ++i) {
        v[i] = EToV[4 * k + kFaceVerts[f][i]];
        if (v[i] < 0 || v[i] >= Nv) return BBW_ERR_MESH;
      }
      std::sort(v, v + 3);
      faces[4 * (size_t)k + f] = {((uint64_t)v[2] << 42) | ((uint64_t)v[1] << 21) | (uint64_t)v[0], k,
                                  f};
    }
  }
  std::sort(faces.begin(), faces.end(), [](const FaceKey &a, const FaceKey &b) {
    return a.key != b.key ? a.key < b.key : (a.elem != b.elem ? a.elem < b.elem : a.face < b.face);
  });
  size_t n = faces.size();
  for (size_t i = 0; i < n;) {
    if (i + 1 < n && faces[i].key == faces[i + 1].key) {
      if (i + 2 < n && faces[i + 2].key == faces[i].key) return BBW_ERR_MESH;  // non-manifold
      const FaceKey &a = faces[i], &b = faces[i + 1];
      EToE[4 * a.elem + a.face] = b.elem;
      EToF[4 * a.elem + a.face] = b.face;
      EToE[4 * b.elem + b.face] = a.elem;
      EToF[4 * b.elem + b.face] = a.face;
      i += 2;
    } else {
      EToE[4 * faces[i].elem + faces[i].face] = faces[i].elem;
      EToF[4 * faces[i].elem + faces[i].face] = faces[i].face;
      i += 1;
    }
  }
  return BBW_OK;
}

extern "C" bbw_status bbw_mesh_geometry(int N, int K, const double *VX, const double *VY,
                                        const double *VZ, const int *EToV, const double *r,
                                        const double *s, const double *t, float *vgeo,
                                        float *fgeo, double *x, double *y, double *z,
                                        float *dt_out) {
  if (N < 1 || N > BBW_MAX_N || K <= 0 || !VX || !VY || !VZ || !EToV) return BBW_ERR_ARG;
  const int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  float FscaleMax = 0.f;
  int bad = 0;
#pragma omp parallel for reduction(max : FscaleMax) reduction(+ : bad)
  for (int k = 0; k < K; ++k) {
    double X[4], Y[4], Z[4];
    for (int v = 0; v < 4; ++v) {
      X[v] = VX[EToV[4 * k + v]];
      Y[v] = VY[EToV[4 * k + v]];
      Z[v] = VZ[EToV[4 * k + v]];
    }
    Geo g = affine_geo(X, Y, Z);
    if (!(g.J > 0)) {
      bad += 1;
      continue;
    }
    if (vgeo) {
      float *G = vgeo + 9 * (size_t)k;
      G[0] = (float)g.rx, G[1] = (float)g.ry, G[2] = (float)g.rz;
      G[3] = (float)g.sx, G[4] = (float)g.sy, G[5] = (float)g.sz;
      G[6] = (float)g.tx, G[7] = (float)g.ty, G[8] = (float)g.tz;
    }
    double nx[4], ny[4], nz[4], sJ[4];
    normals(g, nx, ny, nz, sJ);
    for (int f = 0; f < 4; ++f) {
      const float Fscale = (float)(sJ[f] / g.J);
      FscaleMax = std::max(FscaleMax, Fscale);
      if (fgeo) {
        float *F = fgeo + 16 * (size_t)k + 4 * f;
        F[0] = Fscale, F[1] = (float)nx[f], F[2] = (float)ny[f], F[3] = (float)nz[f];
      }
    }
    if (x && y && z && r && s && t) {
      for (int i = 0; i < Np; ++i) {
        const double a = r[i] + s[i] + t[i] + 1, b = 1. + r[i], c = 1. + s[i], d = 1. + t[i];
        x[(size_t)k * Np + i] = 0.5 * (-X[0] * a + X[1] * b + X[2] * c + X[3] * d);
        y[(size_t)k * Np + i] = 0.5 * (-Y[0] * a + Y[1] * b + Y[2] * c + Y[3] * d);
        z[(size_t)k * Np + i] = 0.5 * (-Z[0] * a + Z[1] * b + Z[2] * c + Z[3] * d);
      }
    }
  }
  if (bad) return BBW_ERR_MESH;  // degenerate or negatively oriented element
  if (dt_out) *dt_out = (float)(.25 / ((N + 1) * (N + 1) * FscaleMax));
  return BBW_OK;
}

extern "C" bbw_status bbw_mesh_vmapP(int N, int K, const int *EToE, const int *EToF,
                                     const int *Fmask, const double *x, const double *y,
                                     const double *z, int *vmapP) {
  if (N < 1 || N > BBW_MAX_N || K <= 0 || !EToE || !EToF || !Fmask || !x || !y || !z || !vmapP)
    return BBW_ERR_ARG;
  const int Np = (N + 1) * (N + 2) * (N + 3) / 6, Nfp = (N + 1) * (N + 2) / 2;
  const double NODETOL = 1e-6;  // cpp/include/Mesh.h:13
  int lost = 0;
#pragma omp parallel for reduction(+ : lost)
  for (int k1 = 0; k1 < K; ++k1) {
    for (int f1 = 0; f1 < 4; ++f1) {
      const int k2 = EToE[4 * k1 + f1], f2 = EToF[4 * k1 + f1];
      for (int n1 = 0; n1 < Nfp; ++n1) {
        const int id1 = n1 + f1 * Nfp + k1 * Nfp * 4;
        const int v1 = Fmask[f1 * Nfp + n1];
        if (k1 == k2) {  // boundary face: the trace maps to itself
          vmapP[id1] = k1 * Np * 4 + v1;
          continue;
        }
        const size_t a = (size_t)k1 * Np + v1;
        int found = -1;
        for (int n2 = 0; n2 < Nfp; ++n2) {
          const size_t b = (size_t)k2 * Np + Fmask[f2 * Nfp + n2];
          const double d = (x[a] - x[b]) * (x[a] - x[b]) + (y[a] - y[b]) * (y[a] - y[b]) +
                           (z[a] - z[b]) * (z[a] - z[b]);
          if (d < NODETOL) {
            found = Fmask[f2 * Nfp + n2];
            break;
          }
        }
        if (found < 0) {
          lost += 1;
          found = v1;
        }
        vmapP[id1] = k2 * Np * 4 + found;  // state index of the + trace, field p
      }
    }
  }
  return lost ? BBW_ERR_MESH : BBW_OK;
}
