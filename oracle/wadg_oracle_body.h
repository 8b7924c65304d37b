/* Body of the CPU restatement of the affine-tet acoustic WADG stage
 * (oracle test infrastructure; included twice by wadg_oracle.c with
 * REAL = float and REAL = double, suffix SFX = _f32 / _f64).
 *
 * Each function restates one reference OKL kernel on whole arrays, with the
 * reference's array layouts and its loop / summation order:
 *   state      Q[k][fld][n]  = Q[n + fld*Np + k*Np*4], fld in {p,u,v,w}
 *   vgeo       [k][9]  {rx,ry,rz,sx,sy,sz,tx,ty,tz}
 *   fgeo       [k][f][4] {Fscale, nx, ny, nz}
 *   operators  column-major (Dr[n + m*Np], LIFT[n + m*Np], Vq[q + j*Nq],
 *              Pq[n + j*Np]), sparse BB ids/vals column-major by nonzero.
 */
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

/* cpp/okl/WaveKernels.okl:44-153 (rk_volume) */
void FN(ora_rk_volume)(int K, int Np, const REAL *vgeo, const REAL *Dr, const REAL *Ds,
                       const REAL *Dt, const REAL *Q, REAL *rhsQ) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k) {
    REAL sp[MAXNP], sUr[MAXNP], sUs[MAXNP], sUt[MAXNP];
    const REAL *G = vgeo + 9 * k;
    for (int n = 0; n < Np; ++n) {
      const int id = n + k * Np * 4;
      const REAL un = Q[id + Np], vn = Q[id + 2 * Np], wn = Q[id + 3 * Np];
      sp[n] = Q[id];
      sUr[n] = un * G[0] + vn * G[1] + wn * G[2];
      sUs[n] = un * G[3] + vn * G[4] + wn * G[5];
      sUt[n] = un * G[6] + vn * G[7] + wn * G[8];
    }
    for (int n = 0; n < Np; ++n) {
      REAL dpdr = 0, dpds = 0, dpdt = 0, divU = 0;
      for (int m = 0; m < Np; ++m) {
        const REAL Dr_m = Dr[n + m * Np], Ds_m = Ds[n + m * Np], Dt_m = Dt[n + m * Np];
        const REAL pm = sp[m];
        dpdr += Dr_m * pm;
        dpds += Ds_m * pm;
        dpdt += Dt_m * pm;
        divU += Dr_m * sUr[m];
        divU += Ds_m * sUs[m];
        divU += Dt_m * sUt[m];
      }
      const REAL dpdx = G[0] * dpdr + G[3] * dpds + G[6] * dpdt;
      const REAL dpdy = G[1] * dpdr + G[4] * dpds + G[7] * dpdt;
      const REAL dpdz = G[2] * dpdr + G[5] * dpds + G[8] * dpdt;
      const int id = n + k * 4 * Np;
      rhsQ[id] = -divU;
      rhsQ[id + Np] = -dpdx;
      rhsQ[id + 2 * Np] = -dpdy;
      rhsQ[id + 3 * Np] = -dpdz;
    }
  }
}

/* upwind flux of one face node, cpp/okl/WaveKernels.okl:184-216;
 * bc = 0: p = 0 wall (the reference), bc = 1: rigid wall u.n = 0 */
static void FN(ora_flux)(const REAL *Q, int idM, int idP, int Np, const REAL *fg, int bc,
                         REAL *pflux, REAL *Uflux) {
  const REAL Fscale = fg[0], nx = fg[1], ny = fg[2], nz = fg[3];
  const int isBoundary = idM == idP;
  const REAL pM = Q[idM], uM = Q[idM + Np], vM = Q[idM + 2 * Np], wM = Q[idM + 3 * Np];
  const REAL pP = Q[idP], uP = Q[idP + Np], vP = Q[idP + 2 * Np], wP = Q[idP + 3 * Np];
  REAL pjump = pP - pM;
  REAL Unjump = (uP - uM) * nx + (vP - vM) * ny + (wP - wM) * nz;
  if (isBoundary) {
    if (bc == 0) {
      pjump = (REAL)(-2.0) * pM;
      Unjump = 0;
    } else {
      pjump = 0;
      Unjump = (REAL)(-2.0) * (uM * nx + vM * ny + wM * nz);
    }
  }
  *pflux = (REAL)0.5 * (pjump - Unjump) * Fscale;
  *Uflux = (REAL)0.5 * (Unjump - pjump) * Fscale;
}

/* cpp/okl/WaveKernels.okl:156-260 (rk_surface): rhsQ += LIFT * flux */
void FN(ora_rk_surface)(int K, int Np, int Nfp, int bc, const REAL *fgeo, const int *Fmask,
                        const int *vmapP, const REAL *LIFT, const REAL *Q, REAL *rhsQ) {
  const int NfpNf = 4 * Nfp;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k) {
    REAL spf[4 * MAXNFP], suf[4 * MAXNFP], snxyz[12];
    for (int n = 0; n < NfpNf; ++n) {
      const int f = n / Nfp;
      const REAL *fg = fgeo + 16 * k + 4 * f;
      snxyz[3 * f] = fg[1];
      snxyz[3 * f + 1] = fg[2];
      snxyz[3 * f + 2] = fg[3];
      FN(ora_flux)(Q, Fmask[n] + k * Np * 4, vmapP[n + k * NfpNf], Np, fg, bc, &spf[n], &suf[n]);
    }
    for (int n = 0; n < Np; ++n) {
      REAL v1 = 0, v2 = 0, v3 = 0, v4 = 0;
      for (int m = 0; m < NfpNf; ++m) {
        const REAL Lnm = LIFT[n + m * Np];
        const int fm = m / Nfp;
        const REAL dfm = suf[m];
        v1 += Lnm * spf[m];
        v2 += Lnm * dfm * snxyz[3 * fm];
        v3 += Lnm * dfm * snxyz[1 + 3 * fm];
        v4 += Lnm * dfm * snxyz[2 + 3 * fm];
      }
      const int id = n + k * 4 * Np;
      rhsQ[id] += v1;
      rhsQ[id + Np] += v2;
      rhsQ[id + 2 * Np] += v3;
      rhsQ[id + 3 * Np] += v4;
    }
  }
}

/* cpp/okl/WaveKernels.okl:262-313 (rk_update) */
void FN(ora_rk_update)(int K, int Np, REAL fa, REAL fb, REAL fdt, const REAL *rhsQ, REAL *resQ,
                       REAL *Q) {
  const long n = (long)K * 4 * Np;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    REAL res = resQ[i];
    res = fa * res + fdt * rhsQ[i];
    resQ[i] = res;
    Q[i] += fb * res;
  }
}

/* cpp/okl/WaveKernelsWADG.okl:1760-1887 (rk_update_WADG), with the optional
 * source term of
 * acous_elas_cpp/okl/ElasKernelsWADG.okl:400-403: ftime * fsrc[k][n] is added
 * to the projected rhs_p (fsrc NULL: no source). */
void FN(ora_rk_update_wadg_src)(int K, int Np, int Nq, const REAL *Vq, const REAL *Pq,
                                const REAL *Jq, const REAL *c2q, REAL fa, REAL fb, REAL fdt,
                                REAL ftime, const REAL *fsrc, const REAL *rhsQ, REAL *resQ,
                                REAL *Q) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k) {
    REAL s[4][MAXNQ], r[4][MAXNQ];
    const REAL *rhs = rhsQ + (long)k * 4 * Np;
    for (int n = 0; n < Nq; ++n) {
      REAL a0 = 0, a1 = 0, a2 = 0, a3 = 0;
      for (int j = 0; j < Np; ++j) {
        const REAL V = Vq[n + j * Nq];
        a0 += V * rhs[j];
        a1 += V * rhs[j + Np];
        a2 += V * rhs[j + 2 * Np];
        a3 += V * rhs[j + 3 * Np];
      }
      r[0][n] = a0, r[1][n] = a1, r[2][n] = a2, r[3][n] = a3;
    }
    for (int n = 0; n < Nq; ++n) {
      const REAL c2 = c2q[n + k * Nq];
      const REAL invJ = (REAL)1 / Jq[n + k * Nq];
      s[0][n] = r[0][n] * invJ * c2;
      s[1][n] = r[1][n] * invJ;
      s[2][n] = r[2][n] * invJ;
      s[3][n] = r[3][n] * invJ;
    }
    for (int n = 0; n < Np; ++n) {
      REAL rp[4] = {0, 0, 0, 0};
      for (int j = 0; j < Nq; ++j) {
        const REAL P = Pq[n + j * Np];
        rp[0] += P * s[0][j];
        rp[1] += P * s[1][j];
        rp[2] += P * s[2][j];
        rp[3] += P * s[3][j];
      }
      if (fsrc) rp[0] += ftime * fsrc[n + (long)k * Np];
      for (int f = 0; f < 4; ++f) {
        const long id = n + f * Np + (long)k * 4 * Np;
        REAL res = fa * resQ[id] + fdt * rp[f];
        resQ[id] = res;
        Q[id] += fb * res;
      }
    }
  }
}

void FN(ora_rk_update_wadg)(int K, int Np, int Nq, const REAL *Vq, const REAL *Pq,
                            const REAL *Jq, const REAL *c2q, REAL fa, REAL fb, REAL fdt,
                            const REAL *rhsQ, REAL *resQ, REAL *Q) {
  FN(ora_rk_update_wadg_src)(K, Np, Nq, Vq, Pq, Jq, c2q, fa, fb, fdt, 0, 0, rhsQ, resQ, Q);
}

/* cpp/okl/WaveKernels.okl:344-474 (rk_volume_bern).  D_idsj[4*i+m] holds
 * column j of operator D(m+1) for row i; Dvals4[4*i+j] the shared values. */
void FN(ora_rk_volume_bern)(int K, int Np, const REAL *vgeo, const int *D1, const int *D2,
                            const int *D3, const int *D4, const REAL *Dvals4, const REAL *Q,
                            REAL *rhsQ) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k) {
    REAL sp[MAXNP], sUr[MAXNP], sUs[MAXNP], sUt[MAXNP];
    const REAL *G = vgeo + 9 * k;
    for (int n = 0; n < Np; ++n) {
      const int id = n + k * Np * 4;
      const REAL un = Q[id + Np], vn = Q[id + 2 * Np], wn = Q[id + 3 * Np];
      sp[n] = Q[id];
      sUr[n] = un * G[0] + vn * G[1] + wn * G[2];
      sUs[n] = un * G[3] + vn * G[4] + wn * G[5];
      sUt[n] = un * G[6] + vn * G[7] + wn * G[8];
    }
    for (int n = 0; n < Np; ++n) {
      const REAL d1 = Dvals4[4 * n], d2 = Dvals4[4 * n + 1], d3 = Dvals4[4 * n + 2],
                 d4 = Dvals4[4 * n + 3];
      const int *a = D1 + 4 * n, *b = D2 + 4 * n, *c = D3 + 4 * n, *e = D4 + 4 * n;
      const REAL p1 = d1 * sp[a[0]] + d2 * sp[b[0]] + d3 * sp[c[0]] + d4 * sp[e[0]];
      const REAL p2 = d1 * sp[a[1]] + d2 * sp[b[1]] + d3 * sp[c[1]] + d4 * sp[e[1]];
      const REAL p3 = d1 * sp[a[2]] + d2 * sp[b[2]] + d3 * sp[c[2]] + d4 * sp[e[2]];
      const REAL p4 = d1 * sp[a[3]] + d2 * sp[b[3]] + d3 * sp[c[3]] + d4 * sp[e[3]];
      REAL dU1 = d1 * (sUr[a[1]] + sUs[a[2]] + sUt[a[3]]);
      dU1 += d2 * (sUr[b[1]] + sUs[b[2]] + sUt[b[3]]);
      dU1 += d3 * (sUr[c[1]] + sUs[c[2]] + sUt[c[3]]);
      dU1 += d4 * (sUr[e[1]] + sUs[e[2]] + sUt[e[3]]);
      REAL dU2 = d1 * (sUr[a[0]] + sUs[a[0]] + sUt[a[0]]);
      dU2 += d2 * (sUr[b[0]] + sUs[b[0]] + sUt[b[0]]);
      dU2 += d3 * (sUr[c[0]] + sUs[c[0]] + sUt[c[0]]);
      dU2 += d4 * (sUr[e[0]] + sUs[e[0]] + sUt[e[0]]);
      const REAL dpdr = (REAL)0.5 * (p2 - p1), dpds = (REAL)0.5 * (p3 - p1),
                 dpdt = (REAL)0.5 * (p4 - p1), divU = (REAL)0.5 * (dU1 - dU2);
      const REAL dpdx = G[0] * dpdr + G[3] * dpds + G[6] * dpdt;
      const REAL dpdy = G[1] * dpdr + G[4] * dpds + G[7] * dpdt;
      const REAL dpdz = G[2] * dpdr + G[5] * dpds + G[8] * dpdt;
      const int id = n + k * 4 * Np;
      rhsQ[id] = -divU;
      rhsQ[id + Np] = -dpdx;
      rhsQ[id + 2 * Np] = -dpdy;
      rhsQ[id + 3 * Np] = -dpdz;
    }
  }
}

/* cpp/okl/WaveKernels.okl:479-647 (rk_surface_bern): flux, per-face L0
 * (Nfp x Nfp, L0_nnz per row), then sparse EEL (Np x 4Nfp, EEL_nnz per
 * row) added to the volume rhs. */
void FN(ora_rk_surface_bern)(int K, int Np, int Nfp, int bc, const REAL *fgeo, const int *Fmask,
                             const int *vmapP, int EEL_nnz, const int *EEL_ids,
                             const REAL *EEL_vals, int L0_nnz, const int *L0_ids,
                             const REAL *L0_vals, const REAL *Q, REAL *rhsQ) {
  const int NfpNf = 4 * Nfp;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < K; ++k) {
    REAL spf[4 * MAXNFP], suf[4 * MAXNFP], spt[4 * MAXNFP], sut[4 * MAXNFP], snxyz[16];
    for (int f = 0; f < 4; ++f) {
      const REAL *fg = fgeo + 16 * k + 4 * f;
      snxyz[4 * f] = fg[1], snxyz[4 * f + 1] = fg[2], snxyz[4 * f + 2] = fg[3];
      snxyz[4 * f + 3] = fg[0];
    }
    for (int n = 0; n < NfpNf; ++n) {
      const int f = n / Nfp;
      FN(ora_flux)(Q, Fmask[n] + k * Np * 4, vmapP[n + k * NfpNf], Np, fgeo + 16 * k + 4 * f, bc,
                   &spf[n], &suf[n]);
    }
    for (int n = 0; n < NfpNf; ++n) {
      const int f = n / Nfp, nt = n % Nfp;
      REAL v1 = 0, v2 = 0;
      for (int j = 0; j < L0_nnz; ++j) {
        const REAL L = L0_vals[nt + j * Nfp];
        const int id = L0_ids[nt + j * Nfp] + f * Nfp;
        v1 += L * spf[id];
        v2 += L * suf[id];
      }
      spt[n] = v1;
      sut[n] = v2;
    }
    for (int n = 0; n < Np; ++n) {
      const int id = n + k * 4 * Np;
      REAL v1 = rhsQ[id], v2 = rhsQ[id + Np], v3 = rhsQ[id + 2 * Np], v4 = rhsQ[id + 3 * Np];
      for (int j = 0; j < EEL_nnz; ++j) {
        const int col = EEL_ids[n + j * Np];
        const REAL E = EEL_vals[n + j * Np];
        const int fcol = col / Nfp;
        const REAL Uf = sut[col];
        v1 += E * spt[col];
        v2 += E * Uf * snxyz[4 * fcol];
        v3 += E * Uf * snxyz[4 * fcol + 1];
        v4 += E * Uf * snxyz[4 * fcol + 2];
      }
      rhsQ[id] = v1;
      rhsQ[id + Np] = v2;
      rhsQ[id + 2 * Np] = v3;
      rhsQ[id + 3 * Np] = v4;
    }
  }
}

#undef FN
#undef CAT
#undef CAT2
