/* bbwadg.h - C ABI of the B200 acoustic WADG time step (affine tetrahedra).
 *
 * Drop-in boundary for the reference's time step (jlchan/bbwadg, cpp/):
 *   - kernel-level entry points replace the OKL kernels the reference builds
 *     with device.buildKernelFromSource() and launches positionally
 *     (cpp/src/WaveOKL3d.cpp:1653-1674, 2084-2106); arguments keep the
 *     reference's order, meaning and array layouts, all pointers are device
 *     pointers, the polynomial degree N is a runtime argument instead of the
 *     p_N define;
 *   - the solver context replaces the module-level device buffers and the
 *     host API of cpp/include/fem.h:49-70 (WaveInitOCCA3d, InitWADG_subelem,
 *     WaveSetData3d, RK_step_WADG_subelem, Wave_RK, WaveGetData3d) with a
 *     fused one-kernel-per-stage path;
 *   - setup entry points restate the reference's host setup (mesh
 *     connectivity, geometric factors, operators).
 *
 * Layouts (all as in the reference):
 *   state   Q[k][fld][n] = Q[n + fld*Np + k*Np*4], fld in {p,u,v,w}, FP32
 *   vgeo    [K][9]  {rx,ry,rz,sx,sy,sz,tx,ty,tz}      (WaveOKL3d.cpp:1561)
 *   fgeo    [K][4][4] {Fscale=sJ/J, nx, ny, nz}       (WaveOKL3d.cpp:1584)
 *   Fmask   [4][Nfp] face-major volume node ids       (StartUp3d.cpp:174)
 *   vmapP   [K][4*Nfp] state index of the + trace     (WaveOKL3d.cpp:1590)
 *   Dr,Ds,Dt [Np x Np], LIFT [Np x 4Nfp], Vq [Nq x Np], Pq [Np x Nq],
 *           column-major (Dr[n + m*Np])
 *   c2q, Jq [K][Nq]                                   (WaveOKL3d.cpp:464)
 *   BB:     D_ids1..4 int4[Np], Dvals4 float4[Np], EEL_ids/vals [Np x EEL_nnz],
 *           L0_ids/vals [Nfp x L0_nnz], cEL [N+1], slice_ids int4[Np]
 *
 * Every function returns a status code and never throws.  Kernel-level
 * functions are asynchronous on the given stream (NULL = legacy default
 * stream), like OCCA kernel launches.
 */
#ifndef BBWADG_H
#define BBWADG_H

#ifdef __cplusplus
extern "C" {
#endif

#define BBW_MAX_N 8

typedef enum bbw_status {
  BBW_OK = 0,
  BBW_ERR_ARG = 1,          /* invalid argument or size */
  BBW_ERR_CUDA = 2,         /* CUDA runtime error (see bbw_last_error) */
  BBW_ERR_NOMEM = 3,        /* device or host allocation failed */
  BBW_ERR_STATE = 4,        /* call out of sequence (e.g. no state set) */
  BBW_ERR_MESH = 5,         /* inconsistent mesh (orientation, pairing) */
  BBW_ERR_NUMERIC = 6,      /* operator construction failed */
  BBW_ERR_UNSUPPORTED = 7,  /* size or option outside the supported range */
  BBW_ERR_TIMEOUT = 8       /* a bounded device wait gave up */
} bbw_status;

enum { BBW_NODAL = 0, BBW_BB = 1 };
/* boundary condition on faces whose + trace is the element itself:
 * PRESSURE_RELEASE is the reference's (p = 0, WaveKernels.okl:211-214),
 * RIGID is u.n = 0 */
enum { BBW_BC_PRESSURE_RELEASE = 0, BBW_BC_RIGID = 1 };

const char *bbw_status_string(bbw_status s);
/* message of the last error raised on the calling thread ("" if none) */
const char *bbw_last_error(void);
/* library version string */
const char *bbw_version(void);

/* ---------------------------------------------------------------- setup */

/* Element-to-element / element-to-face connectivity from EToV [K][4]
 * (0-based).  Replaces FacePair3d, cpp/src/Mesh3d.cpp:335-410; boundary
 * faces map to themselves. */
bbw_status bbw_mesh_connect(int Nv, int K, const int *EToV, int *EToE, int *EToF);

/* Affine geometric factors.  Writes vgeo [K][9] and fgeo [K][4][4] as packed
 * in cpp/src/WaveOKL3d.cpp:1530-1589 (FP32), node coordinates x,y,z [K][Np]
 * (FP64, cpp/src/StartUp3d.cpp:543-574; optional, need r,s,t) and
 * dt = 0.25/((N+1)^2 max Fscale) (cpp/src/WaveOKL3d.cpp:1677).  Any output
 * pointer may be NULL.  Returns BBW_ERR_MESH for non-positive Jacobians. */
bbw_status bbw_mesh_geometry(int N, int K, const double *VX, const double *VY,
                             const double *VZ, const int *EToV, const double *r,
                             const double *s, const double *t, float *vgeo, float *fgeo,
                             double *x, double *y, double *z, float *dt_out);

/* Gordon-Hall curving of the elements that touch the unit sphere
 * (GordonHallSphere, cpp/src/WaveOKL3d.cpp:929-1231): nodes of every edge
 * whose end points lie on the sphere, and of every boundary face whose three
 * vertices do, are projected onto it and the displacements blended into the
 * element.  x, y, z [K][Np] FP64 node coordinates (bbw_mesh_geometry),
 * updated in place; EToF from bbw_mesh_connect; curved[k] = 1 for a curved
 * element, else 0.  Matches the reference for N <= 3; for N >= 4 the
 * reference's face blend reads past a 2-vector (cpp/src/Basis.cpp:353-354)
 * and this function uses the face coordinates it evidently intends. */
bbw_status bbw_gordon_hall_sphere(int N, int K, const int *EToF, double *x, double *y, double *z,
                                  int *curved);

/* Geometric factors at the cubature points of curved elements
 * (InitQuadratureArrays + the packing of InitWADG_curved,
 * cpp/src/StartUp3d.cpp:829-909, cpp/src/WaveOKL3d.cpp:211-233).
 * cub = {rq[Nq], sq, tq}, tri = {rfq[Nfq], sfq} (face-1 coordinates).
 * Writes (FP64) vgeoq [K][9][Nq] (rx sx tx ry sy ty rz sz tz), Jq [K][Nq]
 * and fgeoq [K][4 faces][nx ny nz sJ][Nfq] with sJ the surface Jacobian
 * times J. */
bbw_status bbw_curved_geometry(int N, int K, const double *x, const double *y, const double *z,
                               int Nq, const double *cub, int Nfq, const double *tri,
                               double *vgeoq, double *Jq, double *fgeoq);

/* Trace map vmapP [K][4Nfp] in state indexing (cpp/src/StartUp3d.cpp:643-741
 * followed by the remap of cpp/src/WaveOKL3d.cpp:1590-1603). */
bbw_status bbw_mesh_vmapP(int N, int K, const int *EToE, const int *EToF, const int *Fmask,
                          const double *x, const double *y, const double *z, int *vmapP);

/* Reference-element operators for degree N (cpp/src/StartUp3d.cpp:4-510,
 * cpp/src/WaveOKL3d.cpp:459-483, 894-897).  cub = {rq[Nq], sq, tq, wq} and
 * tri = {rfq[Nfq], sfq, wfq} select the volume / face cubature; pass NULL to
 * use a Stroud conical-product rule of degree 2N+1.  Arrays are read back by
 * name with bbw_ops_get (dtype 0 = FP32 kernel layout, 1 = FP64 column-major,
 * 2 = int32).  Names: Dr Ds Dt LIFT Vq_nodal Pq_nodal Vq_bb Pq_bb cEL
 * Dvals4 EEL_vals L0_vals (FP32 and FP64), V VB invVB LIFTB EEL r s t rq sq tq
 * wq rfq sfq wfq EEL_val_vec (FP64), the curvilinear-path operators Vrq Vsq
 * Vtq [Nq x Np], Prq Psq Ptq [Np x Nq], Vfq [4Nfq x Np], Pfq [Np x 4Nfq],
 * VfqFace [Nfq x Nfp] (FP32 and FP64; cpp/src/StartUp3d.cpp:98-156, 848-856,
 * cpp/src/WaveOKL3d.cpp:238-242), Fmask D_ids1..4 EEL_ids L0_ids slice_ids
 * EEL_id_vec faceVolPerm sizes (int32; sizes = {N,Np,Nfp,Nq,Nfq,EEL_nnz,
 * L0_nnz,EEL_width,L0_width}). */
typedef struct bbw_ops bbw_ops;
bbw_status bbw_ops_build(int N, const double *cub, int Nq, const double *tri, int Nfq,
                         bbw_ops **out);
/* Copies array `name` into dst (capacity *count elements) and sets *count to
 * its length; with dst == NULL only the length is returned. */
bbw_status bbw_ops_get(const bbw_ops *ops, const char *name, int dtype, void *dst,
                       long long *count);
void bbw_ops_free(bbw_ops *ops);

/* Basis functions of degree N at reference points (r, s, t):
 * out[i][n] = phi_n(r_i, s_i, t_i), nodal Lagrange basis on the
 * warp-and-blend nodes (Vandermonde3D(r,s,t) / V, cpp/src/Basis.cpp:286) or
 * Bernstein basis (BernTet, cpp/src/Basis.cpp:539).  Used for receiver interpolation. */
bbw_status bbw_basis_eval(int N, int variant, int npts, const double *r, const double *s,
                          const double *t, double *out);

/* ------------------------------------------------ kernel-level entry points
 * One-to-one replacements of the reference's OKL kernels; same argument
 * order and meaning, device pointers, N at run time.  Node indices are
 * int32 as in the reference's vmapP: K * 4 * Np >= 2^31 returns
 * BBW_ERR_UNSUPPORTED. */

/* cpp/okl/WaveKernels.okl:44-153  rk_volume(K, vgeo, Dr, Ds, Dt, Q, rhsQ) */
bbw_status bbw_rk_volume(int N, int K, const float *vgeo, const float *Dr, const float *Ds,
                         const float *Dt, const float *Q, float *rhsQ, void *stream);

/* cpp/okl/WaveKernels.okl:156-260  rk_surface(K, fgeo, Fmask, vmapP, LIFT, Q, rhsQ);
 * rhsQ += LIFT * flux.  bc selects the wall condition (reference: 0). */
bbw_status bbw_rk_surface(int N, int K, int bc, const float *fgeo, const int *Fmask,
                          const int *vmapP, const float *LIFT, const float *Q, float *rhsQ,
                          void *stream);

/* cpp/okl/WaveKernels.okl:262-313  rk_update(K, fa, fb, fdt, rhsQ, resQ, Q) */
bbw_status bbw_rk_update(int N, int K, float fa, float fb, float fdt, const float *rhsQ,
                         float *resQ, float *Q, void *stream);

/* cpp/okl/WaveKernelsWADG.okl:1760-1887
 * rk_update_WADG(K, Vq, Pq, Jq, c2q, fa, fb, fdt, rhsQ, resQ, Q) */
bbw_status bbw_rk_update_wadg(int N, int K, int Nq, const float *Vq, const float *Pq,
                              const float *Jq, const float *c2q, float fa, float fb, float fdt,
                              const float *rhsQ, float *resQ, float *Q, void *stream);

/* cpp/okl/WaveKernels.okl:344-474
 * rk_volume_bern(K, vgeo, D1_ids, D2_ids, D3_ids, D4_ids, Dvals, Q, rhsQ) */
bbw_status bbw_rk_volume_bern(int N, int K, const float *vgeo, const int *D_ids1,
                              const int *D_ids2, const int *D_ids3, const int *D_ids4,
                              const float *Dvals4, const float *Q, float *rhsQ, void *stream);

/* cpp/okl/WaveKernels.okl:479-647  rk_surface_bern(K, fgeo, Fmask, vmapP,
 * slice_ids, EEL_ids, EEL_vals, L0_ids, L0_vals, cEL, Q, rhsQ); overwrites
 * rhsQ with rhsQ + BB lift of the flux.  EEL_nnz / L0_nnz are the p_EEL_nnz
 * / p_L0_nnz defines (cpp/src/WaveOKL3d.cpp:1625-1626). */
bbw_status bbw_rk_surface_bern(int N, int K, int bc, const float *fgeo, const int *Fmask,
                               const int *vmapP, const int *slice_ids, int EEL_nnz,
                               const int *EEL_ids, const float *EEL_vals, int L0_nnz,
                               const int *L0_ids, const float *L0_vals, const float *cEL,
                               const float *Q, float *rhsQ, void *stream);

/* cpp/okl/WaveKernels.okl:652-939  rk_surface_bern_slice(K, fgeo, Fmask,
 * vmapP, slice_ids, EEL_ids, EEL_vals, L0_ids, L0_vals, cEL, Q, rhsQ): the BB
 * lift slice by slice (the reference's choice for N > 6).  slice_ids is int4
 * [Np]; EEL_ids / EEL_vals are the per-slice packed reduction arrays
 * (EEL_id_vec / EEL_val_vec, 3 entries per node of slices 1..N).  rhsQ +=
 * lift; bc as for bbw_rk_surface. */
bbw_status bbw_rk_surface_bern_slice(int N, int K, int bc, const float *fgeo, const int *Fmask,
                                     const int *vmapP, const int *slice_ids, const int *EEL_ids,
                                     const float *EEL_vals, int L0_nnz, const int *L0_ids,
                                     const float *L0_vals, const float *cEL, const float *Q,
                                     float *rhsQ, void *stream);

/* One LSRK stage as the reference's three launches (rk_volume, rk_surface,
 * rk_update_WADG; arguments as above) for callers that cannot allocate
 * device memory: the rhs buffer is a 16 MiB scratch array inside the
 * library (K * 4 * Np <= 4 Mi floats, else BBW_ERR_UNSUPPORTED).  No
 * reference counterpart (the reference allocates rhsQ at setup).  Make the
 * first call on each device outside stream capture (it looks the scratch
 * address up); calls outside a capture look it up again, so after a
 * cudaDeviceReset make one such call first; nothing in the scratch needs to
 * start at zero; calls that overlap on the same device race on the one
 * scratch; it makes no allocation. */
bbw_status bbw_rk_stage_noalloc(int N, int K, int Nq, int bc, const float *vgeo, const float *Dr,
                                const float *Ds, const float *Dt, const float *fgeo,
                                const int *Fmask, const int *vmapP, const float *LIFT,
                                const float *Vq, const float *Pq, const float *Jq,
                                const float *c2q, float fa, float fb, float fdt, float *resQ,
                                float *Q, void *stream);

/* ---------------------------------------------------------- solver context
 * Owns device copies of the mesh arrays and operators, the state Q (double
 * buffered) and the LSRK residual res.  One stream per context; contexts
 * share no state. */
typedef struct bbw_ctx bbw_ctx;

typedef struct bbw_mesh_desc {
  int N, K, Nq;
  const float *vgeo;  /* [K][9]    host */
  const float *fgeo;  /* [K][4][4] host */
  const int *Fmask;   /* [4][Nfp]  host */
  const int *vmapP;   /* [K][4Nfp] host */
  const float *c2q;   /* [K][Nq]   host */
  const float *Jq;    /* [K][Nq]   host, NULL = all ones (affine) */
} bbw_mesh_desc;

typedef struct bbw_ops_desc {
  /* nodal (variant BBW_NODAL) */
  const float *Dr, *Ds, *Dt, *LIFT;
  /* Bernstein-Bezier (variant BBW_BB) */
  const int *D_ids1, *D_ids2, *D_ids3, *D_ids4;
  const float *Dvals4;
  int EEL_nnz, L0_nnz;
  const int *EEL_ids, *L0_ids;
  const float *EEL_vals, *L0_vals;
  /* WADG projection for the chosen basis */
  const float *Vq, *Pq;
} bbw_ops_desc;

/* Arithmetic of the fused stage.  FP32: CUDA-core FP32 throughout.
 * F16X3: the dense contractions (Dr/Ds/Dt, LIFT, Vq, Pq) on the tensor cores
 * as three FP16 products per split pair (A_hi x_hi + A_hi x_lo + A_lo x_hi,
 * per-tile power-of-two scaling, FP32 accumulation); state, fluxes and the
 * update stay FP32.  BF16X3: the same with BF16 pairs (16 significant bits
 * per pair instead of 22; the split-BF16 form of the precision study).  Both
 * run N in [2, 5] (Np <= 64: each operator's rows fit one M = 64 MMA and all
 * operators one SM's shared memory), Nq <= 128, batched shots and sources,
 * nodal or BB (BB: the dense equivalents of the sparse BB derivative and
 * lift applied to BB coefficients), and the adjoint (its forward and
 * recomputation run the same stage). */
enum { BBW_PREC_FP32 = 0, BBW_PREC_F16X3 = 1, BBW_PREC_BF16X3 = 2, BBW_PREC_TF32 = 3 };
/* Precision-study form: F16X3 and BF16X3 at orders the fused tensor-core
 * stage does not take (N >= 6, or Nq > 128), and TF32 at every order, run
 * the same contractions as GEMMs over all elements (cuBLAS; split pairs as
 * three GEMMs with per-element power-of-two scaling, TF32 as one GEMM with
 * TF32 inputs and FP32 accumulation) around this library's flux, split and
 * update kernels: one shot, no sources, no adjoint (BBW_ERR_UNSUPPORTED);
 * its speed is that of separate launches over HBM intermediates. */

/* Uploads mesh and operators (cpp/src/WaveOKL3d.cpp:1400-1615 and
 * :894-909) to the current CUDA device; state and residual start at zero.
 * bbw_create is bbw_create_ex with BBW_PREC_FP32. */
bbw_status bbw_create(const bbw_mesh_desc *mesh, const bbw_ops_desc *ops, int variant, int bc,
                      bbw_ctx **out);
bbw_status bbw_create_ex(const bbw_mesh_desc *mesh, const bbw_ops_desc *ops, int variant, int bc,
                         int precision, bbw_ctx **out);
bbw_status bbw_destroy(bbw_ctx *ctx);

/* WaveSetData3d / WaveGetData3d (cpp/src/WaveOKL3d.cpp:2527-2537): copy the
 * state from / to host memory ([K][4][Np] FP32).  Synchronous. */
bbw_status bbw_set_state(bbw_ctx *ctx, const float *Q_host);
bbw_status bbw_get_state(bbw_ctx *ctx, float *Q_host);
/* Residual res (LSRK45 register) from / to host memory; zero after create. */
bbw_status bbw_set_residual(bbw_ctx *ctx, const float *res_host);
bbw_status bbw_get_residual(bbw_ctx *ctx, float *res_host);

/* RK_step_WADG_subelem (cpp/src/WaveOKL3d.cpp:2084-2109): one LSRK stage
 * res = fa*res + fdt*P(c2 rhs), Q += fb*res, as one fused kernel.
 * Asynchronous on the context's stream.  bbw_stage_ex also takes the stage
 * time offset c (stage time = clock + c*fdt) used by the sources;
 * bbw_stage uses c = 0. */
bbw_status bbw_stage(bbw_ctx *ctx, float fa, float fb, float fdt);
bbw_status bbw_stage_ex(bbw_ctx *ctx, float fa, float fb, float fdt, float c);

/* nsteps full LSRK45 steps of size dt (the time loop of Wave_RK,
 * cpp/src/WaveOKL3d.cpp:2030-2079, with coefficients cast to float as at
 * :2053-2055).  Asynchronous; captured once as a CUDA graph per nsteps. */
bbw_status bbw_steps(bbw_ctx *ctx, float dt, int nsteps);

/* Wave_RK(mesh, FinalTime, dt) semantics: steps of dt until FinalTime with
 * the last step shortened to land on it (cpp/src/WaveOKL3d.cpp:2048). */
bbw_status bbw_run(bbw_ctx *ctx, double final_time, float dt);

/* Times every variant of the FP32 fused stage on this context's mesh, shots
 * and state (8 or 16 warps per CTA; element tiles of 32 or 16 elements, i.e.
 * rows per thread group ceil(Np / (32 W / E)); operators in shared or global
 * memory; single or double-buffered input tiles), `stages` launches each on
 * scratch copies of the state, and keeps the fastest.  *config (may be NULL)
 * = W | ops_in_smem << 8 | pipelined << 9 | (E == 16) << 10.
 * The state is not modified.  No-op for the tensor-core stage.  The
 * reference's counterpart is its hand-swept KblkV/KblkS/KblkU block sizes
 * (cpp/src/WaveOKL3d.cpp:1618-1650, cpp/profileKernels). */
bbw_status bbw_autotune(bbw_ctx *ctx, float dt, int stages, int *config);
/* Applies a configuration code as returned by bbw_autotune (for instance one
 * cached from an earlier run); BBW_ERR_UNSUPPORTED if it does not fit. */
bbw_status bbw_set_config(bbw_ctx *ctx, int config);
/* Caps the persistent stage kernels (FP32 fused and tensor-core forms) at
 * max_ctas CTAs, each then looping over more element tiles; 0 restores one
 * CTA per SM.  For leaving SMs to concurrent work on other streams, and for
 * checking the per-CTA tile loop on small meshes.  A launch-shape control
 * like the reference's KblkV/KblkS/KblkU (cpp/src/WaveOKL3d.cpp:1618-1650);
 * results do not depend on it. */
bbw_status bbw_set_grid_limit(bbw_ctx *ctx, int max_ctas);

/* ---- element (slab) decomposition across devices.  Elements [0, Kc) of
 * the context are advanced by each stage; elements [Kc, K) are halo copies of
 * neighbouring elements owned elsewhere, read only for their face traces
 * (their faces that leave the local mesh are given as boundary faces in
 * vmapP).  Between stages the caller refreshes the halo: bbw_gather_elements
 * packs the current state of listed elements (all shots,
 * [S][n][4][Np], device idx and buf) and bbw_scatter_elements writes a packed
 * buffer back.  No reference counterpart (the reference runs one device,
 * cpp/src/WaveOKL3d.cpp:1415).  FP32 stage only. */
bbw_status bbw_set_compute_range(bbw_ctx *ctx, int Kc);
bbw_status bbw_gather_elements(bbw_ctx *ctx, int n, const int *idx, float *buf);
bbw_status bbw_scatter_elements(bbw_ctx *ctx, int n, const int *idx, const float *buf);

/* Split stage for overlapping the halo exchange with interior work: each
 * bbw_stage_part advances elements [K0, K1) from the current state into the
 * next state (no buffer swap, context stream); bbw_stage_commit makes the
 * next state current once every element of [0, Kc) has been advanced.
 * Between them bbw_move_elements gathers (dir 0) or scatters (dir 1) listed
 * elements of the current (which 0) or next (which 1) state on `stream`
 * (NULL: the context stream): the interface elements can be packed and
 * sent as soon as their part is done while the interior part runs.  FP32
 * stage only; the caller orders the streams (events).  No reference
 * counterpart. */
bbw_status bbw_stage_part(bbw_ctx *ctx, float fa, float fb, float fdt, int K0, int K1);
bbw_status bbw_stage_commit(bbw_ctx *ctx);
bbw_status bbw_move_elements(bbw_ctx *ctx, int which, int dir, int n, const int *idx, float *buf,
                             void *stream);

/* ---- batched shots, sources, receivers (every precision)
 * S independent shots share mesh, medium and operators; the state, residual
 * and traces hold S consecutive blocks and every stage launch advances all
 * of them.  Resizing drops state (zeroed) and the source table. */
bbw_status bbw_set_shots(bbw_ctx *ctx, int S);

/* Source entries (acous_elas_cpp/src/WaveOKL3d.cpp:765-781 and
 * acous_elas_cpp/okl/ElasKernelsWADG.okl:400-403): entry j adds
 * ricker(t) * vec[j][0..Np) to the WADG-projected rhs_p of element elem[j]
 * of shot shot[j], with ricker(t) = amplitude (1 - 2 a^2) exp(-a^2),
 * a = pi f0 (t - t_delay).  vec is the L2 projection (Pq) of the spatial
 * source profile.  stage_times = 0 evaluates ricker at the step's start time
 * in all five stages, as the reference does; nonzero uses the stage times
 * t + rk4c[s] dt.  nent = 0 clears. */
bbw_status bbw_set_sources(bbw_ctx *ctx, int nent, const int *shot, const int *elem,
                           const float *vec, float f0, float t_delay, float amplitude,
                           int stage_times);

/* Receivers: trace[s][r][step] = sum_n w[r][n] p_n of element elem[r] in
 * shot s, recorded after every full step of bbw_steps / bbw_run (up to
 * max_steps).  R = 0 clears. */
bbw_status bbw_set_receivers(bbw_ctx *ctx, int R, const int *elem, const float *w,
                             int max_steps);
/* Copies traces [S][R][max_steps] and the number of recorded steps. */
bbw_status bbw_get_traces(bbw_ctx *ctx, float *out, int *nsteps);

/* Device clock read by the sources: time at the start of the next step;
 * bbw_set_time also resets the recorded step count. */
bbw_status bbw_set_time(bbw_ctx *ctx, double t);
bbw_status bbw_get_time(bbw_ctx *ctx, double *t, int *step);

/* ---- discrete adjoint: gradient of a receiver-trace loss with respect to
 * c^2 at the cubature points.  No reference counterpart: the adjoint
 * reverses the reference's stage (rk_volume + rk_surface + rk_update_WADG,
 * cpp/okl/WaveKernels.okl:44-260, cpp/okl/WaveKernelsWADG.okl:1760-1887)
 * and its LSRK45 loop (cpp/src/WaveOKL3d.cpp:2014-2109).  Either stage form
 * (FP32 or split-precision tensor-core: the forward pass and its
 * recomputation run the context's stage, the reverse stages the FP32
 * transposed operators); both bases; any number of shots. */
/* ------------------------------------------------------------------
 * Curvilinear WADG path (cpp/src/WaveOKL3d.cpp:164-417 InitWADG_curved,
 * :2111-2185 RK_step_WADG).  Kernel-level entry points take device
 * pointers in the reference's layouts; N, Nq and Nfq are the reference's
 * compile-time p_N, p_Nq, p_Nfq.  A stream of NULL is the legacy stream.
 * ------------------------------------------------------------------ */

/* rk_volume_WADG_skew_combine (cpp/okl/WaveKernelsWADG.okl:514-682): for the
 * K elements Klist[0..K): interpolates u,v,w and grad_rst p to the Nq
 * cubature points, forms J grad p and -J (rst-contravariant U), projects
 * with Pq and Prq/Psq/Ptq and writes rhsQ.  vgeoq [K][9][Nq] (rx sx tx ry
 * sy ty rz sz tz), Jq [K][Nq], Vq/Vrq/Vsq/Vtq [Nq x Np] and
 * Pq/Prq/Psq/Ptq [Np x Nq] column-major.  Vskew/Pskew are accepted and not
 * read, as in the reference kernel (may be NULL). */
bbw_status bbw_rk_volume_wadg_skew_combine(int N, int Nq, int K, const int *Klist,
                                           const float *vgeoq, const float *Jq, const float *Vq,
                                           const float *Vrq, const float *Vsq, const float *Vtq,
                                           const float *Pq, const float *Prq, const float *Psq,
                                           const float *Ptq, const float *Vskew,
                                           const float *Pskew, const float *Q, float *rhsQ,
                                           void *stream);

/* rk_surface_WADG_skew_combine (cpp/okl/WaveKernelsWADG.okl:3024-3195):
 * jumps and averages at the face nodes (pressure-release wall), VfqFace
 * [Nfq x Nfp] to the face cubature, upwind fluxes with fgeoq
 * [K][4][nx ny nz sJ][Nfq], lifted with Pfq [Np x 4Nfq] and ADDED to rhsQ.
 * fgeo is accepted and not read, as in the reference kernel. */
bbw_status bbw_rk_surface_wadg_skew_combine(int N, int Nfq, int K, const int *Klist,
                                            const float *fgeo, const float *fgeoq,
                                            const float *VfqFace, const float *Pfq,
                                            const int *Fmask, const int *vmapP, const float *Q,
                                            float *rhsQ, void *stream);

/* rk_volume_planar (cpp/okl/WaveKernelsWADG.okl:2203-2318): rk_volume on the
 * listed affine elements with the output scaled by J[k]. */
bbw_status bbw_rk_volume_planar(int N, int K, const int *Klist, const float *vgeo,
                                const float *J, const float *Dr, const float *Ds,
                                const float *Dt, const float *Q, float *rhsQ, void *stream);

/* rk_surface_planar (cpp/okl/WaveKernelsWADG.okl:2320-2441): rk_surface
 * (pressure-release wall) on the listed affine elements with Fscale scaled
 * by J[k]; adds to rhsQ. */
bbw_status bbw_rk_surface_planar(int N, int K, const int *Klist, const float *fgeo,
                                 const float *J, const int *Fmask, const int *vmapP,
                                 const float *LIFT, const float *Q, float *rhsQ, void *stream);

/* Arrays InitWADG_curved uploads (host, FP32, reference layouts).  The
 * element lists must partition 0..K-1; the curved-element arrays may be
 * NULL when KCurved == 0.  Vq_reduced/Pq_reduced/Jq_reduced/c2q use the
 * update's cubature of Nq_reduced points (the reference uses the same rule
 * as the volume cubature). */
typedef struct bbw_curved_desc {
  int N, K, Nq, Nfq, Nq_reduced;
  int KCurved, KPlanar;
  const int *KlistCurved, *KlistPlanar;
  const float *vgeo, *fgeo;     /* [K][9], [K][4][4] affine factors */
  const float *Jplanar;         /* [K] J of the planar elements */
  const int *Fmask, *vmapP;     /* [4Nfp], [K][4Nfp] */
  const float *vgeoq, *Jq;      /* [K][9][Nq], [K][Nq] */
  const float *fgeoq;           /* [K][4][4][Nfq] */
  const float *Jq_reduced, *c2q;/* [K][Nq_reduced] */
  const float *Dr, *Ds, *Dt, *LIFT;
  const float *Vq, *Vrq, *Vsq, *Vtq, *Pq, *Prq, *Psq, *Ptq, *VfqFace, *Pfq;
  const float *Vq_reduced, *Pq_reduced;
} bbw_curved_desc;

typedef struct bbw_curved bbw_curved;

/* Uploads the arrays to `device`; state and residual start at zero. */
bbw_status bbw_curved_create(const bbw_curved_desc *desc, int device, bbw_curved **out);
bbw_status bbw_curved_destroy(bbw_curved *h);
/* Host copies of the state [K][4][Np]; set_state also zeroes the residual. */
bbw_status bbw_curved_set_state(bbw_curved *h, const float *Q);
bbw_status bbw_curved_get_state(bbw_curved *h, float *Q);
bbw_status bbw_curved_get_residual(bbw_curved *h, float *res);
/* One stage: RK_step_WADG(mesh, fa, fb, fdt). */
bbw_status bbw_curved_stage(bbw_curved *h, float fa, float fb, float fdt);
/* nsteps LSRK45 steps of size dt (five stages with fa = (float)rk4a[s],
 * fb = (float)rk4b[s]), one CUDA graph launch per step; asynchronous. */
bbw_status bbw_curved_steps(bbw_curved *h, float dt, int nsteps);
bbw_status bbw_curved_sync(bbw_curved *h);
/* The handle's CUDA stream (cudaStream_t). */
void *bbw_curved_stream(bbw_curved *h);
/* Times `stages` whole curved stages (fused planar stage beside the curved
 * kernel) for every fused-stage variant that fits and keeps the fastest;
 * the state and residual are restored.  *config (may be NULL) receives the
 * code bbw_set_config takes, 0 when there is no planar element.  Replaces
 * the reference's hand-run element-block timings of the curved kernels
 * (cpp/runCurvedBlkTimings). */
bbw_status bbw_curved_autotune(bbw_curved *h, float dt, int stages, int *config);

typedef struct bbw_tape bbw_tape;

/* Replaces c^2 / J at the cubature points ([K][Nq], host). */
bbw_status bbw_set_c2q(bbw_ctx *ctx, const float *c2q);

/* Advances nsteps steps of dt exactly as bbw_steps does (receivers must be
 * set; traces land at the current step count onwards) and returns a tape
 * for bbw_backward: bbw_forward_ex with BBW_TAPE_CUBATURE (every stage's
 * cubature values when they fit, else the state at every
 * checkpoint_every-th step start).  No counterpart in the reference. */
bbw_status bbw_forward(bbw_ctx *ctx, float dt, int nsteps, int checkpoint_every,
                       bbw_tape **tape);

/* What a tape keeps (bbw_forward_ex).  CHECKPOINTS: the state every
 * checkpoint_every steps; bbw_backward recomputes each segment once.
 * CUBATURE: every stage's pre-c^2 cubature values Vq S(Q)_p ([S][Nq][K]
 * floats per stage, 5 stages per step), which is all the reverse sweep
 * needs, so bbw_backward recomputes nothing; taken only when the device has
 * room for them with 4 GiB to spare, else the tape falls back to
 * checkpoints.  bbw_forward keeps CUBATURE when it fits. */
#define BBW_TAPE_CHECKPOINTS 0
#define BBW_TAPE_CUBATURE 1
bbw_status bbw_forward_ex(bbw_ctx *ctx, float dt, int nsteps, int checkpoint_every, int keep,
                          bbw_tape **tape);
/* 1 if the tape holds every stage's cubature values, 0 if checkpoints. */
int bbw_tape_kind(const bbw_tape *tape);

/* Given dL/dtraces [S][R][nsteps] (host, for the tape's steps), writes
 * dL/d(c2q) [K][Nq] (host, FP64, summed over shots) and, if dL_dQ0 is not
 * NULL, dL/d(state at the tape's first step) [S][K][4][Np].  From a
 * checkpoint tape it recomputes the forward stages of each segment; the
 * context's own state is left as bbw_forward left it. */
bbw_status bbw_backward(bbw_ctx *ctx, bbw_tape *tape, const float *dL_dtraces, double *dL_dc2q,
                        float *dL_dQ0);
bbw_status bbw_tape_free(bbw_tape *tape);

/* Waits for the context's stream. */
bbw_status bbw_sync(bbw_ctx *ctx);

/* Waits for the stream and reports BBW_ERR_TIMEOUT if a bounded device-side
 * wait (tensor-core completion, bulk copies) gave up since creation. */
bbw_status bbw_check(bbw_ctx *ctx);

/* Device pointers of the current state and residual ([K][4][Np]) and the
 * context's cudaStream_t, for zero-copy interop.  Valid until the next
 * stage. */
bbw_status bbw_device_state(bbw_ctx *ctx, float **Q, float **res, void **stream);

#ifdef __cplusplus
}
#endif
#endif /* BBWADG_H */
