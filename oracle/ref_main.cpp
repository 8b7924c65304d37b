// Driver for the reference build (oracle test infrastructure).
//
// Linked against the reference's own, unmodified host sources
// (cpp/src/{Basis,Mesh3d,StartUp3d,Utils,WaveOKL3d}.cpp) and the OCCA
// stand-in in oracle/shim, so every array below is produced by the
// reference's own setup code and every stage runs the reference's own OKL
// kernels (translated by oracle/okl2c.py, JIT-compiled for the host CPU).
//
// Setup sequence is the one of cpp/main_subelem.cpp:27-58:
//   ReadGmsh3d -> FacePair3d -> StartUp3d -> WaveInitOCCA3d -> InitWADG_subelem
// The time loop is Wave_RK's (cpp/src/WaveOKL3d.cpp:2030-2079) with a fixed
// step count: five RK_step_WADG_subelem calls per step with
// fa=(float)rk4a[s], fb=(float)rk4b[s], fdt=dt.
//
// Usage:
//   ref_driver mesh  MESH OUT.bin                ReadGmsh3d + FacePair3d + StartUp3d
//                                                 outputs (vertices, EToV, EToE,
//                                                 EToF, vmapM/vmapP, nodes)
//   ref_driver dump  MESH OUT.bin [opts]         operators + connectivity
//   ref_driver run   MESH OUT.bin [opts]         IC + stages, final state
//   ref_driver kernel MESH OUT.bin --which NAME  one kernel on given inputs
//   ref_driver bench MESH [opts]                 time steps, print JSON
// opts: --c2 one|sine  --c2q FILE  --q0 FILE  --ic cavity|gauss
//       --stages S  --steps S  --warmup W  --dt DT  --kblk V,S,U
//       --rhs FILE  --res FILE  --fa A --fb B
// standard headers first: the reference's Mesh.h defines min/max macros
#include <omp.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <fstream>
#include <string>

#include "fem.h"

extern occa::memory c_vgeo, c_fgeo, c_vmapP, c_Fmask, c_rhsQ, c_resQ, c_Q;
extern occa::memory c_Dr, c_Ds, c_Dt, c_LIFT, c_Dvals4, c_D_ids1, c_D_ids2, c_D_ids3,
    c_D_ids4, c_EEL_vals, c_EEL_ids, c_L0_vals, c_L0_ids, c_cEL, c_slice_ids;
extern occa::memory c_Vq_reduced, c_Pq_reduced, c_c2q, c_Jq_reduced;
extern occa::kernel rk_volume, rk_surface, rk_volume_bern, rk_surface_bern, rk_update,
    rk_update_WADG;
extern occa::device device;
extern double *VX, *VY, *VZ;  // cpp/src/Mesh3d.cpp:6
extern occa::kernelInfo dgInfo;
dfloat WaveInitOCCA3d(Mesh *mesh, int KblkV, int KblkS, int KblkU, int KblkQ, int KblkQf);

#include "ref_io.h"
using namespace refio;

namespace {

double c2_one(double, double, double) { return 1.0; }
double c2_sine(double x, double y, double z) {
  return 1.0 + 0.5 * sin(M_PI * x) * sin(M_PI * y) * sin(M_PI * z);
}
double ic_cavity(double x, double y, double z, double t) {
  return cos(M_PI * x) * cos(M_PI * y) * cos(M_PI * z) * cos(sqrt(3.0) * M_PI * t);
}
double ic_gauss(double x, double y, double z, double) {
  return exp(-50.0 * (x * x + y * y + z * z));
}

void stage_loop(Mesh *mesh, int nstages, float dt) {
  for (int s = 0; s < nstages; ++s) {
    int INTRK = s % 5 + 1;
    const dfloat fdt = dt;
    const dfloat fa = (float)mesh->rk4a[INTRK - 1];
    const dfloat fb = (float)mesh->rk4b[INTRK - 1];
    RK_step_WADG_subelem(mesh, fa, fb, fdt);
  }
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s dump|run|kernel|bench MESH [OUT] [opts]\n", argv[0]);
    return 1;
  }
  std::string mode = argv[1];
  // the reference prints progress with printf; keep stdout for our JSON
  FILE *log = fopen("/dev/null", "w");
  int saved_stdout = dup(1);
  dup2(fileno(log), 1);

  Mesh *mesh = ReadGmsh3d(argv[2]);
  int KblkV = 1, KblkS = 1, KblkU = 1;
  std::string kb = opt(argc, argv, "--kblk", "");
  if (!kb.empty()) sscanf(kb.c_str(), "%d,%d,%d", &KblkV, &KblkS, &KblkU);
  FacePair3d(mesh);
  StartUp3d(mesh);
  if (mode == "mesh") {  // the mesh reader's and connectivity's own outputs
    fflush(stdout);
    dup2(saved_stdout, 1);
    const int K = mesh->K;
    Writer w(argv[3]);
    w.scal("N", p_N);
    w.scal("K", K);
    w.scal("Nv", mesh->Nv);
    w.rec("VX", 1, VX, (uint64_t)mesh->Nv);
    w.rec("VY", 1, VY, (uint64_t)mesh->Nv);
    w.rec("VZ", 1, VZ, (uint64_t)mesh->Nv);
    std::vector<int> e2v((size_t)K * 4), e2e((size_t)K * 4), e2f((size_t)K * 4);
    std::vector<double> gx((size_t)K * 4), gy((size_t)K * 4), gz((size_t)K * 4);
    for (int k = 0; k < K; ++k)
      for (int f = 0; f < 4; ++f) {
        e2v[4 * k + f] = mesh->EToV[k][f];
        e2e[4 * k + f] = mesh->EToE[k][f];
        e2f[4 * k + f] = mesh->EToF[k][f];
        gx[4 * k + f] = mesh->GX(k, f);
        gy[4 * k + f] = mesh->GY(k, f);
        gz[4 * k + f] = mesh->GZ(k, f);
      }
    w.rec("EToV", 2, e2v.data(), e2v.size());
    w.rec("EToE", 2, e2e.data(), e2e.size());
    w.rec("EToF", 2, e2f.data(), e2f.size());
    w.rec("GX", 1, gx.data(), gx.size());
    w.rec("GY", 1, gy.data(), gy.size());
    w.rec("GZ", 1, gz.data(), gz.size());
    w.rec("vmapM_raw", 2, mesh->vmapM, (uint64_t)K * p_Nfp * p_Nfaces);
    w.rec("vmapP_raw", 2, mesh->vmapP, (uint64_t)K * p_Nfp * p_Nfaces);
    w.f64("x", mesh->x);
    w.f64("y", mesh->y);
    w.f64("z", mesh->z);
    return 0;
  }
  dfloat dt = WaveInitOCCA3d(mesh, KblkV, KblkS, KblkU, 1, 1);
  InitQuadratureArrays(mesh);
  std::string c2 = opt(argc, argv, "--c2", "one");
  InitWADG_subelem(mesh, c2 == "sine" ? &c2_sine : &c2_one);
  std::string c2q = opt(argc, argv, "--c2q", "");
  if (!c2q.empty()) load_into(c_c2q, c2q);
  std::string dts = opt(argc, argv, "--dt", "");
  if (!dts.empty()) dt = (dfloat)atof(dts.c_str());

  const int K = mesh->K;
  std::vector<float> Q((size_t)K * p_Np * p_Nfields, 0.f);
  std::string q0 = opt(argc, argv, "--q0", "");
  if (!q0.empty()) {
    std::vector<char> b = slurp(q0);
    if (b.size() != Q.size() * 4) {
      fprintf(stderr, "--q0 size mismatch\n");
      return 1;
    }
    memcpy(Q.data(), b.data(), b.size());
  } else {
    std::string ic = opt(argc, argv, "--ic", "cavity");
    WaveSetU0(mesh, Q.data(), 0.0, ic == "gauss" ? &ic_gauss : &ic_cavity);
  }
  WaveSetData3d(Q.data());

  fflush(stdout);
  dup2(saved_stdout, 1);

  if (mode == "dump") {
    Writer w(argv[3]);
    w.scal("N", p_N);
    w.scal("USE_BERN", USE_BERN);
    w.scal("K", K);
    w.scal("Nq", mesh->Nq);
    w.scal("Nfq", mesh->Nfq);
    w.scal("EEL_nnz", mesh->EEL_nnz);
    w.scal("L0_nnz", mesh->L0_nnz);
    w.scal("dt", dt);
    w.f32("vgeo", c_vgeo);
    w.f32("fgeo", c_fgeo);
    w.i32("Fmask", c_Fmask);
    w.i32("vmapP", c_vmapP);
    w.f32("Dr", c_Dr);
    w.f32("Ds", c_Ds);
    w.f32("Dt", c_Dt);
    w.f32("LIFT", c_LIFT);
    w.i32("D_ids1", c_D_ids1);
    w.i32("D_ids2", c_D_ids2);
    w.i32("D_ids3", c_D_ids3);
    w.i32("D_ids4", c_D_ids4);
    w.f32("Dvals4", c_Dvals4);
    w.i32("EEL_ids", c_EEL_ids);
    w.f32("EEL_vals", c_EEL_vals);
    w.i32("L0_ids", c_L0_ids);
    w.f32("L0_vals", c_L0_vals);
    w.f32("cEL", c_cEL);
    w.i32("slice_ids", c_slice_ids);
    w.f32("Vq", c_Vq_reduced);
    w.f32("Pq", c_Pq_reduced);
    w.f32("Jq", c_Jq_reduced);
    w.f32("c2q", c_c2q);
    w.f32("Q0", c_Q);
    w.f64v("r", mesh->r);
    w.f64v("s", mesh->s);
    w.f64v("t", mesh->t);
    w.f64v("rq", mesh->rq);
    w.f64v("sq", mesh->sq);
    w.f64v("tq", mesh->tq);
    w.f64v("wq", mesh->wq);
    w.f64v("wfqFace", mesh->wfqFace);
    w.f64v("rfq", mesh->rfq);
    w.f64v("sfq", mesh->sfq);
    w.f64("V64", mesh->V);
    w.f64("Dr64", mesh->Dr);
    w.f64("Ds64", mesh->Ds);
    w.f64("Dt64", mesh->Dt);
    w.f64("LIFT64", mesh->LIFT);
    w.f64("Vq64", mesh->Vq);
    w.f64("VB64", mesh->VB);
    w.f64("invVB64", mesh->invVB);
    w.f64("x", mesh->x);
    w.f64("y", mesh->y);
    w.f64("z", mesh->z);
    w.i32m("faceVolPerm", mesh->faceVolPerm);
    w.f64v("EEL_val_vec", mesh->EEL_val_vec);
    w.rec("EEL_id_vec", 2, mesh->EEL_id_vec.data(), (uint64_t)mesh->EEL_id_vec.size());
    std::vector<int> e2e((size_t)K * 4), e2f((size_t)K * 4);
    for (int k = 0; k < K; ++k)
      for (int f = 0; f < 4; ++f) {
        e2e[4 * k + f] = mesh->EToE[k][f];
        e2f[4 * k + f] = mesh->EToF[k][f];
      }
    w.rec("EToE", 2, e2e.data(), e2e.size());
    w.rec("EToF", 2, e2f.data(), e2f.size());
    w.rec("vmapM_raw", 2, mesh->vmapM, (uint64_t)K * p_Nfp * p_Nfaces);
    w.rec("vmapP_raw", 2, mesh->vmapP, (uint64_t)K * p_Nfp * p_Nfaces);
    std::vector<double> rk(16);
    for (int i = 0; i < 5; ++i) rk[i] = mesh->rk4a[i], rk[5 + i] = mesh->rk4b[i];
    for (int i = 0; i < 6; ++i) rk[10 + i] = mesh->rk4c[i];
    w.rec("rk", 1, rk.data(), 16);
    return 0;
  }

  if (mode == "kernel") {
    // one kernel on given Q/rhs/res; dumps rhsQ, resQ, Q afterwards
    std::string which = opt(argc, argv, "--which", "");
    std::string rhs = opt(argc, argv, "--rhs", ""), res = opt(argc, argv, "--res", "");
    if (!rhs.empty()) load_into(c_rhsQ, rhs);
    if (!res.empty()) load_into(c_resQ, res);
    float fa = (float)atof(opt(argc, argv, "--fa", "0").c_str());
    float fb = (float)atof(opt(argc, argv, "--fb", "1").c_str());
    if (which == "rk_volume")
      rk_volume(K, c_vgeo, c_Dr, c_Ds, c_Dt, c_Q, c_rhsQ);
    else if (which == "rk_surface")
      rk_surface(K, c_fgeo, c_Fmask, c_vmapP, c_LIFT, c_Q, c_rhsQ);
    else if (which == "rk_volume_bern")
      rk_volume_bern(K, c_vgeo, c_D_ids1, c_D_ids2, c_D_ids3, c_D_ids4, c_Dvals4, c_Q,
                     c_rhsQ);
    else if (which == "rk_surface_bern")
      rk_surface_bern(K, c_fgeo, c_Fmask, c_vmapP, c_slice_ids, c_EEL_ids, c_EEL_vals,
                      c_L0_ids, c_L0_vals, c_cEL, c_Q, c_rhsQ);
    else if (which == "rk_surface_bern_slice") {
      occa::kernel ks =
          device.buildKernelFromSource("okl/WaveKernels.okl", "rk_surface_bern_slice", dgInfo);
      occa::memory ids, vals;
      {
        MatrixXi idm = mesh->EEL_id_vec;
        ids = device.malloc(idm.size() * sizeof(int), idm.data());
        std::vector<float> v(mesh->EEL_val_vec.size());
        for (size_t i = 0; i < v.size(); ++i) v[i] = (float)mesh->EEL_val_vec(i);
        vals = device.malloc(v.size() * sizeof(float), v.data());
      }
      ks(K, c_fgeo, c_Fmask, c_vmapP, c_slice_ids, ids, vals, c_L0_ids, c_L0_vals, c_cEL, c_Q,
         c_rhsQ);
    } else if (which == "rk_update")
      rk_update(K, fa, fb, dt, c_rhsQ, c_resQ, c_Q);
    else if (which == "rk_update_WADG")
      rk_update_WADG(K, c_Vq_reduced, c_Pq_reduced, c_Jq_reduced, c_c2q, fa, fb, dt, c_rhsQ,
                     c_resQ, c_Q);
    else {
      fprintf(stderr, "unknown kernel %s\n", which.c_str());
      return 1;
    }
    Writer w(argv[3]);
    w.f32("rhsQ", c_rhsQ);
    w.f32("resQ", c_resQ);
    w.f32("Q", c_Q);
    w.scal("dt", dt);
    return 0;
  }

  if (mode == "run") {
    int stages = atoi(opt(argc, argv, "--stages", "5").c_str());
    stage_loop(mesh, stages, dt);
    Writer w(argv[3]);
    w.f32("Q", c_Q);
    w.f32("resQ", c_resQ);
    w.f32("rhsQ", c_rhsQ);
    w.scal("dt", dt);
    return 0;
  }

  if (mode == "bench") {
    int steps = atoi(opt(argc, argv, "--steps", "5").c_str());
    int warm = atoi(opt(argc, argv, "--warmup", "1").c_str());
    stage_loop(mesh, 5 * warm, dt);
    auto t0 = std::chrono::steady_clock::now();
    stage_loop(mesh, 5 * steps, dt);
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("{\"K\": %d, \"N\": %d, \"bern\": %d, \"steps\": %d, \"seconds\": %.6f, "
           "\"threads\": %d, \"dof_stage_per_s\": %.6e}\n",
           K, p_N, USE_BERN, steps, sec, omp_get_max_threads(),
           (double)K * p_Np * p_Nfields * 5.0 * steps / sec);
    return 0;
  }
  fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 1;
}
