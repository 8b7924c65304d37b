// Driver for the reference's curvilinear WADG path (oracle test
// infrastructure).
//
// Linked against the reference's own, unmodified host sources and the OCCA
// stand-in in oracle/shim, like ref_main.cpp.  Setup sequence is the one of
// cpp/main.cpp:58-99 with GORDON_HALL=1:
//   ReadGmsh3d -> FacePair3d -> StartUp3d -> WaveInitOCCA3d
//   -> GordonHallSphere -> InitQuadratureArrays -> InitWADG_curved
// and every stage is the reference's RK_step_WADG (cpp/src/WaveOKL3d.cpp:
// 2111-2185): rk_volume_WADG_skew_combine + rk_surface_WADG_skew_combine on
// the curved elements, rk_volume_planar + rk_surface_planar on the planar
// ones, rk_update_WADG on all, with fa=(float)rk4a[s], fb=(float)rk4b[s].
//
// Built with -DNDEBUG: GordonHallSphere's face blend calls barytors
// (cpp/src/Basis.cpp:343-356), which reads element 2 of a 2-vector; with
// Eigen's bounds assertions on, every N >= 3 run aborts there.  For N = 3 the
// value read is unused (the face functions are the bubble times a degree-0
// polynomial), so the N = 3 geometry is well defined; for N >= 4 it is not.
//
// Usage:
//   ref_curved_N<N> dump   MESH OUT.bin [--q0 FILE] [--c2q FILE]
//   ref_curved_N<N> kernel MESH OUT.bin --which NAME --q0 FILE [--rhs FILE]
//   ref_curved_N<N> run    MESH OUT.bin --stages S [--q0 FILE] [--c2q FILE] [--dt DT]
//   ref_curved_N<N> bench  MESH [--steps S --warmup W]
#include <omp.h>
#include <unistd.h>

#include <chrono>
#include <string>

#include "fem.h"
#include "ref_io.h"
using namespace refio;

extern occa::memory c_vgeo, c_fgeo, c_vmapP, c_Fmask, c_rhsQ, c_resQ, c_Q;
extern occa::memory c_Dr, c_Ds, c_Dt, c_LIFT;
extern occa::memory c_Vq_reduced, c_Pq_reduced, c_c2q, c_Jq_reduced;
extern occa::memory c_Pq, c_Prq, c_Psq, c_Ptq, c_Pfq, c_VfqFace, c_Vfq, c_Vq, c_Vrq, c_Vsq,
    c_Vtq, c_vgeoq, c_fgeoq, c_Jq, c_Vskew, c_Pskew, c_Jplanar, c_KlistCurved, c_KlistPlanar;
extern occa::kernel rk_volume_WADG_skew_combine, rk_surface_WADG_skew_combine,
    rk_volume_planar, rk_surface_planar;
extern occa::device device;
dfloat WaveInitOCCA3d(Mesh *mesh, int KblkV, int KblkS, int KblkU, int KblkQ, int KblkQf);

namespace {

// cpp/main.cpp:10-15
double bessel(double x, double y, double z, double time) {
  double rad = sqrt(x * x + y * y + z * z);
  return (rad < 1e-10) ? 1.0 : sin(M_PI * rad) / (M_PI * rad) * cos(M_PI * time);
}

void stage_loop(Mesh *mesh, int nstages, float dt) {
  for (int s = 0; s < nstages; ++s) {
    const int i = s % 5;
    RK_step_WADG(mesh, (float)mesh->rk4a[i], (float)mesh->rk4b[i], dt);
  }
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s dump|kernel|run|bench MESH [OUT] [opts]\n", argv[0]);
    return 1;
  }
  std::string mode = argv[1];
  FILE *log = fopen("/dev/null", "w");
  int saved_stdout = dup(1);
  dup2(fileno(log), 1);

  Mesh *mesh = ReadGmsh3d(argv[2]);
  FacePair3d(mesh);
  StartUp3d(mesh);
  dfloat dt = WaveInitOCCA3d(mesh, 1, 1, 1, 1, 1);
  GordonHallSphere(mesh);
  InitQuadratureArrays(mesh);
  InitWADG_curved(mesh);
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
    WaveSetU0(mesh, Q.data(), 0.0, &bessel);
  }
  WaveSetData3d(Q.data());
  fflush(stdout);
  dup2(saved_stdout, 1);

  if (mode == "dump") {
    Writer w(argv[3]);
    w.scal("N", p_N);
    w.scal("K", K);
    w.scal("Nq", mesh->Nq);
    w.scal("Nfq", mesh->Nfq);
    w.scal("KCurved", mesh->KCurved);
    w.scal("KPlanar", mesh->KPlanar);
    w.scal("dt", dt);
    w.i32m("KlistCurved", mesh->KlistCurved);
    w.i32m("KlistPlanar", mesh->KlistPlanar);
    w.f64v("rq", mesh->rq), w.f64v("sq", mesh->sq), w.f64v("tq", mesh->tq);
    w.f64v("wq", mesh->wq), w.f64v("wfqFace", mesh->wfqFace);
    w.f64v("rfq", mesh->rfq), w.f64v("sfq", mesh->sfq);
    w.f64("x", mesh->x);
    w.f64("y", mesh->y);
    w.f64("z", mesh->z);
    w.f64("rxq", mesh->rxq), w.f64("sxq", mesh->sxq), w.f64("txq", mesh->txq);
    w.f64("ryq", mesh->ryq), w.f64("syq", mesh->syq), w.f64("tyq", mesh->tyq);
    w.f64("rzq", mesh->rzq), w.f64("szq", mesh->szq), w.f64("tzq", mesh->tzq);
    w.f64("Jq64", mesh->Jq);
    w.f64("nxq", mesh->nxq), w.f64("nyq", mesh->nyq), w.f64("nzq", mesh->nzq);
    w.f64("sJq", mesh->sJq);
    w.f64("VfqFace64", mesh->VfqFace);
    w.f64("Vfq64", mesh->Vfq);
    w.f64("Vrq64", mesh->Vrq);
    w.f32("vgeoq", c_vgeoq);
    w.f32("fgeoq", c_fgeoq);
    w.f32("Jq", c_Jq);
    w.f32("Jq_reduced", c_Jq_reduced);
    w.f32("Jplanar", c_Jplanar);
    w.f32("c2q", c_c2q);
    w.f32("vgeo", c_vgeo);
    w.f32("fgeo", c_fgeo);
    w.i32("vmapP", c_vmapP);
    w.i32("Fmask", c_Fmask);
    const char *ops[] = {"Vq", "Vrq", "Vsq", "Vtq", "Pq", "Prq", "Psq", "Ptq", "VfqFace", "Pfq",
                         "Vfq", "Vq_reduced", "Pq_reduced", "Dr", "Ds", "Dt", "LIFT"};
    occa::memory *mem[] = {&c_Vq, &c_Vrq, &c_Vsq, &c_Vtq, &c_Pq, &c_Prq, &c_Psq, &c_Ptq,
                           &c_VfqFace, &c_Pfq, &c_Vfq, &c_Vq_reduced, &c_Pq_reduced,
                           &c_Dr, &c_Ds, &c_Dt, &c_LIFT};
    for (int i = 0; i < 17; ++i) w.f32(ops[i], *mem[i]);
    w.f32("Q0", c_Q);
    std::vector<int> e2e((size_t)K * 4), e2f((size_t)K * 4);
    for (int k = 0; k < K; ++k)
      for (int f = 0; f < 4; ++f) e2e[4 * k + f] = mesh->EToE[k][f], e2f[4 * k + f] = mesh->EToF[k][f];
    w.rec("EToE", 2, e2e.data(), e2e.size());
    w.rec("EToF", 2, e2f.data(), e2f.size());
    return 0;
  }

  if (mode == "kernel") {
    std::string which = opt(argc, argv, "--which", "");
    std::string rhs = opt(argc, argv, "--rhs", "");
    if (!rhs.empty()) load_into(c_rhsQ, rhs);
    const int KC = mesh->KCurved, KP = mesh->KPlanar;
    if (which == "rk_volume_WADG_skew_combine")
      rk_volume_WADG_skew_combine(KC, c_KlistCurved, c_vgeoq, c_Jq, c_Vq, c_Vrq, c_Vsq, c_Vtq,
                                  c_Pq, c_Prq, c_Psq, c_Ptq, c_Vskew, c_Pskew, c_Q, c_rhsQ);
    else if (which == "rk_surface_WADG_skew_combine")
      rk_surface_WADG_skew_combine(KC, c_KlistCurved, c_fgeo, c_fgeoq, c_VfqFace, c_Pfq, c_Fmask,
                                   c_vmapP, c_Q, c_rhsQ);
    else if (which == "rk_volume_planar")
      rk_volume_planar(KP, c_KlistPlanar, c_vgeo, c_Jplanar, c_Dr, c_Ds, c_Dt, c_Q, c_rhsQ);
    else if (which == "rk_surface_planar")
      rk_surface_planar(KP, c_KlistPlanar, c_fgeo, c_Jplanar, c_Fmask, c_vmapP, c_LIFT, c_Q,
                        c_rhsQ);
    else {
      fprintf(stderr, "unknown kernel %s\n", which.c_str());
      return 1;
    }
    Writer w(argv[3]);
    w.f32("rhsQ", c_rhsQ);
    return 0;
  }

  if (mode == "run") {
    int stages = atoi(opt(argc, argv, "--stages", "5").c_str());
    stage_loop(mesh, stages, dt);
    Writer w(argv[3]);
    w.f32("Q", c_Q);
    w.f32("resQ", c_resQ);
    w.scal("dt", dt);
    return 0;
  }

  if (mode == "bench") {
    int steps = atoi(opt(argc, argv, "--steps", "2").c_str());
    int warm = atoi(opt(argc, argv, "--warmup", "1").c_str());
    stage_loop(mesh, 5 * warm, dt);
    auto t0 = std::chrono::steady_clock::now();
    stage_loop(mesh, 5 * steps, dt);
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("{\"K\": %d, \"N\": %d, \"KCurved\": %d, \"steps\": %d, \"seconds\": %.6f, "
           "\"threads\": %d, \"dof_stage_per_s\": %.6e}\n",
           K, p_N, (int)mesh->KCurved, steps, sec, omp_get_max_threads(),
           (double)K * p_Np * p_Nfields * 5.0 * steps / sec);
    return 0;
  }
  fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 1;
}
