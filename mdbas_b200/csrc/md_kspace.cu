// md_kspace.cu -- reciprocal space inside the engine's dynamics: MDBas's
// energy() with keyEwald 1 (ewald_rec, src/ewald.c:131-354) or 2
// (spme_energy, src/spme.c:357-700) adds the reciprocal forces before the
// real-space ones (src/energy.c:469-472); the engine adds them to the
// nonbonded forces of every step, on the device, so the step stays one CUDA
// graph.  Each engine owns its k-space buffers (a graph holds their
// addresses).
#include <math.h>

#include <vector>

#include "engine.cuh"

using namespace mdbas;

namespace {

constexpr double kPiK = 3.141592653589793;

// MDBas's non-neutral term -pi C (sum q)^2 / (2 alpha^2 V) (src/ewald.c:325).
double kspace_enn(const mdbas_nb_engine *e) {
  const double a = e->cfg.alpha;
  return -(0.5 * kPiK * e->cfg.chargeConst) *
         ((e->kspaceSystq / a) * (e->kspaceSystq / a) / e->hostBox.vol);
}

int kspace_launch(mdbas_nb_engine *e, double *f, cudaStream_t s) {
  const int n = e->n;
  const double *x = e->x.as<double>(), *y = e->y.as<double>(), *z = e->z.as<double>();
  const double *q = e->q.as<double>();
  double *fy = f + n, *fz = f + 2 * (size_t)n;
  if (e->kspaceKind == 1) {
    MDB_TRY(ewald_launch(*e->kEwald, n, &e->hostBox, e->cfg.alpha, e->cfg.chargeConst,
                         e->kspaceM[0], e->kspaceM[1], e->kspaceM[2], x, y, z, q, f, fy, fz, 0,
                         s));
    return kspace_fix_launch(e->kEwald->sums.as<double>(), e->kEwald->fact1, kspace_enn(e),
                             e->kspaceFix.as<long long>(), s);
  }
  MDB_TRY(spme_launch(*e->kSpme, n, &e->hostBox, e->cfg.alpha, e->cfg.chargeConst,
                      e->kspaceM[0], e->kspaceM[1], e->kspaceM[2], e->kspaceOrder, x, y, z, q, f,
                      fy, fz, s));
  return kspace_fix_launch(e->kSpme->sums.as<double>() + 9, e->kSpme->f1, kspace_enn(e),
                           e->kspaceFix.as<long long>(), s);
}

}  // namespace

int mdbas::md_kspace(mdbas_nb_engine *e, double *f, cudaStream_t s) {
  if (e->kspaceKind == 0) return MDBAS_NB_OK;
  return kspace_launch(e, f, s);
}

void mdbas::kspace_release(mdbas_nb_engine *e) {
  delete e->kEwald;
  delete e->kSpme;
  e->kEwald = nullptr;
  e->kSpme = nullptr;
}

extern "C" {

int mdbas_nb_engine_set_kspace(mdbas_nb_engine *e, int kind, int m1, int m2, int m3, int nbsp) {
  if (!e || kind < 0 || kind > 2) return MDBAS_NB_ERR_ARG;
  if (kind != 0 && e->nRep > 1) return MDBAS_NB_ERR_UNSUPPORTED;
  if (kind != 0 && !e->topoSet) return MDBAS_NB_ERR_STATE;
  if (kind == 1 && (m1 < 0 || m2 < 0 || m3 < 0)) return MDBAS_NB_ERR_ARG;
  if (kind == 2 && (m1 <= 0 || m2 <= 0 || m3 <= 0 || nbsp < 2 || nbsp > 16 || nbsp > m1 ||
                    nbsp > m2 || nbsp > m3))
    return MDBAS_NB_ERR_ARG;
  MDB_CUDA(cudaSetDevice(e->device));
  e->kspaceKind = kind;
  e->kspaceM[0] = m1;
  e->kspaceM[1] = m2;
  e->kspaceM[2] = m3;
  e->kspaceOrder = nbsp;
  e->mdGraphStale = true;  // the dynamics graph holds the old launches
  if (kind == 0) return MDBAS_NB_OK;
  // charge sums of the self and non-neutral terms (src/ewald.c:166-172)
  std::vector<double> hq(e->n);
  MDB_CUDA(cudaMemcpy(hq.data(), e->q.p, sizeof(double) * e->n, cudaMemcpyDeviceToHost));
  double systq = 0., sumq2 = 0.;
  for (int i = 0; i < e->n; ++i) {
    systq += hq[i];
    sumq2 += hq[i] * hq[i];
  }
  e->kspaceSystq = systq;
  e->kspaceSumq2 = sumq2;
  if (kind == 1 && !e->kEwald) e->kEwald = new EwaldWork();
  if (kind == 2 && !e->kSpme) e->kSpme = new SpmeWork();
  MDB_TRY(e->kspaceFix.ensure(sizeof(long long)));
  MDB_TRY(e->kspaceF.ensure(sizeof(double) * 3 * (size_t)e->n));
  // one evaluation now builds the k list / FFT plan and the buffers, so that
  // later launches (also inside a captured step) allocate nothing
  if (e->posSet) {
    LaunchScope ls(e);
    MDB_CUDA(cudaMemsetAsync(e->kspaceF.p, 0, sizeof(double) * 3 * (size_t)e->n, e->stream));
    MDB_TRY(kspace_launch(e, e->kspaceF.as<double>(), e->stream));
    MDB_CUDA(cudaStreamSynchronize(e->stream));
  }
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_kspace(mdbas_nb_engine *e, double *fx, double *fy, double *fz,
                           double out[2]) {
  if (!e || !out || (fx && (!fy || !fz))) return MDBAS_NB_ERR_ARG;
  if (e->kspaceKind == 0 || !e->posSet) return MDBAS_NB_ERR_STATE;
  MDB_CUDA(cudaSetDevice(e->device));
  LaunchScope ls(e);
  cudaStream_t s = e->stream;
  const int n = e->n;
  const size_t bytes = sizeof(double) * (size_t)n;
  double *f = e->kspaceF.as<double>();
  MDB_CUDA(cudaMemsetAsync(f, 0, 3 * bytes, s));
  MDB_TRY(kspace_launch(e, f, s));
  // energy: the reciprocal and non-neutral terms plus the self term
  double sums[10];
  const double *dsums = e->kspaceKind == 1 ? e->kEwald->sums.as<double>()
                                           : e->kSpme->sums.as<double>();
  MDB_CUDA(cudaMemcpyAsync(sums, dsums, sizeof(double) * (e->kspaceKind == 1 ? 7 : 10),
                           cudaMemcpyDeviceToHost, s));
  std::vector<double> h;
  if (fx) {
    h.resize(3 * (size_t)n);
    MDB_CUDA(cudaMemcpyAsync(h.data(), f, 3 * bytes, cudaMemcpyDeviceToHost, s));
  }
  MDB_CUDA(cudaStreamSynchronize(s));
  const double a = e->cfg.alpha, C = e->cfg.chargeConst;
  const double eself = -C * a * e->kspaceSumq2 / kSqrtPi;
  const double enn = kspace_enn(e);
  double erec, st0, st3, st5, fct;
  if (e->kspaceKind == 1) {
    fct = e->kEwald->fact1;
    erec = sums[0];
    st0 = fct * (sums[1] + erec) + enn;
    st3 = fct * (sums[4] + erec) + enn;
    st5 = fct * (sums[6] + erec) + enn;
  } else {
    fct = e->kSpme->f1;
    erec = sums[9];
    st0 = fct * (sums[0] + erec) + enn;
    st3 = fct * (sums[3] + erec) + enn;
    st5 = fct * (sums[5] + erec) + enn;
  }
  out[0] = fct * erec + eself + enn;
  out[1] = -(st0 + st3 + st5);
  if (fx)
    for (int i = 0; i < n; ++i) {
      fx[i] += h[i];
      fy[i] += h[n + i];
      fz[i] += h[2 * (size_t)n + i];
    }
  return MDBAS_NB_OK;
}

}  // extern "C"
