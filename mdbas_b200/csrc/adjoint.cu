// adjoint.cu -- parameter gradients and force-loss adjoint of the real-space
// Ewald + switched LJ energy (mdbas_nb_engine_adjoint).
//
// The energy is MDBas's (src/energy.c:480-621): per in-cut-off pair of the
// half list E = C q_i q_j erfc(a r)/r + vdw_switch(eps_i eps_j, sig_i + sig_j)
// (src/ewald.c:356-369, src/vdw.c:144-184), per excluded pair
// -C q_i q_j erf(a r)/r (src/ewald.c:371-384), and the self term
// -C a/sqrt(pi) sum q^2 (src/ewald.c:165-171).  For upstream weights v on the
// forces F_i = -dE/dx_i the kernel also returns the gradients of v.F with
// respect to the positions (a Hessian-vector product, -H v) and to the
// per-atom parameters.  With d = x_j - x_i, r = |d|, a pair contributes
// v.F = E'(r) (v_i - v_j).d / r, whose gradient in d is
//   ((v_i - v_j).d / r) (E'' - E'/r) d / r + (E'/r) (v_i - v_j).
// Pair terms are recomputed from the list, never stored.  FP64 throughout:
// the adjoint is the gradient harness's reference-quality path.
#include "common.cuh"
#include "engine.cuh"

using namespace mdbas;

namespace {

// Per-unit-charge-product Ewald pair function and its first two radial
// derivatives; `corr` selects the exclusion correction -erf(ar)/r.
struct RadialQ {
  double e, d1, d2;
};

__device__ __forceinline__ RadialQ ewald_unit(const PairParams &p, double r, bool corr) {
  const double ar = p.alpha * r;
  const double g = exp(-(ar * ar));
  const double A = p.chargeConst * 2.0 * p.alpha / kSqrtPi;
  RadialQ o;
  o.e = corr ? -p.chargeConst * erf(ar) / r : p.chargeConst * erfc(ar) / r;
  // E' = -(E + A g)/r holds for both forms, hence E'' = -2E'/r + 2 A a^2 g
  o.d1 = -(o.e + A * g) / r;
  o.d2 = -2.0 * o.d1 / r + 2.0 * A * p.alpha * p.alpha * g;
  return o;
}

// Switched LJ per unit eps_i*eps_j: G, G', G'' and the sigma derivatives
// dG/dsig, dG'/dsig (sig = sig_i + sig_j).
struct RadialLJ {
  double g, d1, d2, s, s1;
};

__device__ __forceinline__ RadialLJ lj_unit(const PairParams &p, double r, double r2,
                                            double sig) {
  RadialLJ o{0., 0., 0., 0., 0.};
  if (!p.vdwSwitch || sig == 0.) return o;
  const double t = sig / r;
  const double s6 = (t * t * t) * (t * t * t);
  const double s12 = s6 * s6;
  const double P = 4.0 * (s12 - s6);
  const double P1 = 24.0 / r * (s6 - 2.0 * s12);
  const double P2 = 4.0 / r2 * (156.0 * s12 - 42.0 * s6);
  const double Ps = 4.0 / sig * (12.0 * s12 - 6.0 * s6);
  const double Ps1 = 24.0 / (r * sig) * (6.0 * s6 - 24.0 * s12);
  if (r2 <= p.cutOn2) {
    o.g = P;
    o.d1 = P1;
    o.d2 = P2;
    o.s = Ps;
    o.s1 = Ps1;
    return o;
  }
  const double a = p.cutOff2 - r2, b = p.cutOn2 - r2;
  const double S = a * a * (p.cutOff2 + 2.0 * r2 - 3.0 * p.cutOn2) * p.switch2;
  const double Su = 6.0 * p.switch2 * a * b;                       // dS/d(r^2)
  const double Suu = -6.0 * p.switch2 * (p.cutOff2 + p.cutOn2 - 2.0 * r2);
  const double S1 = 2.0 * r * Su;
  const double S2 = 2.0 * Su + 4.0 * r2 * Suu;
  o.g = P * S;
  o.d1 = P1 * S + P * S1;
  o.d2 = P2 * S + 2.0 * P1 * S1 + P * S2;
  o.s = Ps * S;
  o.s1 = Ps1 * S + Ps * S1;
  return o;
}

struct AdjOut {
  double *gq, *geps, *gsig;   // dE/d(q_i, eps_i, sig_i)
  double *hx, *hy, *hz;       // d(v.F)/dx_i
  double *pq, *peps, *psig;   // d(v.F)/d(q_i, eps_i, sig_i)
};

__device__ __forceinline__ void adj_pair(const PairParams &p, int i, int j, double dx, double dy,
                                         double dz, double r2, bool corr, const double *q,
                                         const double *eps, const double *sig, const double *vx,
                                         const double *vy, const double *vz, const AdjOut &o,
                                         double (&acc)[10]) {
  const double r = sqrt(r2);
  const double qi = q[i], qj = q[j];
  const RadialQ c = ewald_unit(p, r, corr);
  RadialLJ l{0., 0., 0., 0., 0.};
  double ei = 0., ej = 0., veps = 0.;
  if (!corr) {
    ei = eps[i];
    ej = eps[j];
    veps = ei * ej;
    l = lj_unit(p, r, r2, sig[i] + sig[j]);
  }
  // dE/d parameters (acc: 0 gq_i, 1 geps_i, 2 gsig_i)
  acc[0] += qj * c.e;
  atomicAdd(o.gq + j, qi * c.e);
  if (!corr) {
    acc[1] += ej * l.g;
    acc[2] += veps * l.s;
    atomicAdd(o.geps + j, ei * l.g);
    atomicAdd(o.gsig + j, veps * l.s);
  }
  if (!vx) return;
  const double ux = vx[i] - vx[j], uy = vy[i] - vy[j], uz = vz[i] - vz[j];
  const double ud = (ux * dx + uy * dy + uz * dz) / r;  // (v_i - v_j).d / r
  const double qq = qi * qj;
  const double E1 = qq * c.d1 + veps * l.d1;
  const double E2 = qq * c.d2 + veps * l.d2;
  const double a = ud * (E2 - E1 / r) / r, b = E1 / r;
  const double hx = a * dx + b * ux, hy = a * dy + b * uy, hz = a * dz + b * uz;
  acc[3] -= hx;
  acc[4] -= hy;
  acc[5] -= hz;
  atomicAdd(o.hx + j, hx);
  atomicAdd(o.hy + j, hy);
  atomicAdd(o.hz + j, hz);
  // d(v.F)/d parameters (acc: 6 pq_i, 7 peps_i, 8 psig_i)
  acc[6] += qj * c.d1 * ud;
  atomicAdd(o.pq + j, qi * c.d1 * ud);
  if (!corr) {
    acc[7] += ej * l.d1 * ud;
    acc[8] += veps * l.s1 * ud;
    atomicAdd(o.peps + j, ei * l.d1 * ud);
    atomicAdd(o.psig + j, veps * l.s1 * ud);
  }
}

__device__ __forceinline__ void adj_flush(int i, const double (&acc)[10], bool hvp,
                                          const AdjOut &o) {
  atomicAdd(o.gq + i, acc[0]);
  atomicAdd(o.geps + i, acc[1]);
  atomicAdd(o.gsig + i, acc[2]);
  if (!hvp) return;
  atomicAdd(o.hx + i, acc[3]);
  atomicAdd(o.hy + i, acc[4]);
  atomicAdd(o.hz + i, acc[5]);
  atomicAdd(o.pq + i, acc[6]);
  atomicAdd(o.peps + i, acc[7]);
  atomicAdd(o.psig + i, acc[8]);
}

// One thread per atom (neighOrder position) over its half-list entries.
__global__ void __launch_bounds__(128)
k_adjoint_pairs(int n, DevBox b, PairParams p, const int *__restrict__ order,
                const int *__restrict__ neighPair, const long long *__restrict__ off,
                const int *__restrict__ list, const double *__restrict__ x,
                const double *__restrict__ y, const double *__restrict__ z,
                const double *__restrict__ q, const double *__restrict__ eps,
                const double *__restrict__ sig, const double *__restrict__ vx,
                const double *__restrict__ vy, const double *__restrict__ vz, AdjOut o) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = order[t];
  const long long start = off[t];
  const int cnt = neighPair[i];
  double acc[10] = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0.};
  for (int k = 0; k < cnt; ++k) {
    const int j = list[start + k];
    double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
    const double r2 = dist_d(b, dx, dy, dz);
    if (r2 <= p.cutOff2)
      adj_pair(p, i, j, dx, dy, dz, r2, false, q, eps, sig, vx, vy, vz, o, acc);
  }
  adj_flush(i, acc, vx != nullptr, o);
}

// Excluded pairs (j > i of each row, no cut-off) and the self term.
__global__ void __launch_bounds__(128)
k_adjoint_excl(int n, DevBox b, PairParams p, const int *__restrict__ exclStart,
               const int *__restrict__ exclFlat, const double *__restrict__ x,
               const double *__restrict__ y, const double *__restrict__ z,
               const double *__restrict__ q, const double *__restrict__ eps,
               const double *__restrict__ sig, const double *__restrict__ vx,
               const double *__restrict__ vy, const double *__restrict__ vz, AdjOut o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc[10] = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0.};
  acc[0] = -2.0 * p.chargeConst * p.alpha * q[i] / kSqrtPi;  // self term
  const int e = exclStart[i + 1];
  for (int k = exclStart[i]; k < e; ++k) {
    const int j = exclFlat[k];
    if (j <= i) continue;
    double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
    const double r2 = dist_d(b, dx, dy, dz);
    adj_pair(p, i, j, dx, dy, dz, r2, true, q, eps, sig, vx, vy, vz, o, acc);
  }
  adj_flush(i, acc, vx != nullptr, o);
}

}  // namespace

extern "C" int mdbas_nb_engine_adjoint(mdbas_nb_engine *e, const double *vx, const double *vy,
                                       const double *vz, double *gq, double *geps, double *gsig,
                                       double *hx, double *hy, double *hz, double *pq,
                                       double *peps, double *psig, int device_ptrs) {
  if (!e || !gq || !geps || !gsig) return MDBAS_NB_ERR_ARG;
  const bool hvp = vx != nullptr;
  if (hvp && (!vy || !vz || !hx || !hy || !hz || !pq || !peps || !psig)) return MDBAS_NB_ERR_ARG;
  if (e->cfg.precision != 0) {
    set_last_status(MDBAS_NB_ERR_UNSUPPORTED, "the adjoint runs on the FP64 form (precision 0)");
    return MDBAS_NB_ERR_UNSUPPORTED;
  }
  if (!e->built) return MDBAS_NB_ERR_STATE;
  MDB_CUDA(cudaSetDevice(e->device));
  LaunchScope ls(e);
  const int n = e->n;
  cudaStream_t s = e->stream;
  // device scratch: 3 (v) + 9 (outputs) arrays of n
  MDB_TRY(e->adjBuf.ensure(sizeof(double) * 12 * (size_t)n));
  double *buf = e->adjBuf.as<double>();
  double *dv = buf, *outs = buf + 3 * (size_t)n;
  MDB_CUDA(cudaMemsetAsync(outs, 0, sizeof(double) * 9 * (size_t)n, s));
  const cudaMemcpyKind in = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind outk = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t bytes = sizeof(double) * (size_t)n;
  if (hvp) {
    MDB_CUDA(cudaMemcpyAsync(dv, vx, bytes, in, s));
    MDB_CUDA(cudaMemcpyAsync(dv + n, vy, bytes, in, s));
    MDB_CUDA(cudaMemcpyAsync(dv + 2 * (size_t)n, vz, bytes, in, s));
  }
  AdjOut o;
  double *const ptrs[9] = {outs, outs + n, outs + 2 * (size_t)n, outs + 3 * (size_t)n,
                           outs + 4 * (size_t)n, outs + 5 * (size_t)n, outs + 6 * (size_t)n,
                           outs + 7 * (size_t)n, outs + 8 * (size_t)n};
  o.gq = ptrs[0]; o.geps = ptrs[1]; o.gsig = ptrs[2];
  o.hx = ptrs[3]; o.hy = ptrs[4]; o.hz = ptrs[5];
  o.pq = ptrs[6]; o.peps = ptrs[7]; o.psig = ptrs[8];
  const double *dvx = hvp ? dv : nullptr, *dvy = hvp ? dv + n : nullptr,
               *dvz = hvp ? dv + 2 * (size_t)n : nullptr;
  MDB_LAUNCH(k_adjoint_pairs, grid_for(n, 128), 128, 0, s, n, e->box, e->pp,
             e->ref.order.as<int>(), e->ref.neighPair.as<int>(), e->ref.off.as<long long>(),
             e->ref.list.as<int>(), e->x.as<double>(), e->y.as<double>(), e->z.as<double>(),
             e->q.as<double>(), e->eps.as<double>(), e->sig.as<double>(), dvx, dvy, dvz, o);
  MDB_LAUNCH(k_adjoint_excl, grid_for(n, 128), 128, 0, s, n, e->box, e->pp,
             e->exclStart.as<int>(), e->exclFlat.as<int>(), e->x.as<double>(),
             e->y.as<double>(), e->z.as<double>(), e->q.as<double>(), e->eps.as<double>(),
             e->sig.as<double>(), dvx, dvy, dvz, o);
  double *dst[9] = {gq, geps, gsig, hx, hy, hz, pq, peps, psig};
  for (int k = 0; k < (hvp ? 9 : 3); ++k)
    MDB_CUDA(cudaMemcpyAsync(dst[k], ptrs[k], bytes, outk, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  return MDBAS_NB_OK;
}
