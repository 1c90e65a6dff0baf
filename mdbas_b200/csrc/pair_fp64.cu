// pair_fp64.cu -- the plain FP64 GPU form of MDBas's pair loops.
//
// One thread per atom i (in neighOrder position), walking i's entries of the
// MDBas half list exactly as ewald_energy / nonbond_energy do
// (src/energy.c:480-561, :240-318): min-image by dist(), cut-off test,
// Ewald direct (src/ewald.c:356-369) or cut-off Coulomb (src/elec.c:137-263)
// plus vdw_switch (src/vdw.c:144-184), Newton's third law with the j update
// done by an FP64 atomic.  Exclusion corrections (src/energy.c:567-621) run
// one thread per atom over its j>i exclusion rows.
//
// This translation unit is compiled with --fmad=false and every expression
// keeps MDBas's association order; results differ from MDBas's CPU build only
// through CUDA's erfc/erf/exp (a few ulp from glibc) and the order of the
// FP64 atomic additions.
#include "common.cuh"
#include "pair_fp64.cuh"

namespace mdbas {

namespace {

__device__ __forceinline__ double ewald_dir_d(const PairParams &p, double &dE, double qel, double r,
                                              double rt) {
  const double alphar = p.alpha * r;
  const double e = qel * erfc(alphar) * rt;
  dE = 2.0 * qel * p.alpha * exp(-(alphar * alphar)) / kSqrtPi;
  dE = -(e + dE) * rt;
  return e;
}

__device__ __forceinline__ double ewald_corr_d(const PairParams &p, double &dE, double qel,
                                               double r, double rt) {
  const double alphar = p.alpha * r;
  const double e = -qel * erf(alphar) * rt;
  dE = 2.0 * qel * p.alpha * exp(-(alphar * alphar)) / kSqrtPi;
  dE = -(e + dE) * rt;
  return e;
}

__device__ __forceinline__ double vdw_switch_d(const PairParams &p, double &dvdw, double veps,
                                               double vsig, double r2, double rt) {
  if (!p.vdwSwitch) {
    dvdw = 0.;
    return 0.;
  }
  const double t = vsig * rt;
  const double v6 = (t * t * t) * (t * t * t);
  const double v12 = v6 * v6;
  if (r2 <= p.cutOn2) {
    dvdw = 24. * veps * rt * (v6 - 2. * v12);
    return 4. * veps * (v12 - v6);
  }
  const double s1 = p.cutOff2 - r2;
  const double sf = (s1 * s1) * (p.cutOff2 + 2. * r2 - 3. * p.cutOn2) * p.switch2;
  const double dsf = 12. * r2 * s1 * (p.cutOn2 - r2) * p.switch2;
  const double pv = 4. * veps * (v12 - v6);
  const double dpv = 24. * veps * (v6 - 2. * v12);
  dvdw = pv * dsf + dpv * sf;
  dvdw *= rt;
  return pv * sf;
}

// coulomb_shift1 / shift2 / switch / none (src/elec.c:25-263).
__device__ __forceinline__ double coulomb_d(const PairParams &p, double &delec, double qel,
                                            double r2, double rt) {
  double s1, s2, sf, dsf, pelec;
  switch (p.elecType) {
    case SHIFT1:
      s1 = rt * r2 * p.rcutOff;
      s2 = r2 * p.rcutOff2;
      sf = 1. - 2. * s1 + s2;
      dsf = 2. * (s2 - s1);
      pelec = p.chargeConst * qel * rt;
      delec = pelec * rt * (dsf - sf);
      return pelec * sf;
    case SHIFT2:
      s1 = r2 * p.rcutOff2;
      s2 = s1 * s1;
      sf = 1. - 2. * s1 + s2;
      dsf = 4. * (s2 - s1);
      pelec = p.chargeConst * qel * rt;
      delec = pelec * rt * (dsf - sf);
      return pelec * sf;
    case SWITCH:
      if (r2 <= p.cutOn2) {
        pelec = p.chargeConst * qel * rt;
        delec = -pelec * rt;
        return pelec;
      }
      s1 = p.cutOff2 - r2;
      sf = (s1 * s1) * (p.cutOff2 + 2. * r2 - 3. * p.cutOn2) * p.switch2;
      dsf = 12. * r2 * s1 * (p.cutOn2 - r2) * p.switch2;
      pelec = p.chargeConst * qel * rt;
      delec = pelec * rt * (dsf - sf);
      return pelec * sf;
    default:
      delec = 0.;
      return 0.;
  }
}

// acc[0..4]: elec, vdw, virelec, virvdw, in-cut-off pairs.
template <bool EWALD>
__global__ void __launch_bounds__(128)
k_pairs_fp64(int n, DevBox b, PairParams p, const int *__restrict__ order,
             const int *__restrict__ neighPair, const long long *__restrict__ off,
             const int *__restrict__ list, const double *__restrict__ x,
             const double *__restrict__ y, const double *__restrict__ z,
             const double *__restrict__ q, const double *__restrict__ eps,
             const double *__restrict__ sig, double *__restrict__ fx, double *__restrict__ fy,
             double *__restrict__ fz, double *__restrict__ acc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double eel = 0., evdw = 0., virel = 0., virvdw = 0., npair = 0.;
  if (t < n) {
    const int i = order[t];
    const long long start = off[t];
    const int cnt = neighPair[i];
    const double xi = x[i], yi = y[i], zi = z[i], qi = q[i], ei = eps[i], si = sig[i];
    double fxi = 0., fyi = 0., fzi = 0.;
    for (int k = 0; k < cnt; ++k) {
      const int j = list[start + k];
      double dx = x[j] - xi, dy = y[j] - yi, dz = z[j] - zi;
      const double r2 = dist_d(b, dx, dy, dz);
      const double r = sqrt(r2);
      const double rt = 1. / r;
      if (r2 <= p.cutOff2) {
        double delec, dvdw;
        npair += 1.;
        if (EWALD) {
          const double qel = p.chargeConst * qi * q[j];
          eel += ewald_dir_d(p, delec, qel, r, rt);
        } else {
          eel += coulomb_d(p, delec, qi * q[j], r2, rt);
        }
        evdw += vdw_switch_d(p, dvdw, ei * eps[j], si + sig[j], r2, rt);
        virel += delec * r;
        virvdw += dvdw * r;
        const double fxj = (delec + dvdw) * dx * rt;
        const double fyj = (delec + dvdw) * dy * rt;
        const double fzj = (delec + dvdw) * dz * rt;
        fxi += fxj;
        fyi += fyj;
        fzi += fzj;
        atomicAdd(fx + j, -fxj);
        atomicAdd(fy + j, -fyj);
        atomicAdd(fz + j, -fzj);
      }
    }
    atomicAdd(fx + i, fxi);
    atomicAdd(fy + i, fyi);
    atomicAdd(fz + i, fzi);
  }
  eel = warp_sum_d(eel);
  evdw = warp_sum_d(evdw);
  virel = warp_sum_d(virel);
  virvdw = warp_sum_d(virvdw);
  npair = warp_sum_d(npair);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc + 0, eel);
    atomicAdd(acc + 1, evdw);
    atomicAdd(acc + 2, virel);
    atomicAdd(acc + 3, virvdw);
    atomicAdd(acc + 4, npair);
  }
}

// Exclusion correction (src/energy.c:567-621): every excluded pair j>i, no
// cut-off.  acc[5], acc[6]: eCorr, virCorr.
__global__ void __launch_bounds__(128)
k_excl_fp64(int n, DevBox b, PairParams p, const int *__restrict__ exclStart,
            const int *__restrict__ exclFlat, const double *__restrict__ x,
            const double *__restrict__ y, const double *__restrict__ z,
            const double *__restrict__ q, double *__restrict__ fx, double *__restrict__ fy,
            double *__restrict__ fz, double *__restrict__ acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ecorr = 0., vcorr = 0.;
  if (i < n) {
    double fxi = 0., fyi = 0., fzi = 0.;
    const int e = exclStart[i + 1];
    for (int k = exclStart[i]; k < e; ++k) {
      const int j = exclFlat[k];
      if (j <= i) continue;
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      const double r2 = dist_d(b, dx, dy, dz);
      const double r = sqrt(r2);
      const double rt = 1. / r;
      const double qel = p.chargeConst * q[i] * q[j];
      double dE;
      ecorr += ewald_corr_d(p, dE, qel, r, rt);
      vcorr += dE * r;
      const double fxj = dE * dx * rt;
      const double fyj = dE * dy * rt;
      const double fzj = dE * dz * rt;
      fxi += fxj;
      fyi += fyj;
      fzi += fzj;
      atomicAdd(fx + j, -fxj);
      atomicAdd(fy + j, -fyj);
      atomicAdd(fz + j, -fzj);
    }
    if (fxi != 0. || fyi != 0. || fzi != 0.) {
      atomicAdd(fx + i, fxi);
      atomicAdd(fy + i, fyi);
      atomicAdd(fz + i, fzi);
    }
  }
  ecorr = warp_sum_d(ecorr);
  vcorr = warp_sum_d(vcorr);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc + 5, ecorr);
    atomicAdd(acc + 6, vcorr);
  }
}

// Ewald self term (src/ewald.c:165-171): sum q^2, each term rounded to a
// multiple of 2^-40 and summed as an integer, so the total does not depend on
// the atom order.  *acc receives the int64 sum.
__global__ void k_sum_q2(int n, const double *__restrict__ q, long long *__restrict__ acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  long long v = (i < n) ? __double2ll_rn(q[i] * q[i] * 1099511627776.0) : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red_add(acc, v);
}

// 1-4 pairs: ewald14_energy (src/energy.c:654-742) with ewald_dir14/corr14
// (src/ewald.c:386-413) and vdw14_switch (src/vdw.c:270-311), or
// nonbond14_energy (src/energy.c:356-439) with coulomb14_* (src/elec.c:265-465).
// One thread per pair; acc[0..3] += elec, vdw, virelec, virvdw.
template <bool EWALD>
__global__ void __launch_bounds__(128)
k_pairs14(int npair, DevBox b, PairParams p, const int *__restrict__ list14,
          const double *__restrict__ x, const double *__restrict__ y,
          const double *__restrict__ z, const double *__restrict__ q,
          const double *__restrict__ eps, const double *__restrict__ sig,
          double *__restrict__ fx, double *__restrict__ fy, double *__restrict__ fz,
          double *__restrict__ acc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double eel = 0., evdw = 0., virel = 0., virvdw = 0.;
  if (k < npair) {
    const int i = list14[2 * k], j = list14[2 * k + 1];
    double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
    const double r2 = dist_d(b, dx, dy, dz);
    const double r = sqrt(r2);
    const double rt = 1. / r;
    double delec = 0., dcorr = 0., dvdw = 0.;
    if (EWALD) {
      const double qel = p.chargeConst * q[i] * q[j];
      const double alphar = p.alpha * r;
      const double ed = p.scal14 * qel * erfc(alphar) * rt;
      delec = 2.0 * p.scal14 * qel * p.alpha * exp(-(alphar * alphar)) / kSqrtPi;
      delec = -(ed + delec) * rt;
      const double ec = (p.scal14 - 1.0) * qel * erf(alphar) * rt;
      dcorr = 2.0 * (p.scal14 - 1.0) * qel * p.alpha * exp(-(alphar * alphar)) / kSqrtPi;
      dcorr = (dcorr - ec) * rt;
      eel = ed + ec;
      virel = delec * r + dcorr * r;
    } else {
      const double qel = q[i] * q[j];
      double s1, s2, sf, dsf, pelec;
      switch (p.elecType) {
        case SHIFT1:
          if (r2 <= p.cutOff2) {
            s1 = rt * r2 * p.rcutOff;
            s2 = r2 * p.rcutOff2;
            sf = 1. - 2. * s1 + s2;
            dsf = 2. * (s2 - s1);
            pelec = p.scal14 * p.chargeConst * qel * rt;
            eel = pelec * sf;
            delec = pelec * rt * (dsf - sf);
          }
          break;
        case SHIFT2:
          if (r2 <= p.cutOff2) {
            s1 = r2 * p.rcutOff2;
            s2 = s1 * s1;
            sf = 1. - 2. * s1 + s2;
            dsf = 4. * (s2 - s1);
            pelec = p.scal14 * p.chargeConst * qel * rt;
            eel = pelec * sf;
            delec = pelec * rt * (dsf - sf);
          }
          break;
        case SWITCH:
          if (r2 <= p.cutOn2) {
            pelec = p.scal14 * p.chargeConst * qel * rt;
            eel = pelec;
            delec = -pelec * rt;
          } else if (r2 <= p.cutOff2) {
            s1 = p.cutOff2 - r2;
            sf = (s1 * s1) * (p.cutOff2 + 2. * r2 - 3. * p.cutOn2) * p.switch2;
            dsf = 12. * r2 * s1 * (p.cutOn2 - r2) * p.switch2;
            pelec = p.scal14 * p.chargeConst * qel * rt;
            eel = pelec * sf;
            delec = pelec * rt * (dsf - sf);
          }
          break;
        default:
          break;
      }
      virel = delec * r;
    }
    if (p.vdwSwitch) {
      const double veps = eps[i] * eps[j], vsig = sig[i] + sig[j];
      const double t = vsig * rt;
      const double v6 = (t * t * t) * (t * t * t);
      const double v12 = v6 * v6;
      if (r2 <= p.cutOn2) {
        evdw = 4. * p.scal14 * veps * (v12 - v6);
        dvdw = 24. * p.scal14 * veps * rt * (v6 - 2. * v12);
      } else if (r2 <= p.cutOff2) {
        const double s1 = p.cutOff2 - r2;
        const double sf = (s1 * s1) * (p.cutOff2 + 2. * r2 - 3. * p.cutOn2) * p.switch2;
        const double dsf = 12. * r2 * s1 * (p.cutOn2 - r2) * p.switch2;
        const double pv = 4. * p.scal14 * veps * (v12 - v6);
        const double dpv = 24. * p.scal14 * veps * (v6 - 2. * v12);
        evdw = pv * sf;
        dvdw = pv * dsf + dpv * sf;
        dvdw *= rt;
      }
    }
    virvdw = dvdw * r;
    const double fxj = (delec + dcorr + dvdw) * dx * rt;
    const double fyj = (delec + dcorr + dvdw) * dy * rt;
    const double fzj = (delec + dcorr + dvdw) * dz * rt;
    atomicAdd(fx + i, fxj);
    atomicAdd(fy + i, fyj);
    atomicAdd(fz + i, fzj);
    atomicAdd(fx + j, -fxj);
    atomicAdd(fy + j, -fyj);
    atomicAdd(fz + j, -fzj);
  }
  eel = warp_sum_d(eel);
  evdw = warp_sum_d(evdw);
  virel = warp_sum_d(virel);
  virvdw = warp_sum_d(virvdw);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc + 0, eel);
    atomicAdd(acc + 1, evdw);
    atomicAdd(acc + 2, virel);
    atomicAdd(acc + 3, virvdw);
  }
}

}  // namespace

int pairs_fp64(int ewald, int n, const DevBox &b, const PairParams &p, const int *order,
               const int *neighPair, const long long *off, const int *list, const double *x,
               const double *y, const double *z, const double *q, const double *eps,
               const double *sig, double *fx, double *fy, double *fz, double *acc,
               cudaStream_t s) {
  if (n <= 0) return MDBAS_NB_OK;
  if (ewald)
    MDB_LAUNCH(k_pairs_fp64<true>, grid_for(n, 128), 128, 0, s, n, b, p, order, neighPair, off,
               list, x, y, z, q, eps, sig, fx, fy, fz, acc);
  else
    MDB_LAUNCH(k_pairs_fp64<false>, grid_for(n, 128), 128, 0, s, n, b, p, order, neighPair, off,
               list, x, y, z, q, eps, sig, fx, fy, fz, acc);
  return MDBAS_NB_OK;
}

int excl_fp64(int n, const DevBox &b, const PairParams &p, const int *exclStart,
              const int *exclFlat, const double *x, const double *y, const double *z,
              const double *q, double *fx, double *fy, double *fz, double *acc,
              cudaStream_t s) {
  if (n <= 0) return MDBAS_NB_OK;
  MDB_LAUNCH(k_excl_fp64, grid_for(n, 128), 128, 0, s, n, b, p, exclStart, exclFlat, x, y, z, q,
             fx, fy, fz, acc);
  return MDBAS_NB_OK;
}

int pairs14_fp64(int ewald, int npair, const DevBox &b, const PairParams &p, const int *list14,
                 const double *x, const double *y, const double *z, const double *q,
                 const double *eps, const double *sig, double *fx, double *fy, double *fz,
                 double *acc, cudaStream_t s) {
  if (npair <= 0) return MDBAS_NB_OK;
  if (ewald)
    MDB_LAUNCH(k_pairs14<true>, grid_for(npair, 128), 128, 0, s, npair, b, p, list14, x, y, z, q,
               eps, sig, fx, fy, fz, acc);
  else
    MDB_LAUNCH(k_pairs14<false>, grid_for(npair, 128), 128, 0, s, npair, b, p, list14, x, y, z,
               q, eps, sig, fx, fy, fz, acc);
  return MDBAS_NB_OK;
}

int sum_q2(int n, const double *q, long long *acc, cudaStream_t s) {
  if (n <= 0) return MDBAS_NB_OK;
  MDB_LAUNCH(k_sum_q2, grid_for(n, 256), 256, 0, s, n, q, acc);
  return MDBAS_NB_OK;
}

}  // namespace mdbas
