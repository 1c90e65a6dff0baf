// ewald_rec.cu -- MDBas's explicit reciprocal-space Ewald sum on the GPU:
// init_ewald, ewald_free and ewald_rec (include/ewald.h; src/ewald.c:10-354).
//
// MDBas sums over every k = 2 pi (m1 u + m2 v + m3 w) inside the reciprocal
// cut-off, in the order m1 = 0..m1max, m2, m3 (half space: the (0, 0, m3 > 0)
// row first), with per-atom tables of cos/sin(m s) built by the angle-
// addition recurrence.  Here:
//
//   * the k list (and e^{-k^2/4a^2}/k^2, the virial factor) is built on the
//     host with MDBas's expressions and cached per box, alpha and m-range;
//   * k_ewald_sf: one thread per k-vector sums q_i e^{i k.r_i} over a range
//     of atoms; a tile of atoms at a time has its cos/sin tables built in
//     shared memory with MDBas's recurrence; partial sums per atom range are
//     added in a fixed order by k_ewald_kdata (deterministic);
//   * k_ewald_forces: one thread per atom walks the k list in MDBas's order
//     (rows of fixed (m1, m2), m3 contiguous), so each force component is
//     accumulated in MDBas's order; its m3 table sits in shared memory.
//
// This file is compiled with --fmad=false: the table recurrences and the
// per-(atom, k) products are MDBas's operations; only cos/sin of the first
// table entry (CUDA's vs the host's) and the order of the sums over atoms
// differ.
#include <math.h>
#include <string.h>

#include <vector>

#include "kspace.cuh"

namespace mdbas {
namespace {

constexpr double kTwoPi = 6.283185307179586;  // include/global.h:54
constexpr double kPi = 3.141592653589793;
constexpr int kSfThreads = 256;               // k-vectors per structure-factor block

struct EwBox {
  double u1, u2, u3, v1, v2, v3, w1, w2, w3;
};

// scaled fractional coordinate of one dimension, MDBas's expression
__device__ __forceinline__ double frac_s(const EwBox &b, int d, double x, double y, double z) {
  if (d == 0) return kTwoPi * (x * b.u1 + y * b.u2 + z * b.u3);
  if (d == 1) return kTwoPi * (x * b.v1 + y * b.v2 + z * b.v3);
  return kTwoPi * (x * b.w1 + y * b.w2 + z * b.w3);
}

// c[m] = cos(m s), sn[m] = sin(m s) for m = 0..M by MDBas's recurrence
// (src/ewald.c:196-227); stride between entries `st`.
__device__ __forceinline__ void ew_table(double s, int M, double *c, double *sn, int st) {
  c[0] = 1.0;
  sn[0] = 0.0;
  if (M < 1) return;
  const double c1 = cos(s), s1 = sin(s);
  c[st] = c1;
  sn[st] = s1;
  double cp = c1, sp = s1;
  for (int m = 2; m <= M; ++m) {
    const double cn = cp * c1 - sp * s1;
    const double snn = sp * c1 + cp * s1;
    c[(size_t)m * st] = cn;
    sn[(size_t)m * st] = snn;
    cp = cn;
    sp = snn;
  }
}

// Structure factors: part[(2p) K + k], part[(2p+1) K + k] = sum over the atoms
// of range p of q_i cos(k.r_i), q_i sin(k.r_i).
__global__ void __launch_bounds__(kSfThreads)
    k_ewald_sf(int n, int K, int perPart, int tile, EwBox b, int M1, int M2, int M3,
               const int4 *__restrict__ km, const double *__restrict__ x,
               const double *__restrict__ y, const double *__restrict__ z,
               const double *__restrict__ q, double *__restrict__ part) {
  extern __shared__ double sh[];
  const int W = 2 * (M1 + M2 + M3 + 3);  // doubles per atom
  double *qs = sh + (size_t)tile * W;
  const int o1s = M1 + 1, o2c = 2 * (M1 + 1), o2s = o2c + M2 + 1, o3c = o2s + M2 + 1,
            o3s = o3c + M3 + 1;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  int m1 = 0, am2 = 0, am3 = 0;
  double sg2 = 1., sg3 = 1.;
  if (k < K) {
    const int4 t = km[k];
    m1 = t.x;
    am2 = abs(t.y);
    am3 = abs(t.z);
    sg2 = t.y < 0 ? -1. : 1.;
    sg3 = t.z < 0 ? -1. : 1.;
  }
  double sc = 0., ss = 0.;
  const int a0 = blockIdx.y * perPart;
  const int a1 = min(n, a0 + perPart);
  for (int t0 = a0; t0 < a1; t0 += tile) {
    const int na = min(tile, a1 - t0);
    __syncthreads();
    for (int task = threadIdx.x; task < 3 * na; task += blockDim.x) {
      const int a = task / 3, d = task - 3 * a, i = t0 + a;
      const double s = frac_s(b, d, x[i], y[i], z[i]);
      double *base = sh + (size_t)a * W;
      if (d == 0) {
        ew_table(s, M1, base, base + o1s, 1);
        qs[a] = q[i];
      } else if (d == 1) {
        ew_table(s, M2, base + o2c, base + o2s, 1);
      } else {
        ew_table(s, M3, base + o3c, base + o3s, 1);
      }
    }
    __syncthreads();
    if (k < K) {
      for (int a = 0; a < na; ++a) {
        const double *base = sh + (size_t)a * W;
        const double c1 = base[m1], s1 = base[o1s + m1];
        const double c2 = base[o2c + am2], s2 = sg2 * base[o2s + am2];
        const double c3 = base[o3c + am3], s3 = sg3 * base[o3s + am3];
        const double cm = c1 * c2 - s1 * s2;
        const double smv = s1 * c2 + c1 * s2;
        const double qa = qs[a];
        sc += qa * (cm * c3 - smv * s3);
        ss += qa * (smv * c3 + cm * s3);
      }
    }
  }
  if (k < K) {
    part[(size_t)(2 * blockIdx.y) * K + k] = sc;
    part[(size_t)(2 * blockIdx.y + 1) * K + k] = ss;
  }
}

// Per k: the structure factor (range sums in order), its energy term and
// virial/stress terms (src/ewald.c:300-318); block partials of
// {energy, stress 0..5} into bpart[q * gridDim.x + block].
__global__ void k_ewald_kdata(int K, int P, const double *__restrict__ part,
                              const double4 *__restrict__ kv, const double *__restrict__ vam,
                              double2 *__restrict__ S, double *__restrict__ bpart) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double v[7] = {0., 0., 0., 0., 0., 0., 0.};
  if (k < K) {
    double sc = 0., ss = 0.;
    for (int p = 0; p < P; ++p) {
      sc += part[(size_t)(2 * p) * K + k];
      ss += part[(size_t)(2 * p + 1) * K + k];
    }
    S[k] = make_double2(sc, ss);
    const double4 t = kv[k];
    double virtmp = sc * sc + ss * ss;
    v[0] = t.w * virtmp;
    virtmp *= vam[k];
    v[1] = -(virtmp * t.x * t.x);
    v[2] = -(virtmp * t.x * t.y);
    v[3] = -(virtmp * t.x * t.z);
    v[4] = -(virtmp * t.y * t.y);
    v[5] = -(virtmp * t.y * t.z);
    v[6] = -(virtmp * t.z * t.z);
  }
  __shared__ double red[7][8];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const double s = warp_sum_d(v[j]);
    if (lane == 0) red[j][w] = s;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double s = 0.;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) s += red[threadIdx.x][j];
    bpart[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void k_ewald_finish(int nPart, const double *__restrict__ bpart,
                               double *__restrict__ sums) {
  __shared__ double red[8];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = 0; j < 7; ++j) {
    double s = 0.;
    for (int b = threadIdx.x; b < nPart; b += blockDim.x) s += bpart[(size_t)j * nPart + b];
    s = warp_sum_d(s);
    if (lane == 0) red[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
      sums[j] = t;
    }
    __syncthreads();
  }
}

// Forces: one thread per atom walks the rows in MDBas's order.  scaleInput:
// MDBas's ewald_rec multiplies the whole force arrays by fact0 at the end
// (src/ewald.c:335-340), f = fact0 (f_in + sum); otherwise f = f_in +
// fact0 sum.  t12: the atom's m1 and m2 tables, SoA [m][n] scratch.
__global__ void k_ewald_forces(int n, EwBox b, int M1, int M2, int M3, int nRows,
                               const int4 *__restrict__ rows, const int *__restrict__ rowK,
                               const double4 *__restrict__ kv, const double2 *__restrict__ S,
                               const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ q,
                               double *__restrict__ t12, double fact0, int scaleInput,
                               double *__restrict__ fx, double *__restrict__ fy,
                               double *__restrict__ fz) {
  extern __shared__ double sh[];
  const int T = blockDim.x;
  double *c3 = sh, *s3 = sh + (size_t)(M3 + 1) * T;
  const int i = blockIdx.x * T + threadIdx.x;
  if (i >= n) return;  // no block-wide synchronisation below
  const double xi = x[i], yi = y[i], zi = z[i], qi = q[i];
  double *c1 = t12, *s1 = c1 + (size_t)(M1 + 1) * n;
  double *c2 = s1 + (size_t)(M1 + 1) * n, *s2 = c2 + (size_t)(M2 + 1) * n;
  ew_table(frac_s(b, 0, xi, yi, zi), M1, c1 + i, s1 + i, n);
  ew_table(frac_s(b, 1, xi, yi, zi), M2, c2 + i, s2 + i, n);
  ew_table(frac_s(b, 2, xi, yi, zi), M3, c3 + threadIdx.x, s3 + threadIdx.x, T);
  double ax = fx[i], ay = fy[i], az = fz[i];
  if (!scaleInput) ax = ay = az = 0.;
  for (int r = 0; r < nRows; ++r) {
    const int4 row = rows[r];  // m1, m2, first m3, last m3
    const int am2 = abs(row.y);
    const double sg2 = row.y < 0 ? -1. : 1.;
    const double a1c = c1[(size_t)row.x * n + i], a1s = s1[(size_t)row.x * n + i];
    const double a2c = c2[(size_t)am2 * n + i], a2s = sg2 * s2[(size_t)am2 * n + i];
    const double cm = a1c * a2c - a1s * a2s;
    const double smv = a1s * a2c + a1c * a2s;
    int k = rowK[r];
    for (int m3 = row.z; m3 <= row.w; ++m3, ++k) {
      const int am3 = abs(m3);
      const double sg3 = m3 < 0 ? -1. : 1.;
      const double t3c = c3[(size_t)am3 * T + threadIdx.x];
      const double t3s = sg3 * s3[(size_t)am3 * T + threadIdx.x];
      const double cms = qi * (cm * t3c - smv * t3s);
      const double sms = qi * (smv * t3c + cm * t3s);
      const double4 kk = kv[k];
      const double2 sk = S[k];
      const double de = kk.w * (sms * sk.x - cms * sk.y);
      ax += kk.x * de;
      ay += kk.y * de;
      az += kk.z * de;
    }
  }
  if (scaleInput) {
    fx[i] = ax * fact0;
    fy[i] = ay * fact0;
    fz[i] = az * fact0;
  } else {
    fx[i] += ax * fact0;
    fy[i] += ay * fact0;
    fz[i] += az * fact0;
  }
}

// The standalone calls' state (the engine keeps its own).
EwaldWork &ewald_ctx() {
  static EwaldWork c;
  return c;
}

// k list of one box / alpha / m-range, built on the host with MDBas's
// expressions (src/ewald.c:146-150, 255-300).
int build_klist(EwaldKList &kl, const PBC *box, double alpha, int M1, int M2, int M3) {
  const double key[12] = {box->u1, box->u2, box->u3, box->v1, box->v2, box->v3, box->w1,
                          box->w2, box->w3, alpha, box->u + box->v + box->w,
                          (double)M1 + 1000. * M2 + 1.e6 * M3};
  if (kl.valid && memcmp(key, kl.key, sizeof(key)) == 0) return MDBAS_NB_OK;
  kl.valid = false;
  const double rAlpha2 = -0.25 / (alpha * alpha);
  double rc = fmin(((double)M1 * box->u), ((double)M2 * box->v));
  rc = fmin(rc, (double)M3 * box->w);
  rc = rc * 1.05 * kTwoPi;
  const double rc2 = rc * rc;
  std::vector<int4> km, rows;
  std::vector<double4> kv;
  std::vector<double> vam;
  std::vector<int> rowK;
  int m2min = 0, m3min = 1;
  for (int m1 = 0; m1 <= M1; ++m1) {
    const double rm1x = kTwoPi * box->u1 * (double)m1;
    const double rm1y = kTwoPi * box->u2 * (double)m1;
    const double rm1z = kTwoPi * box->u3 * (double)m1;
    for (int m2 = m2min; m2 <= M2; ++m2) {
      const double rm2x = rm1x + (kTwoPi * box->v1 * (double)m2);
      const double rm2y = rm1y + (kTwoPi * box->v2 * (double)m2);
      const double rm2z = rm1z + (kTwoPi * box->v3 * (double)m2);
      int lo = 0, last = 0;
      bool open = false;
      for (int m3 = m3min; m3 <= M3; ++m3) {
        const double rmx = rm2x + (kTwoPi * box->w1 * (double)m3);
        const double rmy = rm2y + (kTwoPi * box->w2 * (double)m3);
        const double rmz = rm2z + (kTwoPi * box->w3 * (double)m3);
        const double rm = rmx * rmx + rmy * rmy + rmz * rmz;
        if (rm <= rc2) {
          // in-cut-off m3 of a row are contiguous (|a + m3 b|^2 is convex in m3)
          if (open && m3 != last + 1) {
            rows.push_back(make_int4(m1, m2, lo, last));
            rowK.push_back((int)km.size() - (last - lo + 1));
            open = false;
          }
          if (!open) {
            lo = m3;
            open = true;
          }
          last = m3;
          const double rrm = 1.0 / rm;
          const double am = exp(rAlpha2 * rm) * rrm;
          km.push_back(make_int4(m1, m2, m3, 0));
          kv.push_back(make_double4(rmx, rmy, rmz, am));
          vam.push_back(2.0 * am * (rrm - rAlpha2));
        }
      }
      if (open) {
        rows.push_back(make_int4(m1, m2, lo, last));
        rowK.push_back((int)km.size() - (last - lo + 1));
      }
      m3min = -M3;
    }
    m2min = -M2;
  }
  kl.K = (int)km.size();
  kl.nRows = (int)rows.size();
  kl.M1 = M1;
  kl.M2 = M2;
  kl.M3 = M3;
  const size_t K1 = km.empty() ? 1 : km.size(), R1 = rows.empty() ? 1 : rows.size();
  MDB_TRY(kl.km.ensure(sizeof(int4) * K1));
  MDB_TRY(kl.kv.ensure(sizeof(double4) * K1));
  MDB_TRY(kl.vam.ensure(sizeof(double) * K1));
  MDB_TRY(kl.rows.ensure(sizeof(int4) * R1));
  MDB_TRY(kl.rowK.ensure(sizeof(int) * R1));
  if (kl.K) {
    MDB_CUDA(cudaMemcpy(kl.km.p, km.data(), sizeof(int4) * km.size(), cudaMemcpyHostToDevice));
    MDB_CUDA(cudaMemcpy(kl.kv.p, kv.data(), sizeof(double4) * kv.size(), cudaMemcpyHostToDevice));
    MDB_CUDA(cudaMemcpy(kl.vam.p, vam.data(), sizeof(double) * vam.size(),
                        cudaMemcpyHostToDevice));
    MDB_CUDA(cudaMemcpy(kl.rows.p, rows.data(), sizeof(int4) * rows.size(),
                        cudaMemcpyHostToDevice));
    MDB_CUDA(cudaMemcpy(kl.rowK.p, rowK.data(), sizeof(int) * rowK.size(),
                        cudaMemcpyHostToDevice));
  }
  memcpy(kl.key, key, sizeof(key));
  kl.valid = true;
  return MDBAS_NB_OK;
}

EwBox make_ew_box(const PBC *p) {
  EwBox b;
  b.u1 = p->u1; b.u2 = p->u2; b.u3 = p->u3;
  b.v1 = p->v1; b.v2 = p->v2; b.v3 = p->v3;
  b.w1 = p->w1; b.w2 = p->w2; b.w3 = p->w3;
  return b;
}

int ewald_launch_impl(EwaldWork &c, int n, const PBC *box, double alpha, double chargeConst,
                      int M1, int M2, int M3, const double *x, const double *y, const double *z,
                      const double *q, double *fx, double *fy, double *fz, int scaleInput,
                      cudaStream_t s) {
  int dev = 0;
  MDB_CUDA(cudaGetDevice(&dev));
  if (c.device != dev) {
    c.kl.valid = false;
    c.device = dev;
  }
  MDB_TRY(build_klist(c.kl, box, alpha, M1, M2, M3));
  const EwaldKList &kl = c.kl;
  const EwBox b = make_ew_box(box);
  const int K = kl.K;
  // shared memory: the k-thread kernel's atom tile, the atom kernel's m3 table
  int maxSmem = 0;
  MDB_CUDA(cudaDeviceGetAttribute(&maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t perAtom = sizeof(double) * (2 * (size_t)(M1 + M2 + M3 + 3) + 1);
  int tile = (int)((size_t)(maxSmem / 2) / perAtom);
  if (tile > 64) tile = 64;
  int fThreads = 128;
  while (fThreads > 32 && sizeof(double) * 2 * (size_t)(M3 + 1) * fThreads > (size_t)maxSmem / 2)
    fThreads /= 2;
  if (tile < 1 || sizeof(double) * 2 * (size_t)(M3 + 1) * fThreads > (size_t)maxSmem) {
    set_last_status(MDBAS_NB_ERR_UNSUPPORTED, "reciprocal m-range too large for shared memory");
    return MDBAS_NB_ERR_UNSUPPORTED;
  }
  const size_t smemF = sizeof(double) * 2 * (size_t)(M3 + 1) * fThreads;
  MDB_TRY(c.t12.ensure(sizeof(double) * 2 * (size_t)(M1 + M2 + 2) * n));
  MDB_TRY(c.S.ensure(sizeof(double2) * (size_t)(K > 0 ? K : 1)));
  MDB_TRY(c.sums.ensure(sizeof(double) * 8));
  if (K == 0) MDB_CUDA(cudaMemsetAsync(c.sums.p, 0, sizeof(double) * 8, s));
  if (K > 0) {
    const int kBlocks = (K + kSfThreads - 1) / kSfThreads;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int P = (4 * sms + kBlocks - 1) / kBlocks;
    P = P < 1 ? 1 : P > 32 ? 32 : P;
    if (P > n) P = n;
    const int perPart = (n + P - 1) / P;
    const size_t smemSf = perAtom * (size_t)tile;
    MDB_CUDA(cudaFuncSetAttribute(k_ewald_sf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smemSf));
    MDB_TRY(c.part.ensure(sizeof(double) * 2 * (size_t)P * K));
    const int kdBlocks = (K + 255) / 256;
    MDB_TRY(c.bpart.ensure(sizeof(double) * 7 * (size_t)kdBlocks));
    MDB_LAUNCH(k_ewald_sf, dim3(kBlocks, P), kSfThreads, smemSf, s, n, K, perPart, tile, b, M1,
               M2, M3, kl.km.as<int4>(), x, y, z, q, c.part.as<double>());
    MDB_LAUNCH(k_ewald_kdata, kdBlocks, 256, 0, s, K, P, c.part.as<double>(),
               kl.kv.as<double4>(), kl.vam.as<double>(), c.S.as<double2>(),
               c.bpart.as<double>());
    MDB_LAUNCH(k_ewald_finish, 1, 256, 0, s, kdBlocks, c.bpart.as<double>(),
               c.sums.as<double>());
  }
  const double rVol = kTwoPi / box->vol;
  const double fact1 = 2.0 * rVol * chargeConst;
  const double fact0 = 2.0 * fact1;
  MDB_CUDA(cudaFuncSetAttribute(k_ewald_forces, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smemF));
  MDB_LAUNCH(k_ewald_forces, grid_for(n, fThreads), fThreads, smemF, s, n, b, M1, M2, M3,
             kl.nRows, kl.rows.as<int4>(), kl.rowK.as<int>(), kl.kv.as<double4>(),
             c.S.as<double2>(), x, y, z, q, c.t12.as<double>(), fact0, scaleInput, fx, fy, fz);
  c.fact1 = fact1;
  return MDBAS_NB_OK;
}

// Device arrays; out[0] = energy (reciprocal + self + non-neutral), out[1] =
// virial, out[2..7] = stress.
int ewald_run(int n, const PBC *box, double alpha, double chargeConst, int M1, int M2, int M3,
              const double *x, const double *y, const double *z, const double *q, double systq,
              double sumq2, double *fx, double *fy, double *fz, int scaleInput, double out[8],
              cudaStream_t s) {
  EwaldWork &c = ewald_ctx();
  MDB_TRY(ewald_launch_impl(c, n, box, alpha, chargeConst, M1, M2, M3, x, y, z, q, fx, fy, fz,
                            scaleInput, s));
  double h[7];
  MDB_CUDA(cudaMemcpyAsync(h, c.sums.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  const double fact1 = c.fact1;
  // src/ewald.c:323-352
  const double eself = -chargeConst * alpha * sumq2 / kSqrtPi;
  const double enn = -(0.5 * kPi * chargeConst) * ((systq / alpha) * (systq / alpha) / box->vol);
  const double etmp = h[0];
  double st[6];
  st[0] = fact1 * (h[1] + etmp) + enn;
  st[1] = fact1 * h[2];
  st[2] = fact1 * h[3];
  st[3] = fact1 * (h[4] + etmp) + enn;
  st[4] = fact1 * h[5];
  st[5] = fact1 * (h[6] + etmp) + enn;
  out[0] = fact1 * etmp + eself + enn;
  out[1] = -(st[0] + st[3] + st[5]);
  for (int k = 0; k < 6; ++k) out[2 + k] = st[k];
  return MDBAS_NB_OK;
}

int nint_h(double x) { return (x >= 0.) ? (int)(x + 0.5) : (int)(x - 0.5); }

// host arrays staged through device buffers
int ewald_host(int n, const PBC *box, double alpha, double chargeConst, int M1, int M2, int M3,
               const double *x, const double *y, const double *z, const double *q, double *fx,
               double *fy, double *fz, int scaleInput, double out[8]) {
  EwaldWork &c = ewald_ctx();
  double systq = 0., sumq2 = 0.;
  for (int i = 0; i < n; ++i) {  // src/ewald.c:166-172
    systq += q[i];
    sumq2 += q[i] * q[i];
  }
  cudaStream_t s = nullptr;
  MDB_TRY(c.xyzq.ensure(sizeof(double) * 4 * (size_t)n));
  MDB_TRY(c.f.ensure(sizeof(double) * 3 * (size_t)n));
  double *d = c.xyzq.as<double>(), *f = c.f.as<double>();
  const size_t bytes = sizeof(double) * (size_t)n;
  MDB_CUDA(cudaMemcpyAsync(d, x, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d + n, y, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d + 2 * (size_t)n, z, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d + 3 * (size_t)n, q, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(f, fx, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(f + n, fy, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(f + 2 * (size_t)n, fz, bytes, cudaMemcpyHostToDevice, s));
  MDB_TRY(ewald_run(n, box, alpha, chargeConst, M1, M2, M3, d, d + n, d + 2 * (size_t)n,
                    d + 3 * (size_t)n, systq, sumq2, f, f + n, f + 2 * (size_t)n, scaleInput,
                    out, s));
  MDB_CUDA(cudaMemcpy(fx, f, bytes, cudaMemcpyDeviceToHost));
  MDB_CUDA(cudaMemcpy(fy, f + n, bytes, cudaMemcpyDeviceToHost));
  MDB_CUDA(cudaMemcpy(fz, f + 2 * (size_t)n, bytes, cudaMemcpyDeviceToHost));
  return MDBAS_NB_OK;
}

__global__ void k_kspace_fix(const double *__restrict__ src, double scale, double add,
                             long long *__restrict__ dst) {
  if (threadIdx.x == 0 && blockIdx.x == 0) dst[0] = fix_e(scale * src[0] + add);
}

}  // namespace

int ewald_launch(EwaldWork &c, int n, const PBC *box, double alpha, double chargeConst, int M1,
                 int M2, int M3, const double *x, const double *y, const double *z,
                 const double *q, double *fx, double *fy, double *fz, int scaleInput,
                 cudaStream_t s) {
  return ewald_launch_impl(c, n, box, alpha, chargeConst, M1, M2, M3, x, y, z, q, fx, fy, fz,
                           scaleInput, s);
}

int kspace_fix_launch(const double *src, double scale, double add, long long *dst,
                      cudaStream_t s) {
  MDB_LAUNCH(k_kspace_fix, 1, 32, 0, s, src, scale, add, dst);
  return MDBAS_NB_OK;
}

}  // namespace mdbas

using namespace mdbas;

extern "C" {

int mdbas_nb_ewald_rec(int nAtom, const PBC *box, double alpha, double chargeConst, int m1max,
                       int m2max, int m3max, const double *x, const double *y, const double *z,
                       const double *q, double *fx, double *fy, double *fz, double out[8],
                       int device_ptrs, void *stream) {
  if (nAtom <= 0 || !box || !x || !y || !z || !q || !fx || !fy || !fz || !out ||
      !(alpha > 0.) || m1max < 0 || m2max < 0 || m3max < 0 || !(box->vol > 0.))
    return MDBAS_NB_ERR_ARG;
  if (!device_ptrs)
    return ewald_host(nAtom, box, alpha, chargeConst, m1max, m2max, m3max, x, y, z, q, fx, fy,
                      fz, 0, out);
  std::vector<double> hq(nAtom);
  MDB_CUDA(cudaMemcpy(hq.data(), q, sizeof(double) * nAtom, cudaMemcpyDeviceToHost));
  double systq = 0., sumq2 = 0.;
  for (int i = 0; i < nAtom; ++i) {
    systq += hq[i];
    sumq2 += hq[i] * hq[i];
  }
  return ewald_run(nAtom, box, alpha, chargeConst, m1max, m2max, m3max, x, y, z, q, systq, sumq2,
                   fx, fy, fz, 0, out, static_cast<cudaStream_t>(stream));
}

// MDBas's init_ewald (src/ewald.c:10-99): tolerances, alpha, the m-range and
// mmax (the number of k-vectors).  MDBas also allocates its per-atom
// tables here; the GPU keeps its own, so nothing is allocated.
void init_ewald(CTRL *ctrl, PARAM *param, EWALD *ewald, PBC *box) {
  ewald->prec = fmin(fabs(ewald->prec), 0.5);
  ewald->tol = sqrt(fabs(log(ewald->prec * param->cutOff)));
  if (!ctrl->keyAlpha)
    ewald->alpha = sqrt(fabs(log(ewald->prec * param->cutOff * ewald->tol))) / param->cutOff;
  const double ta = 2.0 * ewald->tol * ewald->alpha;
  ewald->tol1 = sqrt(-log(ewald->prec * param->cutOff * (ta * ta)));
  if (!ctrl->keyMmax) {
    ewald->m1max = nint_h(0.25 + box->pa * ewald->alpha * ewald->tol1 / kPi);
    ewald->m2max = nint_h(0.25 + box->pb * ewald->alpha * ewald->tol1 / kPi);
    ewald->m3max = nint_h(0.25 + box->pc * ewald->alpha * ewald->tol1 / kPi);
  }
  double rc = fmin(((double)ewald->m1max * box->u), ((double)ewald->m2max * box->v));
  rc = fmin(rc, (double)ewald->m3max * box->w);
  rc = rc * 1.05 * kTwoPi;
  const double rc2 = rc * rc;
  ewald->mmax = 0;
  int m2min = 0, m3min = 1;
  for (int m1 = 0; m1 <= ewald->m1max; m1++) {
    const double rm1x = kTwoPi * box->u1 * (double)m1;
    const double rm1y = kTwoPi * box->u2 * (double)m1;
    const double rm1z = kTwoPi * box->u3 * (double)m1;
    for (int m2 = m2min; m2 <= ewald->m2max; m2++) {
      const double rm2x = rm1x + (kTwoPi * box->v1 * (double)m2);
      const double rm2y = rm1y + (kTwoPi * box->v2 * (double)m2);
      const double rm2z = rm1z + (kTwoPi * box->v3 * (double)m2);
      for (int m3 = m3min; m3 <= ewald->m3max; m3++) {
        const double rmx = rm2x + (kTwoPi * box->w1 * (double)m3);
        const double rmy = rm2y + (kTwoPi * box->w2 * (double)m3);
        const double rmz = rm2z + (kTwoPi * box->w3 * (double)m3);
        if (rmx * rmx + rmy * rmy + rmz * rmz <= rc2) ewald->mmax++;
      }
      m3min = -ewald->m3max;
    }
    m2min = -ewald->m2max;
  }
}

void ewald_free(EWALD *ewald) { (void)ewald; }

// MDBas's ewald_rec (src/ewald.c:131-354) on the GPU.  As in MDBas the whole
// force arrays are multiplied by 2 fact1 after the reciprocal forces are
// added (energy() calls it first, on zeroed arrays).
double ewald_rec(PARAM *param, EWALD *ewald, PBC *box, const double x[], const double y[],
                 const double z[], double fx[], double fy[], double fz[], const double q[],
                 double stress[6], double *virEwaldRec) {
  double out[8];
  const int st = ewald_host(param->nAtom, box, ewald->alpha, param->chargeConst, ewald->m1max,
                            ewald->m2max, ewald->m3max, x, y, z, q, fx, fy, fz, 1, out);
  if (st != MDBAS_NB_OK) {
    fprintf(stderr, "ewald_rec (GPU): %s: %s\n", mdbas_nb_status_string(st),
            mdbas_nb_last_message());
    exit(1);
  }
  for (int k = 0; k < 6; ++k) stress[k] = out[2 + k];
  *virEwaldRec = out[1];
  return out[0];
}

}  // extern "C"
