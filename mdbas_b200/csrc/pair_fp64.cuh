// pair_fp64.cuh -- plain FP64 pair kernels (MDBas's loops, one thread per i).
#pragma once

#include "common.cuh"

namespace mdbas {

// Accumulator layout (FP64, device): 0 elec, 1 vdw, 2 virelec, 3 virvdw,
// 4 in-cut-off pairs, 5 eCorr, 6 virCorr, 7 sum q^2.
constexpr int kFp64AccCount = 8;

int pairs_fp64(int ewald, int n, const DevBox &b, const PairParams &p, const int *order,
               const int *neighPair, const long long *off, const int *list, const double *x,
               const double *y, const double *z, const double *q, const double *eps,
               const double *sig, double *fx, double *fy, double *fz, double *acc,
               cudaStream_t s);
int excl_fp64(int n, const DevBox &b, const PairParams &p, const int *exclStart,
              const int *exclFlat, const double *x, const double *y, const double *z,
              const double *q, double *fx, double *fy, double *fz, double *acc, cudaStream_t s);
// sum of q^2 in units of 2^-40 (int64, order independent) added to *acc.
int sum_q2(int n, const double *q, long long *acc, cudaStream_t s);
constexpr double kQ2Scale = 1099511627776.0;  // 2^40
// 1-4 pairs (MDBas neighList14 layout: i0 j0 i1 j1 ...); acc[0..3] += elec,
// vdw, virelec, virvdw.
int pairs14_fp64(int ewald, int npair, const DevBox &b, const PairParams &p, const int *list14,
                 const double *x, const double *y, const double *z, const double *q,
                 const double *eps, const double *sig, double *fx, double *fy, double *fz,
                 double *acc, cudaStream_t s);

}  // namespace mdbas
