// kspace.cuh -- device state of the reciprocal-space sums (ewald_rec.cu,
// spme.cu), shared by the standalone calls and the engine's dynamics.
#pragma once

#include <cufft.h>

#include "common.cuh"

namespace mdbas {

// k-vector list of the explicit Ewald sum for one box / alpha / m-range.
struct EwaldKList {
  bool valid = false;
  double key[12] = {};
  int M1 = 0, M2 = 0, M3 = 0;
  int K = 0, nRows = 0;
  DBuf km, kv, vam, rows, rowK;
};

struct EwaldWork {
  EwaldKList kl;
  int device = -1;
  DBuf part, S, bpart, sums, t12, xyzq, f;
  double fact1 = 0.;  // 2 (2 pi / V) C of the last launch
};

struct SpmeWork {
  int device = -1;
  int m1 = 0, m2 = 0, m3 = 0, nbsp = 0, n = 0;
  cufftHandle plan = 0;
  bool planValid = false;
  DBuf qsp, ft, bmod, spl, cell, fr, sums, xyzq, fout;
  // deterministic spreading: atoms binned by the 8^3 grid tile of their
  // base cell, each tile's atoms in ascending index order
  DBuf tileOf, tileCount, tileStart, tileFill, tileList, tileSorted, scanTmp;
  DBuf halo;         // per tile: the (8 + p - 1)^3 halo box of its atoms' stencils
  int haloSmem = 0;  // dynamic shared memory the halo kernel is allowed
  DBuf part;         // per-block partial sums (fixed-order reductions)
  double f1 = 0.;  // (2 pi / V) C of the last launch
  ~SpmeWork() {
    if (planValid) cufftDestroy(plan);
  }
};

// Explicit Ewald reciprocal forces added to fx/fy/fz (device arrays; with
// scaleInput, MDBas's f = fact0 (f_in + sum) instead of f_in + fact0 sum);
// c.sums[0..6] = {sum_k a_k |S_k|^2, stress sums} on the device.  Once the k
// list and buffers exist for these arguments the call only launches kernels
// (it can be captured into a CUDA graph).
int ewald_launch(EwaldWork &c, int n, const PBC *box, double alpha, double chargeConst, int M1,
                 int M2, int M3, const double *x, const double *y, const double *z,
                 const double *q, double *fx, double *fy, double *fz, int scaleInput,
                 cudaStream_t s);
// SPME reciprocal forces minus their mean added to fx/fy/fz (device arrays);
// c.sums[9] = the grid energy sum, c.sums[0..5] stress sums.  Capturable
// once the plan and buffers exist for these arguments.
int spme_launch(SpmeWork &c, int n, const PBC *box, double alpha, double chargeConst, int m1,
                int m2, int m3, int nbsp, const double *x, const double *y, const double *z,
                const double *q, double *fx, double *fy, double *fz, cudaStream_t s);
// *dst = fixed point (2^-24) of scale * (*src) + add, on the device.
int kspace_fix_launch(const double *src, double scale, double add, long long *dst,
                      cudaStream_t s);

}  // namespace mdbas
