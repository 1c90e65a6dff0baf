// pair_fp32.cuh -- mixed-precision cluster-pair kernel interface.
#pragma once

#include "cluster.cuh"

namespace mdbas {

// FP32 constants of the pair kernel, folded from PairParams.
struct PairConstF {
  float rc2, ron2;
  float p_alpha;       // erfc fit p * alpha
  float c_ex;          // alpha^2 * log2(e), for exp(-(alpha r)^2) = 2^(-c_ex r^2)
  float two_a_sqrtpi;  // 2 alpha / sqrt(pi)
  float sw_a, sw_b, sw_c;  // switch: S = (rc2-r2)^2 (sw_a r2 + sw_b), dS = sw_c r2 (rc2-r2)(ron2-r2)
  // the same switch in u = r2 - ron2 (half-cluster kernel): D = rc2 - ron2,
  // sw_3d = 3 D, sw_6 = 6 / D^3, sw_m12 = -12 / D^3
  float sw_d, sw_3d, sw_6, sw_m12;
  int vdw;
};

PairConstF make_pair_const(const PairParams &p);
// Pair kernel variants: dense (all 64 pairs of an entry per warp step, scalar
// FP32), compacted (only in-cut-off pairs reach the interaction arithmetic),
// packed (the dense mapping in f32x2 arithmetic), bulk (packed, j data staged
// by bulk copies) -- these four walk the full list -- and half (two 4-atom
// j-cluster halves per warp step in f32x2 arithmetic over the inner list
// while it is current, else over the full list; the default), half3 (the
// same at up to 80 registers, three blocks of 256 threads per SM), quad
// (4 x 4 units: i-cluster halves against j-cluster halves of the inner list;
// over the full list it runs as half).
enum {
  kPairDense = 0, kPairCompact = 1, kPairPacked = 2, kPairBulk = 3, kPairHalf = 4,
  kPairHalf3 = 5, kPairQuad = 6, kPairHalfLean = 7
};
// The pair kernel over all work items (grid-stride, item count read on the
// device, so the launch needs no host synchronisation).  grid*block is the
// number of threads of the dense variant; the compacted one uses the same
// number of warps.
int pair_fp32_launch(ClusterWork &w, const PairParams &p, int grid, int block, cudaStream_t s,
                     int variant = kPairHalf);
// Ewald exclusion correction of every excluded pair (j > i), each replica's
// pairs with its own box.
int excl_fix_launch(ClusterWork &w, int n, const PairParams &p, const int *exclStart,
                    const int *exclFlat, const double *x, const double *y, const double *z,
                    const double *q, cudaStream_t s);
int forces_out_launch(ClusterWork &w, int n, int add, double *fx, double *fy, double *fz,
                      cudaStream_t s);

}  // namespace mdbas
