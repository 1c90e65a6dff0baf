// common.cuh -- shared device/host helpers of libmdbas_nb.so (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/mdbas_nb.h"

namespace mdbas {

// ---------------------------------------------------------------------------
// Status plumbing.  Every CUDA runtime call goes through MDB_CUDA, which turns
// a failure into MDBAS_NB_ERR_CUDA and records the CUDA message.
// ---------------------------------------------------------------------------
void set_last_status(int st, const char *msg);
int cuda_fail(cudaError_t err, const char *what, const char *file, int line);

#define MDB_CUDA(call)                                                         \
  do {                                                                         \
    cudaError_t e__ = (call);                                                  \
    if (e__ != cudaSuccess) return ::mdbas::cuda_fail(e__, #call, __FILE__, __LINE__); \
  } while (0)

#define MDB_TRY(expr)                                                          \
  do {                                                                         \
    int s__ = (expr);                                                          \
    if (s__ != MDBAS_NB_OK) return s__;                                        \
  } while (0)

// Launch bookkeeping: every kernel launch of the library goes through
// MDB_LAUNCH so the engine can report how many of its kernels ran.
extern thread_local long long *g_launch_counter;
#define MDB_LAUNCH(kernel, grid, block, smem, stream, ...)                     \
  do {                                                                         \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                \
    if (::mdbas::g_launch_counter) ++(*::mdbas::g_launch_counter);             \
    cudaError_t e__ = cudaGetLastError();                                      \
    if (e__ != cudaSuccess) return ::mdbas::cuda_fail(e__, #kernel, __FILE__, __LINE__); \
  } while (0)

// ---------------------------------------------------------------------------
// Device buffer that only grows.
// ---------------------------------------------------------------------------
struct DBuf {
  void *p = nullptr;
  size_t bytes = 0;
  int ensure(size_t n);
  void release();
  template <class T> T *as() const { return static_cast<T *>(p); }
  ~DBuf() { release(); }
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
};

// ---------------------------------------------------------------------------
// Box as the hot path reads it (MDBas PBC fields, include/global.h:175-184).
// ---------------------------------------------------------------------------
struct DevBox {
  int type;  // enum BOX_TYPE
  double a1, a2, a3, b1, b2, b3, c1, c2, c3;
  double u1, u2, u3, v1, v2, v3, w1, w2, w3;
  double pa, pb, pc, vol;
};

inline DevBox make_devbox(const PBC *b) {
  DevBox d;
  d.type = (int)b->type;
  d.a1 = b->a1; d.a2 = b->a2; d.a3 = b->a3;
  d.b1 = b->b1; d.b2 = b->b2; d.b3 = b->b3;
  d.c1 = b->c1; d.c2 = b->c2; d.c3 = b->c3;
  d.u1 = b->u1; d.u2 = b->u2; d.u3 = b->u3;
  d.v1 = b->v1; d.v2 = b->v2; d.v3 = b->v3;
  d.w1 = b->w1; d.w2 = b->w2; d.w3 = b->w3;
  d.pa = b->pa; d.pb = b->pb; d.pc = b->pc; d.vol = b->vol;
  return d;
}

// Pair-potential constants of one evaluation (MDBas PARAM/EWALD fields).
struct PairParams {
  double chargeConst, alpha;
  double cutOff2, cutOn2, switch2, rcutOff, rcutOff2, scal14;
  int vdwSwitch;   // 1 = vdw_switch, 0 = vdw_none
  int elecType;    // enum ELEC_TYPE for the cut-off Coulomb kernels
};

constexpr double kSqrtPi = 1.772453850905516;  // include/global.h:62
constexpr double kTolList = 0.01;              // include/global.h:59 TOLLIST

// ---------------------------------------------------------------------------
// FP64 helpers with MDBas's exact operation order.  __dadd_rn/__dmul_rn are
// never contracted into FMAs, so these reproduce MDBas's x86 (SSE2, no FMA)
// results bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

// nint (src/utils.c:606-609): round half away from zero, truncate to int.
__device__ __forceinline__ int nint_d(double x) {
  return (x >= 0.) ? __double2int_rz(dadd(x, 0.5)) : __double2int_rz(dsub(x, 0.5));
}

// dist (src/utils.c:38-80): minimum image in place, returns r^2.
__device__ __forceinline__ double dist_d(const DevBox &b, double &dx, double &dy, double &dz) {
  if (b.type == CUBIC) {
    dx = dsub(dx, dmul(b.a1, (double)nint_d(dmul(dx, b.u1))));
    dy = dsub(dy, dmul(b.a1, (double)nint_d(dmul(dy, b.u1))));
    dz = dsub(dz, dmul(b.a1, (double)nint_d(dmul(dz, b.u1))));
  } else if (b.type == ORBIC) {
    dx = dsub(dx, dmul(b.a1, (double)nint_d(dmul(dx, b.u1))));
    dy = dsub(dy, dmul(b.b2, (double)nint_d(dmul(dy, b.v2))));
    dz = dsub(dz, dmul(b.c3, (double)nint_d(dmul(dz, b.w3))));
  } else if (b.type == TCLIN) {
    double xt = dadd(dadd(dmul(dx, b.u1), dmul(dy, b.u2)), dmul(dz, b.u3));
    double yt = dadd(dadd(dmul(dx, b.v1), dmul(dy, b.v2)), dmul(dz, b.v3));
    double zt = dadd(dadd(dmul(dx, b.w1), dmul(dy, b.w2)), dmul(dz, b.w3));
    xt = dsub(xt, (double)nint_d(xt));
    yt = dsub(yt, (double)nint_d(yt));
    zt = dsub(zt, (double)nint_d(zt));
    dx = dadd(dadd(dmul(xt, b.a1), dmul(yt, b.b1)), dmul(zt, b.c1));
    dy = dadd(dadd(dmul(xt, b.a2), dmul(yt, b.b2)), dmul(zt, b.c2));
    dz = dadd(dadd(dmul(xt, b.a3), dmul(yt, b.b3)), dmul(zt, b.c3));
  }
  return dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
}

// image_update (src/utils.c:162-218) of one position, in place.
__device__ __forceinline__ void image_d(const DevBox &b, double &xi, double &yi, double &zi) {
  if (b.type == CUBIC) {
    xi = dsub(xi, dmul(b.a1, (double)nint_d(dmul(xi, b.u1))));
    yi = dsub(yi, dmul(b.a1, (double)nint_d(dmul(yi, b.u1))));
    zi = dsub(zi, dmul(b.a1, (double)nint_d(dmul(zi, b.u1))));
  } else if (b.type == ORBIC) {
    xi = dsub(xi, dmul(b.a1, (double)nint_d(dmul(xi, b.u1))));
    yi = dsub(yi, dmul(b.b2, (double)nint_d(dmul(yi, b.v2))));
    zi = dsub(zi, dmul(b.c3, (double)nint_d(dmul(zi, b.w3))));
  } else if (b.type == TCLIN) {
    double xt = dadd(dadd(dmul(xi, b.u1), dmul(yi, b.u2)), dmul(zi, b.u3));
    double yt = dadd(dadd(dmul(xi, b.v1), dmul(yi, b.v2)), dmul(zi, b.v3));
    double zt = dadd(dadd(dmul(xi, b.w1), dmul(yi, b.w2)), dmul(zi, b.w3));
    xt = dsub(xt, (double)nint_d(xt));
    yt = dsub(yt, (double)nint_d(yt));
    zt = dsub(zt, (double)nint_d(zt));
    xi = dadd(dadd(dmul(xt, b.a1), dmul(yt, b.b1)), dmul(zt, b.c1));
    yi = dadd(dadd(dmul(xt, b.a2), dmul(yt, b.b2)), dmul(zt, b.c2));
    zi = dadd(dadd(dmul(xt, b.a3), dmul(yt, b.b3)), dmul(zt, b.c3));
  }
}

// ---------------------------------------------------------------------------
// Fixed-point accumulation.  Forces are summed as int64 in units of 2^-32
// internal units, energies and virials in units of 2^-24.  Integer addition
// is associative, so the totals do not depend on the order in which blocks
// finish.  The largest magnitudes representable are 2^31 (forces, ~5e6
// kcal/mol/A) and 2^39 (energies, ~1.3e9 kcal/mol).
// ---------------------------------------------------------------------------
constexpr double kForceScale = 4294967296.0;    // 2^32
constexpr double kEnergyScale = 16777216.0;     // 2^24
constexpr float kForceScaleF = 4294967296.0f;
constexpr float kForceLimitF = 1.0e9f;          // |f| per conversion, < 2^31 / 2

__device__ __forceinline__ long long fix_f(float v) {
  return __float2ll_rn(v * kForceScaleF);
}
__device__ __forceinline__ long long fix_fd(double v) { return __double2ll_rn(v * kForceScale); }
__device__ __forceinline__ long long fix_e(double v) { return __double2ll_rn(v * kEnergyScale); }

__device__ __forceinline__ void red_add(long long *addr, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(addr), static_cast<unsigned long long>(v));
}
// The same reduction issued under a predicate (no branch around it).
__device__ __forceinline__ void red_add_if(bool p, long long *addr, long long v) {
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.u32 q, %2, 0;\n @q red.global.add.u64 [%0], %1;\n}"
      ::"l"(addr), "l"(v), "r"((unsigned)p)
      : "memory");
}

// Accumulator slots (int64, units 2^-24) of one evaluation.
enum AccSlot {
  ACC_E_DIR = 0, ACC_E_CORR, ACC_E_VDW, ACC_V_DIR, ACC_V_CORR, ACC_V_VDW, ACC_NPAIR,
  ACC_FLAGS,
  ACC_WORK,       // work counter of kernels that hand out items dynamically (zeroed
                  // with the accumulators before every evaluation)
  ACC_COUNT = 9
};
// Bits of the device error word (ACC_FLAGS slot).
enum DevFlag {
  FLAG_OVERFLOW = 1, FLAG_CAPACITY = 2, FLAG_NONFINITE = 4, FLAG_OUTSIDE = 8, FLAG_CELL = 16,
  FLAG_STAGE = 32  // a bulk copy into shared memory did not complete in time
};

__device__ __forceinline__ void raise_flag(long long *acc, int bit) {
  atomicOr(reinterpret_cast<unsigned long long *>(acc + ACC_FLAGS), (unsigned long long)bit);
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Device-wide exclusive scan of int32 counts into int64 offsets; total (the
// sum) is written to out[n].  tmp must hold scan_tmp_bytes(n).
size_t scan_tmp_bytes(int n);
int exclusive_scan(const int *in, long long *out, int n, void *tmp, cudaStream_t s);
// Same for int32 -> int32 (sizes known to fit).
int exclusive_scan32(const int *in, int *out, int n, void *tmp, cudaStream_t s);

inline int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 0x7fffffffLL) g = 0x7fffffff;
  return (int)g;
}

}  // namespace mdbas
