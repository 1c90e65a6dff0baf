// pair_fp32.cu -- mixed-precision cluster-pair kernel (FP32 pair arithmetic,
// 64-bit fixed-point accumulation) and its FP64 companions.
//
// Mapping.  One warp runs one work item: an i cluster (8 atoms) against up
// to 32 j clusters.  Lane L owns i atom L%8 and j atoms L/8 and L/8+4 of each
// j cluster, i.e. exactly bits L and 32+L of the entry's 64-bit interaction
// mask.  Per j cluster the warp computes all 64 pairs with MDBas's formulas
// (Ewald direct term, src/ewald.c:356-369; vdw_switch, src/vdw.c:144-184):
//   - displacement: FP32 j-relative coordinates + the entry's FP32 shift
//     (origin-to-origin vector formed in FP64) - FP32 i-relative coordinates;
//   - erfc(x) = t P(t) exp(-x^2), t = 1/(1+px), P of degree 7 (own refit of
//     the Abramowitz-Stegun 7.1.26 form, fit_erfc.py, max relative error
//     2.4e-8 on [0, 6]); hardware rsqrt/rcp/ex2 (3 MUFU per pair);
// the j forces are reduced across the 8 i lanes with a 3-step shuffle
// reduce-scatter (6 shuffles for 6 values) and each j atom component is added
// once per cluster pair (Newton's third law) as a 64-bit fixed-point
// integer; i forces stay in registers for the whole item.  Energies and
// virials are summed in FP32 per lane within an item and converted to fixed
// point once per item.  Every quantity that reaches an accumulator is a
// fixed-point integer computed from one cluster pair, one item or one
// excluded pair, so the totals do not depend on the order in which warps or
// blocks run, nor on the order in which the list builder emitted items.
#include "cluster.cuh"
#include "pair_fp32.cuh"

namespace mdbas {

namespace {

// erfc fit constants (fit_erfc.py)
constexpr float kErfcP = 3.225531683e-01f;
constexpr float kErfcC0 = 1.826605733e-01f;
constexpr float kErfcC1 = 1.717395874e-01f;
constexpr float kErfcC2 = 2.389294945e-01f;
constexpr float kErfcC3 = -8.776152576e-02f;
constexpr float kErfcC4 = 6.608865734e-01f;
constexpr float kErfcC5 = -6.320509922e-01f;
constexpr float kErfcC6 = 6.305108379e-01f;
constexpr float kErfcC7 = -1.649145727e-01f;

__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// One pair.  d = x_j - x_i.  Returns whether it interacted; adds energy and
// virial terms; f = (dE/dr)/r * d is the force on i (minus the force on j).
template <bool VDW>
__device__ __forceinline__ bool interact(const PairConstF &c, const float4 xj, const float2 lj,
                                         const float sx, const float sy, const float sz,
                                         const float qi, const float2 li, const bool bit,
                                         float &fx, float &fy, float &fz, float &ec, float &ev,
                                         float &vc, float &vv) {
  const float dx = xj.x + sx, dy = xj.y + sy, dz = xj.z + sz;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const bool in = bit && (r2 <= c.rc2);
  const float r2s = in ? r2 : 1.0f;
  const float rinv = rsqrt_approx(r2s);
  const float r = r2s * rinv;
  const float qq = in ? qi * xj.w : 0.f;
  const float t = rcp_approx(fmaf(c.p_alpha, r, 1.0f));
  const float ex = ex2_approx(-c.c_ex * r2s);
  float poly = fmaf(kErfcC7, t, kErfcC6);
  poly = fmaf(poly, t, kErfcC5);
  poly = fmaf(poly, t, kErfcC4);
  poly = fmaf(poly, t, kErfcC3);
  poly = fmaf(poly, t, kErfcC2);
  poly = fmaf(poly, t, kErfcC1);
  poly = fmaf(poly, t, kErfcC0);
  const float qr = qq * rinv;
  const float e_c = qr * (t * poly * ex);
  const float de_c = -fmaf(qq * c.two_a_sqrtpi, ex, e_c) * rinv;
  ec += e_c;
  vc = fmaf(de_c, r, vc);
  float F = de_c;
  if (VDW) {
    const float eps = in ? li.x * lj.x : 0.f;  // 4 eps_i eps_j
    const float sg = (li.y + lj.y) * rinv;
    const float s2 = sg * sg;
    const float s6 = s2 * s2 * s2;
    const float s12 = s6 * s6;
    const float pv = eps * (s12 - s6);
    const float dpv = eps * fmaf(-12.f, s12, 6.f * s6);  // r dE/dr
    const bool sw = r2s > c.ron2;
    const float s1 = c.rc2 - r2s;
    const float S = sw ? s1 * s1 * fmaf(c.sw_a, r2s, c.sw_b) : 1.f;
    const float dS = sw ? c.sw_c * r2s * s1 * (c.ron2 - r2s) : 0.f;
    const float de_v = fmaf(pv, dS, dpv * S) * rinv;
    ev = fmaf(pv, S, ev);
    vv = fmaf(de_v, r, vv);
    F += de_v;
  }
  F *= rinv;
  fx = F * dx;
  fy = F * dy;
  fz = F * dz;
  return in;
}

template <bool VDW>
__global__ void __launch_bounds__(256)
k_pair_fp32(const long long *__restrict__ counters, const int4 *__restrict__ items,
            const CPairEntry *__restrict__ entries, const uint2 *__restrict__ masks,
            const float4 *__restrict__ xq, const float2 *__restrict__ lj, PairConstF c,
            long long *__restrict__ facc, int fstride, long long *__restrict__ acc) {
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, jh = lane >> 3;
  const bool up = il & 4, mid = il & 2, lo = il & 1;
  const int comp = mid ? (lo ? 3 : 2) : (lo ? 1 : 0);
  const long long nItems = counters[1];
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long *fcomp = facc + (size_t)(comp < 3 ? comp : 0) * fstride;
  long long Ec = 0, Ev = 0, Vc = 0, Vv = 0;  // fixed point, summed per item
  long long npair = 0;
  bool overflow = false;

  for (long long it = gw; it < nItems; it += nw) {
    const int4 item = items[it];
    const int ci = item.x, e0 = item.y, ne = item.z;
    const float4 xi = xq[ci * kClusterSize + il];
    const float2 li = lj[ci * kClusterSize + il];
    float fix = 0.f, fiy = 0.f, fiz = 0.f;
    float ec = 0.f, ev = 0.f, vc = 0.f, vv = 0.f;
    for (int e = e0; e < e0 + ne; ++e) {
      const CPairEntry en = entries[e];
      const uint2 mk = masks[e];
      const float sx = en.sx - xi.x, sy = en.sy - xi.y, sz = en.sz - xi.z;
      const int jb = en.j * kClusterSize + jh;
      const float4 xa = xq[jb];
      const float2 la = lj[jb];
      const float4 xb = xq[jb + 4];
      const float2 lb = lj[jb + 4];
      float ax, ay, az, bx, by, bz;
      const bool ina = interact<VDW>(c, xa, la, sx, sy, sz, xi.w, li, (mk.x >> lane) & 1u, ax,
                                     ay, az, ec, ev, vc, vv);
      const bool inb = interact<VDW>(c, xb, lb, sx, sy, sz, xi.w, li, (mk.y >> lane) & 1u, bx,
                                     by, bz, ec, ev, vc, vv);
      fix += ax + bx;
      fiy += ay + by;
      fiz += az + bz;
      const unsigned ba = __ballot_sync(0xffffffffu, ina);
      const unsigned bb = __ballot_sync(0xffffffffu, inb);
      if ((ba | bb) == 0u) continue;
      npair += __popc(ba) + __popc(bb);
      // reduce-scatter of the two j atoms' forces over the 8 i lanes
      float k0 = up ? bx : ax, k1 = up ? by : ay, k2 = up ? bz : az;
      const float s0 = up ? ax : bx, s1 = up ? ay : by, s2 = up ? az : bz;
      k0 += __shfl_xor_sync(0xffffffffu, s0, 4);
      k1 += __shfl_xor_sync(0xffffffffu, s1, 4);
      k2 += __shfl_xor_sync(0xffffffffu, s2, 4);
      const float t0 = mid ? k0 : k2, t1 = mid ? k1 : 0.f;
      float u0 = mid ? k2 : k0, u1 = mid ? 0.f : k1;
      u0 += __shfl_xor_sync(0xffffffffu, t0, 2);
      u1 += __shfl_xor_sync(0xffffffffu, t1, 2);
      const float w = lo ? u0 : u1;
      float v = lo ? u1 : u0;
      v += __shfl_xor_sync(0xffffffffu, w, 1);
      if (comp < 3 && v != 0.f) {
        overflow |= !(fabsf(v) < kForceLimitF);
        red_add(fcomp + en.j * kClusterSize + (up ? jh + 4 : jh), fix_f(-v));
      }
    }
    // i forces: sum over the four j lanes of each i atom
    fix += __shfl_xor_sync(0xffffffffu, fix, 8);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 8);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 8);
    fix += __shfl_xor_sync(0xffffffffu, fix, 16);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 16);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 16);
    if (jh < 3) {
      const float v = (jh == 0) ? fix : (jh == 1 ? fiy : fiz);
      if (v != 0.f) {
        overflow |= !(fabsf(v) < kForceLimitF);
        red_add(facc + (size_t)jh * fstride + ci * kClusterSize + il, fix_f(v));
      }
    }
    // Each item's energy is converted to fixed point on its own, so totals
    // do not depend on which warp ran which item.
    Ec += fix_e(warp_sum_d((double)ec));
    Ev += fix_e(warp_sum_d((double)ev));
    Vc += fix_e(warp_sum_d((double)vc));
    Vv += fix_e(warp_sum_d((double)vv));
  }
  if (__any_sync(0xffffffffu, overflow) && lane == 0) raise_flag(acc, FLAG_OVERFLOW);
  if (lane == 0) {
    red_add(acc + ACC_E_DIR, Ec);
    red_add(acc + ACC_E_VDW, Ev);
    red_add(acc + ACC_V_DIR, Vc);
    red_add(acc + ACC_V_VDW, Vv);
    red_add(acc + ACC_NPAIR, npair);
  }
}


// ---------------------------------------------------------------------------
// Packed variant (default).  The same mapping and results as k_pair_fp32, with
// a lane's two pairs (j atoms h and h+4) evaluated together in f32x2
// arithmetic (__ffma2_rn / __fmul2_rn / __fadd2_rn, one instruction for both
// pairs on sm_100): the kernel is issue-bound, and this halves the issue
// slots of its FP32 arithmetic.  The j data come from the pair-interleaved
// copies xp/ljp, so each operand pair already sits in a register pair.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// The lane's two displacements and squared distances; ina / inb: listed and
// inside the cut-off.
__device__ __forceinline__ void distance2(const PairConstF &c, const float2 jx, const float2 jy,
                                          const float2 jz, const float sx, const float sy,
                                          const float sz, const bool bita, const bool bitb,
                                          float2 &dx, float2 &dy, float2 &dz, float2 &r2,
                                          bool &ina, bool &inb) {
  dx = __fadd2_rn(jx, f2(sx));
  dy = __fadd2_rn(jy, f2(sy));
  dz = __fadd2_rn(jz, f2(sz));
  r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
  ina = bita && (r2.x <= c.rc2);
  inb = bitb && (r2.y <= c.rc2);
}

// Energies, virials and forces of the lane's two pairs (pairs outside the
// cut-off or the list contribute exact zeros).
template <bool VDW>
__device__ __forceinline__ void interact2(const PairConstF &c, const float2 dx, const float2 dy,
                                          const float2 dz, const float2 r2, const float2 jq,
                                          const float2 jeps, const float2 jsig, const float qi,
                                          const float2 li, const bool ina, const bool inb,
                                          float2 &fx, float2 &fy, float2 &fz, float2 &ec,
                                          float2 &ev, float2 &vc, float2 &vv) {
  const float2 r2s = make_float2(ina ? r2.x : 1.0f, inb ? r2.y : 1.0f);
  const float2 m = make_float2(ina ? 1.0f : 0.f, inb ? 1.0f : 0.f);
  const float2 rinv = make_float2(rsqrt_approx(r2s.x), rsqrt_approx(r2s.y));
  const float2 nrinv = __fmul2_rn(rinv, f2(-1.0f));
  const float2 r = __fmul2_rn(r2s, rinv);
  const float2 qq = __fmul2_rn(__fmul2_rn(f2(qi), jq), m);
  const float2 targ = __ffma2_rn(f2(c.p_alpha), r, f2(1.0f));
  const float2 t = make_float2(rcp_approx(targ.x), rcp_approx(targ.y));
  const float2 earg = __fmul2_rn(f2(-c.c_ex), r2s);
  const float2 ex = make_float2(ex2_approx(earg.x), ex2_approx(earg.y));
  float2 poly = __ffma2_rn(f2(kErfcC7), t, f2(kErfcC6));
  poly = __ffma2_rn(poly, t, f2(kErfcC5));
  poly = __ffma2_rn(poly, t, f2(kErfcC4));
  poly = __ffma2_rn(poly, t, f2(kErfcC3));
  poly = __ffma2_rn(poly, t, f2(kErfcC2));
  poly = __ffma2_rn(poly, t, f2(kErfcC1));
  poly = __ffma2_rn(poly, t, f2(kErfcC0));
  const float2 qr = __fmul2_rn(qq, rinv);
  const float2 e_c = __fmul2_rn(qr, __fmul2_rn(__fmul2_rn(t, poly), ex));
  const float2 de_c =
      __fmul2_rn(__ffma2_rn(__fmul2_rn(qq, f2(c.two_a_sqrtpi)), ex, e_c), nrinv);
  ec = __fadd2_rn(ec, e_c);
  vc = __ffma2_rn(de_c, r, vc);
  float2 F = de_c;
  if (VDW) {
    const float2 eps = __fmul2_rn(__fmul2_rn(f2(li.x), jeps), m);  // 4 eps_i eps_j
    const float2 sg = __fmul2_rn(__fadd2_rn(f2(li.y), jsig), rinv);
    const float2 s2 = __fmul2_rn(sg, sg);
    const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
    const float2 s12 = __fmul2_rn(s6, s6);
    const float2 pv = __fmul2_rn(eps, __ffma2_rn(s6, f2(-1.0f), s12));
    const float2 dpv = __fmul2_rn(eps, __ffma2_rn(f2(-12.f), s12, __fmul2_rn(f2(6.f), s6)));
    const float2 s1 = __ffma2_rn(r2s, f2(-1.0f), f2(c.rc2));
    const float2 Sv = __fmul2_rn(__fmul2_rn(s1, s1), __ffma2_rn(f2(c.sw_a), r2s, f2(c.sw_b)));
    const float2 dSv = __fmul2_rn(__fmul2_rn(__fmul2_rn(f2(c.sw_c), r2s), s1),
                                  __ffma2_rn(r2s, f2(-1.0f), f2(c.ron2)));
    const bool swa = r2s.x > c.ron2, swb = r2s.y > c.ron2;
    const float2 S = make_float2(swa ? Sv.x : 1.f, swb ? Sv.y : 1.f);
    const float2 dS = make_float2(swa ? dSv.x : 0.f, swb ? dSv.y : 0.f);
    const float2 de_v = __fmul2_rn(__ffma2_rn(pv, dS, __fmul2_rn(dpv, S)), rinv);
    ev = __ffma2_rn(pv, S, ev);
    vv = __ffma2_rn(de_v, r, vv);
    F = __fadd2_rn(F, de_v);
  }
  F = __fmul2_rn(F, rinv);
  fx = __fmul2_rn(F, dx);
  fy = __fmul2_rn(F, dy);
  fz = __fmul2_rn(F, dz);
}

// Per-warp staging area of the packed kernel: up to kStage entries of an item
// with their j clusters' pair-interleaved data, loaded in one batch so that
// all of a chunk's global loads are in flight together.
constexpr int kStage = 8;
struct StageWarp {
  float4 en[kStage];            // j (as int bits), shift x, y, z
  uint2 mk[kStage];             // interaction masks
  float4 jd[kStage * 12];       // per entry and h: xp pair 0, xp pair 1, ljp
};

// (at most 80 registers: three blocks of 256 threads per SM)
template <bool VDW>
__global__ void __launch_bounds__(256, 3)
k_pair_fp32x2(const long long *__restrict__ counters, const int4 *__restrict__ items,
              const CPairEntry *__restrict__ entries, const uint2 *__restrict__ masks,
              const float4 *__restrict__ xq, const float2 *__restrict__ lj,
              const float4 *__restrict__ xp, const float4 *__restrict__ ljp, PairConstF c,
              long long *__restrict__ facc, int fstride, long long *__restrict__ acc) {
  __shared__ StageWarp stage[8];
  StageWarp &S = stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, jh = lane >> 3;
  const bool up = il & 4, mid = il & 2, lo = il & 1;
  const int comp = mid ? (lo ? 3 : 2) : (lo ? 1 : 0);
  const long long nItems = counters[1];
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long *fcomp = facc + (size_t)(comp < 3 ? comp : 0) * fstride;
  long long Ec = 0, Ev = 0, Vc = 0, Vv = 0;  // fixed point, summed per item
  long long npair = 0;
  bool overflow = false;

  for (long long it = gw; it < nItems; it += nw) {
    const int4 item = items[it];
    const int ci = item.x, e0 = item.y, ne = item.z;
    const float4 xi = xq[ci * kClusterSize + il];
    const float2 li = lj[ci * kClusterSize + il];
    float2 fi_x = f2(0.f), fi_y = f2(0.f), fi_z = f2(0.f);
    float2 ec = f2(0.f), ev = f2(0.f), vc = f2(0.f), vv = f2(0.f);
    for (int c0 = 0; c0 < ne; c0 += kStage) {
      const int nc = min(kStage, ne - c0);
      // stage: entries and masks (lanes 0..nc-1), then each lane three of
      // the chunk's 12*nc float4 of j data
      CPairEntry my{};
      if (lane < nc) {
        my = entries[e0 + c0 + lane];
        S.en[lane] = make_float4(__int_as_float(my.j), my.sx, my.sy, my.sz);
        S.mk[lane] = masks[e0 + c0 + lane];
      }
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const int idx = lane + 32 * r;             // < 96
        const int k = idx / 12, q = idx - 12 * k;  // entry, (h, part)
        const int jk = __shfl_sync(0xffffffffu, my.j, k & 7);
        if (k < nc) {
          const int h = q / 3, part = q - 3 * h;
          const size_t jp = (size_t)jk * 4 + h;
          S.jd[idx] = part < 2 ? xp[2 * jp + part] : ljp[jp];
        }
      }
      __syncwarp();
      for (int k = 0; k < nc; ++k) {
        const float4 en = S.en[k];
        const uint2 mk = S.mk[k];
        const int j = __float_as_int(en.x);
        const float sx = en.y - xi.x, sy = en.z - xi.y, sz = en.w - xi.z;
        const float4 p0 = S.jd[k * 12 + jh * 3], p1 = S.jd[k * 12 + jh * 3 + 1],
                     lp = S.jd[k * 12 + jh * 3 + 2];
        float2 dx, dy, dz, r2;
        bool ina, inb;
        distance2(c, make_float2(p0.x, p0.y), make_float2(p0.z, p0.w), make_float2(p1.x, p1.y),
                  sx, sy, sz, (mk.x >> lane) & 1u, (mk.y >> lane) & 1u, dx, dy, dz, r2, ina,
                  inb);
        const unsigned ba = __ballot_sync(0xffffffffu, ina);
        const unsigned bb = __ballot_sync(0xffffffffu, inb);
        // a cluster pair listed at the list radius with no pair inside the
        // cut-off now contributes nothing: skip it (exact zeros otherwise)
        if ((ba | bb) == 0u) continue;
        float2 fx, fy, fz;
        interact2<VDW>(c, dx, dy, dz, r2, make_float2(p1.z, p1.w), make_float2(lp.x, lp.y),
                       make_float2(lp.z, lp.w), xi.w, li, ina, inb, fx, fy, fz, ec, ev, vc, vv);
        fi_x = __fadd2_rn(fi_x, fx);
        fi_y = __fadd2_rn(fi_y, fy);
        fi_z = __fadd2_rn(fi_z, fz);
        npair += __popc(ba) + __popc(bb);
        // reduce-scatter of the two j atoms' forces over the 8 i lanes
        const float ax = fx.x, ay = fy.x, az = fz.x, bx = fx.y, by = fy.y, bz = fz.y;
        float k0 = up ? bx : ax, k1 = up ? by : ay, k2 = up ? bz : az;
        const float s0 = up ? ax : bx, s1 = up ? ay : by, s2 = up ? az : bz;
        k0 += __shfl_xor_sync(0xffffffffu, s0, 4);
        k1 += __shfl_xor_sync(0xffffffffu, s1, 4);
        k2 += __shfl_xor_sync(0xffffffffu, s2, 4);
        const float t0 = mid ? k0 : k2, t1 = mid ? k1 : 0.f;
        float u0 = mid ? k2 : k0, u1 = mid ? 0.f : k1;
        u0 += __shfl_xor_sync(0xffffffffu, t0, 2);
        u1 += __shfl_xor_sync(0xffffffffu, t1, 2);
        const float w = lo ? u0 : u1;
        float v = lo ? u1 : u0;
        v += __shfl_xor_sync(0xffffffffu, w, 1);
        if (comp < 3 && v != 0.f) {
          overflow |= !(fabsf(v) < kForceLimitF);
          red_add(fcomp + j * kClusterSize + (up ? jh + 4 : jh), fix_f(-v));
        }
      }
      __syncwarp();
    }
    // i forces: the lane's two pairs, then the four j lanes of each i atom
    float fix = fi_x.x + fi_x.y, fiy = fi_y.x + fi_y.y, fiz = fi_z.x + fi_z.y;
    fix += __shfl_xor_sync(0xffffffffu, fix, 8);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 8);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 8);
    fix += __shfl_xor_sync(0xffffffffu, fix, 16);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 16);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 16);
    if (jh < 3) {
      const float v = (jh == 0) ? fix : (jh == 1 ? fiy : fiz);
      if (v != 0.f) {
        overflow |= !(fabsf(v) < kForceLimitF);
        red_add(facc + (size_t)jh * fstride + ci * kClusterSize + il, fix_f(v));
      }
    }
    // Each item's energy is converted to fixed point on its own, so totals
    // do not depend on which warp ran which item.
    Ec += fix_e(warp_sum_d((double)ec.x + (double)ec.y));
    Ev += fix_e(warp_sum_d((double)ev.x + (double)ev.y));
    Vc += fix_e(warp_sum_d((double)vc.x + (double)vc.y));
    Vv += fix_e(warp_sum_d((double)vv.x + (double)vv.y));
  }
  if (__any_sync(0xffffffffu, overflow) && lane == 0) raise_flag(acc, FLAG_OVERFLOW);
  if (lane == 0) {
    red_add(acc + ACC_E_DIR, Ec);
    red_add(acc + ACC_E_VDW, Ev);
    red_add(acc + ACC_V_DIR, Vc);
    red_add(acc + ACC_V_VDW, Vv);
    red_add(acc + ACC_NPAIR, npair);
  }
}

// ---------------------------------------------------------------------------
// Bulk-staged variant (kPairBulk).  The packed kernel's arithmetic and
// results, with each chunk's j data brought into shared memory by
// asynchronous bulk copies (cp.async.bulk, completion counted by an mbarrier)
// instead of per-lane loads: a j cluster's pair-interleaved copies are two
// contiguous blocks (xp: 128 B, ljp: 64 B), one copy each.  Two buffers per
// warp: while a chunk is computed the next chunk's copies are in flight and
// the entries of the one after are being loaded.  Waits are bounded: a copy
// that does not complete sets FLAG_STAGE and the warp stops.  Once FLAG_STAGE
// is raised every force, energy and virial of that evaluation is invalid (a
// late copy may still land in shared memory the next block on the SM uses):
// the engine's result calls (get_forces, energies) and the dynamics return
// MDBAS_NB_ERR_CUDA for it instead of any result.
// ---------------------------------------------------------------------------
struct BulkBuf {
  float4 en[kStage];       // j (as int bits), shift x, y, z
  uint2 mk[kStage];        // interaction masks
  float4 jd[kStage * 12];  // per entry: xp (8 float4: h, pair part) then ljp (4 float4: h)
};
struct BulkWarp {
  BulkBuf buf[2];
  unsigned long long bar[2];
};
constexpr unsigned kBulkBytes = 12 * 16;     // bytes copied per entry
constexpr int kBulkWaitLimit = 1 << 20;      // try_wait rounds before giving up

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  unsigned long long state;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
               : "=l"(state)
               : "r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile("" ::"l"(state));
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_to_smem(void *dst, const void *src, unsigned bytes,
                                             unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Every lane waits for the buffer's phase (bounded, so each lane's later
// reads see the copied data); true when all lanes saw it complete.
__device__ __forceinline__ bool bulk_wait(unsigned long long *bar, unsigned parity) {
  bool ok = false;
  for (int r = 0; r < kBulkWaitLimit && !ok; ++r) ok = mbar_try_wait(bar, parity);
  return __all_sync(0xffffffffu, ok);
}

// Stage one chunk: entries and masks by the lanes that hold them, then the
// copies of the j data (the buffer's previous contents were read two chunks
// ago, before a __syncwarp).
__device__ __forceinline__ void bulk_issue(BulkBuf &B, unsigned long long *bar, int nc, int lane,
                                           const CPairEntry &en, const uint2 &mk,
                                           const float4 *__restrict__ xp,
                                           const float4 *__restrict__ ljp) {
  fence_proxy_async_smem();
  if (lane < nc) {
    B.en[lane] = make_float4(__int_as_float(en.j), en.sx, en.sy, en.sz);
    B.mk[lane] = mk;
  }
  if (lane == 0) mbar_expect_tx(bar, (unsigned)nc * kBulkBytes);
  __syncwarp();
  if (lane < nc) {
    bulk_to_smem(&B.jd[lane * 12], xp + (size_t)en.j * 8, 128, bar);
    bulk_to_smem(&B.jd[lane * 12 + 8], ljp + (size_t)en.j * 4, 64, bar);
  }
}

template <bool VDW>
__global__ void __launch_bounds__(256, 3)
k_pair_fp32x2_bulk(const long long *__restrict__ counters, const int4 *__restrict__ items,
                   const CPairEntry *__restrict__ entries, const uint2 *__restrict__ masks,
                   const float4 *__restrict__ xq, const float2 *__restrict__ lj,
                   const float4 *__restrict__ xp, const float4 *__restrict__ ljp, PairConstF c,
                   long long *__restrict__ facc, int fstride, long long *__restrict__ acc) {
  __shared__ __align__(16) BulkWarp bw[8];
  BulkWarp &W = bw[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, jh = lane >> 3;
  const bool up = il & 4, mid = il & 2, lo = il & 1;
  const int comp = mid ? (lo ? 3 : 2) : (lo ? 1 : 0);
  const long long nItems = counters[1];
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long *fcomp = facc + (size_t)(comp < 3 ? comp : 0) * fstride;
  long long Ec = 0, Ev = 0, Vc = 0, Vv = 0;
  long long npair = 0;
  bool overflow = false;
  if (lane == 0) {
    mbar_init(&W.bar[0]);
    mbar_init(&W.bar[1]);
    fence_mbar_init();
    fence_proxy_async_smem();
  }
  __syncwarp();
  unsigned ph0 = 0, ph1 = 0;  // parity of each buffer's next phase
  int b = 0;                  // buffer of the chunk being computed

  for (long long it = gw; it < nItems; it += nw) {
    const int4 item = items[it];
    const int ci = item.x, e0 = item.y, ne = item.z;
    // an empty item stages nothing (an arrival with no copies would complete
    // a buffer phase that no wait consumes)
    if (ne == 0) continue;
    const float4 xi = xq[ci * kClusterSize + il];
    const float2 li = lj[ci * kClusterSize + il];
    float2 fi_x = f2(0.f), fi_y = f2(0.f), fi_z = f2(0.f);
    float2 ec = f2(0.f), ev = f2(0.f), vc = f2(0.f), vv = f2(0.f);
    const int nch = (ne + kStage - 1) / kStage;
    // chunk 0 now; the entries of chunk 1 into registers
    CPairEntry nen{};
    uint2 nmk = make_uint2(0u, 0u);
    {
      const int nc = min(kStage, ne);
      if (lane < nc) {
        nen = entries[e0 + lane];
        nmk = masks[e0 + lane];
      }
      bulk_issue(W.buf[b], &W.bar[b], nc, lane, nen, nmk, xp, ljp);
    }
    if (nch > 1) {
      const int nc = min(kStage, ne - kStage);
      if (lane < nc) {
        nen = entries[e0 + kStage + lane];
        nmk = masks[e0 + kStage + lane];
      }
    }
    for (int ch = 0; ch < nch; ++ch) {
      if (ch + 1 < nch) {
        const int nc1 = min(kStage, ne - (ch + 1) * kStage);
        bulk_issue(W.buf[b ^ 1], &W.bar[b ^ 1], nc1, lane, nen, nmk, xp, ljp);
        if (ch + 2 < nch) {
          const int nc2 = min(kStage, ne - (ch + 2) * kStage);
          if (lane < nc2) {
            nen = entries[e0 + (ch + 2) * kStage + lane];
            nmk = masks[e0 + (ch + 2) * kStage + lane];
          }
        }
      }
      const unsigned par = b ? ph1 : ph0;
      if (!bulk_wait(&W.bar[b], par)) {
        // a copy did not complete: report, give the other buffer's copies
        // (if any) a bounded time, and stop this warp
        if (lane == 0) raise_flag(acc, FLAG_STAGE);
        if (ch + 1 < nch) bulk_wait(&W.bar[b ^ 1], b ? ph0 : ph1);
        return;
      }
      if (b) ph1 ^= 1u; else ph0 ^= 1u;
      const BulkBuf &S = W.buf[b];
      const int nc = min(kStage, ne - ch * kStage);
      for (int k = 0; k < nc; ++k) {
        const float4 en = S.en[k];
        const uint2 mk = S.mk[k];
        const int j = __float_as_int(en.x);
        const float sx = en.y - xi.x, sy = en.z - xi.y, sz = en.w - xi.z;
        const float4 p0 = S.jd[k * 12 + jh * 2], p1 = S.jd[k * 12 + jh * 2 + 1],
                     lp = S.jd[k * 12 + 8 + jh];
        float2 dx, dy, dz, r2;
        bool ina, inb;
        distance2(c, make_float2(p0.x, p0.y), make_float2(p0.z, p0.w), make_float2(p1.x, p1.y),
                  sx, sy, sz, (mk.x >> lane) & 1u, (mk.y >> lane) & 1u, dx, dy, dz, r2, ina,
                  inb);
        const unsigned ba = __ballot_sync(0xffffffffu, ina);
        const unsigned bb = __ballot_sync(0xffffffffu, inb);
        if ((ba | bb) == 0u) continue;
        float2 fx, fy, fz;
        interact2<VDW>(c, dx, dy, dz, r2, make_float2(p1.z, p1.w), make_float2(lp.x, lp.y),
                       make_float2(lp.z, lp.w), xi.w, li, ina, inb, fx, fy, fz, ec, ev, vc, vv);
        fi_x = __fadd2_rn(fi_x, fx);
        fi_y = __fadd2_rn(fi_y, fy);
        fi_z = __fadd2_rn(fi_z, fz);
        npair += __popc(ba) + __popc(bb);
        const float ax = fx.x, ay = fy.x, az = fz.x, bx = fx.y, by = fy.y, bz = fz.y;
        float k0 = up ? bx : ax, k1 = up ? by : ay, k2 = up ? bz : az;
        const float s0 = up ? ax : bx, s1 = up ? ay : by, s2 = up ? az : bz;
        k0 += __shfl_xor_sync(0xffffffffu, s0, 4);
        k1 += __shfl_xor_sync(0xffffffffu, s1, 4);
        k2 += __shfl_xor_sync(0xffffffffu, s2, 4);
        const float t0 = mid ? k0 : k2, t1 = mid ? k1 : 0.f;
        float u0 = mid ? k2 : k0, u1 = mid ? 0.f : k1;
        u0 += __shfl_xor_sync(0xffffffffu, t0, 2);
        u1 += __shfl_xor_sync(0xffffffffu, t1, 2);
        const float w = lo ? u0 : u1;
        float v = lo ? u1 : u0;
        v += __shfl_xor_sync(0xffffffffu, w, 1);
        if (comp < 3 && v != 0.f) {
          overflow |= !(fabsf(v) < kForceLimitF);
          red_add(fcomp + j * kClusterSize + (up ? jh + 4 : jh), fix_f(-v));
        }
      }
      __syncwarp();
      b ^= 1;
    }
    float fix = fi_x.x + fi_x.y, fiy = fi_y.x + fi_y.y, fiz = fi_z.x + fi_z.y;
    fix += __shfl_xor_sync(0xffffffffu, fix, 8);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 8);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 8);
    fix += __shfl_xor_sync(0xffffffffu, fix, 16);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 16);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 16);
    if (jh < 3) {
      const float v = (jh == 0) ? fix : (jh == 1 ? fiy : fiz);
      if (v != 0.f) {
        overflow |= !(fabsf(v) < kForceLimitF);
        red_add(facc + (size_t)jh * fstride + ci * kClusterSize + il, fix_f(v));
      }
    }
    Ec += fix_e(warp_sum_d((double)ec.x + (double)ec.y));
    Ev += fix_e(warp_sum_d((double)ev.x + (double)ev.y));
    Vc += fix_e(warp_sum_d((double)vc.x + (double)vc.y));
    Vv += fix_e(warp_sum_d((double)vv.x + (double)vv.y));
  }
  if (__any_sync(0xffffffffu, overflow) && lane == 0) raise_flag(acc, FLAG_OVERFLOW);
  if (lane == 0) {
    red_add(acc + ACC_E_DIR, Ec);
    red_add(acc + ACC_E_VDW, Ev);
    red_add(acc + ACC_V_DIR, Vc);
    red_add(acc + ACC_V_VDW, Vv);
    red_add(acc + ACC_NPAIR, npair);
  }
}

// ---------------------------------------------------------------------------
// Compacted variant.  Same work items, entries and results as k_pair_fp32,
// but only in-cut-off pairs reach the expensive arithmetic:
//   staging: a chunk of 8 entries and their 64 j atoms are loaded into shared
//     memory in one batch, so all global loads of a chunk are in flight
//     together;
//   filter: per entry the warp tests its 64 pairs (r^2 <= rc^2 and the mask
//     bit) and appends the survivors to per-i-atom queues in shared memory
//     (ballot + prefix count inside each group of 4 lanes that share an i
//     atom), LJ pairs (both eps != 0) before Coulomb-only pairs; the j
//     clusters' slot data are staged in shared memory on the way;
//   compute: lane L keeps i atom L%8 and walks that atom's queue with the
//     three other lanes of its group, one pair per lane per round; rounds
//     past every queue's LJ part skip the LJ code (water: H atoms carry no
//     LJ site, so most rounds are Coulomb-only);
//   accumulation: i forces stay in registers for the whole item; each pair
//     stores its force in its own (j atom, i atom) slot in shared memory, and
//     at the end of a chunk one lane per j atom sums its slots in i order and
//     adds the sum to the global fixed-point accumulators -- no atomics on
//     shared memory, and the order of every FP32 sum is fixed.
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Half-cluster kernel (kPairHalf, the default).  One warp runs one work item,
// an i cluster (8 atoms) against a run of j-cluster halves (4 atoms each),
// two halves A and B per step: lane L owns i atom L % 8 and half atom L / 8,
// its pair with half A in the .x and its pair with half B in the .y lane of
// packed f32x2 arithmetic, and bit L of each half's 32-bit mask.  INNER: the
// halves come from the inner list (any two halves of the item, each with its
// own shift and mask: only halves holding a pair within the inner radius);
// otherwise each entry of the full list supplies its own two halves, and a
// step whose pairs all lie beyond the cut-off is skipped after the distance
// test.  Per chunk of kHIt steps the warp stages, per step and half atom,
// the j coordinates with the step's shift already added, the charges and the
// LJ parameters, interleaved so that each lane reads its two pairs' operands
// as register pairs (three 16-byte shared loads per step).
//
// Arithmetic per pair (MDBas's formulas, src/ewald.c:356-369 and
// src/vdw.c:144-184, rearranged):
//   Coulomb: erfc(x) = t P(t) e^{-x^2}, t = 1/(1 + p x) (own fit, max
//     relative error 2.4e-8); with w = t P(t)/r + 2a/sqrt(pi) and
//     qe = q_i q_j e^{-(a r)^2}: g = qe w = -r dE/dr, E = g - qe 2a/sqrt(pi);
//   LJ: p = 4 eps (s^12 - s^6), r dp/dr = -6 eps' (2 s^12 - s^6) with
//     eps' = 4 eps; switch with u = max(r^2 - ron^2, 0) and D = rc^2 - ron^2:
//     S = 1 - u^2 (3D - 2u)/D^3 (exactly 1 inside ron), r dS/dr =
//     -12 r^2 (D - u) u / D^3 (exactly 0 inside ron);
//   force on i: (r dE/dr) / r^2 * (x_j - x_i).
// Energies and virials are summed per lane in FP32 within an item and
// converted to fixed point per lane and item; j forces are reduce-scattered
// over the 8 i lanes and added once per step and j atom in fixed point; i
// forces once per item.  Totals do not depend on which warp ran which item.
// ---------------------------------------------------------------------------
constexpr int kHIt = 8;  // steps per staged chunk
// Two copies of each step's data: in order (half A in .x, B in .y) for lanes
// with i atom 0-3, swapped for lanes with i atom 4-7, so that in the first
// round of the j-force reduce-scatter every lane keeps .x and passes .y.
struct HalfStage {
  float4 jd[2][kHIt * 4 * 3];  // [order][step][half atom]: (x,x,y,y), (z,z,q,q), (eps,eps,sig,sig)
  int4 mj[2][kHIt];            // [order][step]: masks of the two halves, their first slots
  float sh[kHIt][8];           // per step: sxA, sxB, syA, syB, szA, szB
  int2 js[kHIt];               // per step: first slot of half A, of half B
  uint2 mk[kHIt];              // per step: masks of half A, of half B
};

template <bool VDW, bool INNER, int MINB, bool EXACT>
__global__ void __launch_bounds__(256, MINB)
k_pair_half(const long long *__restrict__ counters, const int4 *__restrict__ items,
            const void *__restrict__ entriesV, const void *__restrict__ masksV,
            const float4 *__restrict__ xq, const float2 *__restrict__ lj, PairConstF c,
            long long *__restrict__ facc, int fstride, long long *__restrict__ acc) {
  __shared__ __align__(16) HalfStage stage[8];
  HalfStage &S = stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, jl = lane >> 3;
  const bool up = il & 4, mid = il & 2, lo = il & 1;
  const int comp = mid ? (lo ? 3 : 2) : (lo ? 1 : 0);
  const long long nItems = counters[1];
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long *fcomp = facc + (size_t)(comp < 3 ? comp : 0) * fstride;
  const float two_a = c.two_a_sqrtpi;
  const unsigned lanebit = 1u << lane;
  long long Ec = 0, Ev = 0, Vc = 0, Vv = 0;  // fixed point, per lane and item
  int npair = 0;
  bool overflow = false;

  // items handed out by a counter, the next index fetched while the
  // current item runs
  unsigned long long *work = reinterpret_cast<unsigned long long *>(acc + ACC_WORK);
  unsigned long long nxt = 0ull;
  if (lane == 0) nxt = atomicAdd(work, 1ull);
  long long it = (long long)__shfl_sync(0xffffffffu, nxt, 0);
  (void)nw;
  while (it < nItems) {
    if (lane == 0) nxt = atomicAdd(work, 1ull);
    const int4 item = items[it];
    const int ci = item.x, e0 = item.y, ne = item.z;
    const int nsteps = INNER ? (ne + 1) >> 1 : ne;
    const float4 xi = xq[ci * kClusterSize + il];
    const float2 li = lj[ci * kClusterSize + il];
    const float2 nx = f2(-xi.x), ny = f2(-xi.y), nz = f2(-xi.z);
    float2 fi_x = f2(0.f), fi_y = f2(0.f), fi_z = f2(0.f);
    float2 ec = f2(0.f), ev6 = f2(0.f), gs = f2(0.f), hs = f2(0.f);
    for (int s0 = 0; s0 < nsteps; s0 += kHIt) {
      const int nIt = min(kHIt, nsteps - s0);
      if (INNER) {
        const HalfEntry *__restrict__ hent = static_cast<const HalfEntry *>(entriesV);
        const unsigned *__restrict__ hmask = static_cast<const unsigned *>(masksV);
        const int nh = min(2 * kHIt, ne - 2 * s0);
        if (lane < nh) {
          const HalfEntry he = hent[e0 + 2 * s0 + lane];
          const unsigned m = hmask[e0 + 2 * s0 + lane];
          const int k = lane >> 1, side = lane & 1;
          float *sh = S.sh[k];
          int *js = reinterpret_cast<int *>(&S.js[k]);
          unsigned *mk = reinterpret_cast<unsigned *>(&S.mk[k]);
          sh[side] = he.sx;
          sh[2 + side] = he.sy;
          sh[4 + side] = he.sz;
          js[side] = he.jh * 4;
          mk[side] = m;
          if (side == 0 && lane == nh - 1) {  // a last half without a partner
            sh[1] = he.sx;
            sh[3] = he.sy;
            sh[5] = he.sz;
            js[1] = he.jh * 4;
            mk[1] = 0u;
          }
        }
      } else {
        const CPairEntry *__restrict__ ent = static_cast<const CPairEntry *>(entriesV);
        const uint2 *__restrict__ msk = static_cast<const uint2 *>(masksV);
        if (lane < nIt) {
          const CPairEntry en = ent[e0 + s0 + lane];
          *reinterpret_cast<float4 *>(S.sh[lane]) = make_float4(en.sx, en.sx, en.sy, en.sy);
          *reinterpret_cast<float2 *>(S.sh[lane] + 4) = make_float2(en.sz, en.sz);
          S.js[lane] = make_int2(en.j * kClusterSize, en.j * kClusterSize + 4);
          S.mk[lane] = msk[e0 + s0 + lane];
        }
      }
      __syncwarp();
      {
        const int k = lane >> 2, a = lane & 3;
        if (k < nIt) {
          const int2 js = S.js[k];
          const float4 sxy = *reinterpret_cast<const float4 *>(S.sh[k]);
          const float2 sz = *reinterpret_cast<const float2 *>(S.sh[k] + 4);
          const float4 xa = xq[js.x + a], xb = xq[js.y + a];
          const float2 la = lj[js.x + a], lb = lj[js.y + a];
          const float ax = xa.x + sxy.x, bx = xb.x + sxy.y, ay = xa.y + sxy.z, by = xb.y + sxy.w;
          const float az = xa.z + sz.x, bz = xb.z + sz.y;
          float4 *d = &S.jd[0][(k * 4 + a) * 3];
          d[0] = make_float4(ax, bx, ay, by);
          d[1] = make_float4(az, bz, xa.w, xb.w);
          d[2] = make_float4(la.x, lb.x, la.y, lb.y);
          float4 *e = &S.jd[1][(k * 4 + a) * 3];
          e[0] = make_float4(bx, ax, by, ay);
          e[1] = make_float4(bz, az, xb.w, xa.w);
          e[2] = make_float4(lb.x, la.x, lb.y, la.y);
          if (a == 0) {
            const uint2 mk = S.mk[k];
            S.mj[0][k] = make_int4((int)mk.x, (int)mk.y, js.x, js.y);
            S.mj[1][k] = make_int4((int)mk.y, (int)mk.x, js.y, js.x);
          }
        }
      }
      __syncwarp();
      const float4 *__restrict__ jdl = S.jd[up ? 1 : 0];
      const int4 *__restrict__ mjl = S.mj[up ? 1 : 0];
      for (int k = 0; k < nIt; ++k) {
        // this lane's two pairs: .x with the half it keeps in the reduction
        const float4 p0 = jdl[(k * 4 + jl) * 3], p1 = jdl[(k * 4 + jl) * 3 + 1];
        const int4 mj = mjl[k];
        const uint2 mk = make_uint2((unsigned)mj.x, (unsigned)mj.y);
        const float2 dx = __fadd2_rn(make_float2(p0.x, p0.y), nx);
        const float2 dy = __fadd2_rn(make_float2(p0.z, p0.w), ny);
        const float2 dz = __fadd2_rn(make_float2(p1.x, p1.y), nz);
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        // EXACT: the inner list was written by the search from these same
        // FP32 distances against this same rc^2, so its bits are the test
        const bool ina = (mk.x & lanebit) && (EXACT || r2.x <= c.rc2);
        const bool inb = (mk.y & lanebit) && (EXACT || r2.y <= c.rc2);
        if (!INNER && !__any_sync(0xffffffffu, ina || inb)) continue;
        if (!EXACT) {
          if (ina) ++npair;
          if (inb) ++npair;
        }
        const float2 r2s = make_float2(ina ? r2.x : 1.0f, inb ? r2.y : 1.0f);
        const float2 rinv = make_float2(rsqrt_approx(r2s.x), rsqrt_approx(r2s.y));
        const float2 rinv2 = __fmul2_rn(rinv, rinv);
        const float2 r = __fmul2_rn(r2s, rinv);
        const float2 qq0 = __fmul2_rn(f2(xi.w), make_float2(p1.z, p1.w));
        const float2 qq = make_float2(ina ? qq0.x : 0.f, inb ? qq0.y : 0.f);
        const float2 targ = __ffma2_rn(f2(c.p_alpha), r, f2(1.0f));
        const float2 t = make_float2(rcp_approx(targ.x), rcp_approx(targ.y));
        const float2 earg = __fmul2_rn(f2(-c.c_ex), r2s);
        const float2 ex = make_float2(ex2_approx(earg.x), ex2_approx(earg.y));
        float2 poly = __ffma2_rn(f2(kErfcC7), t, f2(kErfcC6));
        poly = __ffma2_rn(poly, t, f2(kErfcC5));
        poly = __ffma2_rn(poly, t, f2(kErfcC4));
        poly = __ffma2_rn(poly, t, f2(kErfcC3));
        poly = __ffma2_rn(poly, t, f2(kErfcC2));
        poly = __ffma2_rn(poly, t, f2(kErfcC1));
        poly = __ffma2_rn(poly, t, f2(kErfcC0));
        const float2 w = __ffma2_rn(__fmul2_rn(rinv, t), poly, f2(two_a));
        const float2 qe = __fmul2_rn(qq, ex);
        const float2 g = __fmul2_rn(qe, w);  // -r dE_c/dr
        ec = __fadd2_rn(ec, __ffma2_rn(qe, f2(-two_a), g));
        gs = __fadd2_rn(gs, g);
        float2 F = g;  // -(r dE/dr) while VDW adds to it below
        if (VDW) {
          const float4 lp = jdl[(k * 4 + jl) * 3 + 2];
          const float2 eps0 = __fmul2_rn(f2(li.x), make_float2(lp.x, lp.y));
          const float2 eps = make_float2(ina ? eps0.x : 0.f, inb ? eps0.y : 0.f);
          const float2 sg = __fadd2_rn(f2(li.y), make_float2(lp.z, lp.w));
          const float2 s2 = __fmul2_rn(__fmul2_rn(sg, sg), rinv2);
          const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
          const float2 s12 = __fmul2_rn(s6, s6);
          const float2 a = __ffma2_rn(s6, f2(-1.0f), s12);  // s12 - s6
          const float2 b = __fadd2_rn(a, s12);              // 2 s12 - s6
          const float2 u0 = __fadd2_rn(r2s, f2(-c.ron2));
          const float2 u = make_float2(fmaxf(u0.x, 0.f), fmaxf(u0.y, 0.f));
          const float2 m = __fmul2_rn(__fmul2_rn(u, u), __ffma2_rn(u, f2(-2.0f), f2(c.sw_3d)));
          const float2 S6 = __ffma2_rn(m, f2(c.sw_6), f2(-6.0f));  // -6 S
          const float2 dS = __fmul2_rn(__fmul2_rn(__ffma2_rn(u, f2(-1.0f), f2(c.sw_d)), u),
                                       __fmul2_rn(r2s, f2(c.sw_m12)));  // r dS/dr
          const float2 pv = __fmul2_rn(eps, a);
          ev6 = __ffma2_rn(pv, S6, ev6);
          const float2 hv = __fmul2_rn(eps, __ffma2_rn(a, dS, __fmul2_rn(b, S6)));  // r dE_v/dr
          hs = __fadd2_rn(hs, hv);
          F = __ffma2_rn(F, f2(-1.0f), hv);  // r dE/dr
        } else {
          F = __fmul2_rn(F, f2(-1.0f));
        }
        // F = r dE/dr: the force on i is F / r^2 (x_j - x_i)
        const float2 Fr = __fmul2_rn(F, rinv2);
        const float2 fx = __fmul2_rn(Fr, dx), fy = __fmul2_rn(Fr, dy), fz = __fmul2_rn(Fr, dz);
        fi_x = __fadd2_rn(fi_x, fx);
        fi_y = __fadd2_rn(fi_y, fy);
        fi_z = __fadd2_rn(fi_z, fz);
        // reduce-scatter of the two j atoms' forces over the 8 i lanes: every
        // lane keeps its .x atom (half A for i atoms 0-3, B for 4-7) and
        // passes its .y atom to the lane of i atom i ^ 4, which keeps it
        float k0 = fx.x + __shfl_xor_sync(0xffffffffu, fx.y, 4);
        float k1 = fy.x + __shfl_xor_sync(0xffffffffu, fy.y, 4);
        float k2 = fz.x + __shfl_xor_sync(0xffffffffu, fz.y, 4);
        const float t0 = mid ? k0 : k2, t1 = mid ? k1 : 0.f;
        float u0 = mid ? k2 : k0, u1 = mid ? 0.f : k1;
        u0 += __shfl_xor_sync(0xffffffffu, t0, 2);
        u1 += __shfl_xor_sync(0xffffffffu, t1, 2);
        const float wv = lo ? u0 : u1;
        float v = lo ? u1 : u0;
        v += __shfl_xor_sync(0xffffffffu, wv, 1);
        const bool put = comp < 3 && v != 0.f;
        overflow |= put && !(fabsf(v) < kForceLimitF);
        red_add_if(put, fcomp + mj.z + jl, fix_f(-v));
      }
      __syncwarp();
    }
    // i forces: the lane's two pairs, then the four j lanes of each i atom
    float fix = fi_x.x + fi_x.y, fiy = fi_y.x + fi_y.y, fiz = fi_z.x + fi_z.y;
    fix += __shfl_xor_sync(0xffffffffu, fix, 8);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 8);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 8);
    fix += __shfl_xor_sync(0xffffffffu, fix, 16);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 16);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 16);
    if (jl < 3) {
      const float v = (jl == 0) ? fix : (jl == 1 ? fiy : fiz);
      if (v != 0.f) {
        overflow |= !(fabsf(v) < kForceLimitF);
        red_add(facc + (size_t)jl * fstride + ci * kClusterSize + il, fix_f(v));
      }
    }
    // each lane's share of the item in fixed point on its own
    Ec += fix_e((double)ec.x + (double)ec.y);
    Ev += fix_e(((double)ev6.x + (double)ev6.y) * (-1.0 / 6.0));
    Vc += fix_e(-((double)gs.x + (double)gs.y));
    Vv += fix_e((double)hs.x + (double)hs.y);
    it = (long long)__shfl_sync(0xffffffffu, nxt, 0);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Ec += __shfl_xor_sync(0xffffffffu, Ec, o);
    Ev += __shfl_xor_sync(0xffffffffu, Ev, o);
    Vc += __shfl_xor_sync(0xffffffffu, Vc, o);
    Vv += __shfl_xor_sync(0xffffffffu, Vv, o);
    npair += __shfl_xor_sync(0xffffffffu, npair, o);
  }
  if (__any_sync(0xffffffffu, overflow) && lane == 0) raise_flag(acc, FLAG_OVERFLOW);
  if (lane == 0) {
    red_add(acc + ACC_E_DIR, Ec);
    red_add(acc + ACC_E_VDW, Ev);
    red_add(acc + ACC_V_DIR, Vc);
    red_add(acc + ACC_V_VDW, Vv);
    // EXACT: the pairs were counted by the search (inner-list counter 4)
    if (EXACT) {
      if (gw == 0) red_add(acc + ACC_NPAIR, counters[4]);
    } else {
      red_add(acc + ACC_NPAIR, (long long)npair);
    }
  }
}

// Lean form of k_pair_half over the inner list (exact, or pruned with the
// cut-off tested here; the default): the same pairs and arithmetic with fewer
// instructions and registers per step -- pairs outside the mask get
// r^2 = 1e30 instead of zeroed charge and LJ products (their terms vanish:
// exp underflows to 0, the LJ powers to 0, the switch variable is clamped at
// D so S and dS stay finite), per step only the largest |j force| is kept
// for the range check (a NaN shows up in the i forces, checked per item),
// the per-lane 64-bit energy sums live in shared memory, and warps take items
// from a counter.  Forces and energies equal k_pair_half's bit for bit.
template <bool VDW, bool INNER, bool EXACT>
__global__ void __launch_bounds__(256, 4)
k_pair_half_lean(const long long *__restrict__ counters, const int4 *__restrict__ items,
            const void *__restrict__ entriesV, const void *__restrict__ masksV,
            const float4 *__restrict__ xq, const float2 *__restrict__ lj, PairConstF c,
            long long *__restrict__ facc, int fstride, long long *__restrict__ acc) {
  __shared__ __align__(16) HalfStage stage[8];
  __shared__ long long esum[4][256];  // per lane: Ec, Ev, Vc, Vv
  HalfStage &S = stage[threadIdx.x >> 5];
  const float kFar = 1e30f;
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, jl = lane >> 3;
  const bool up = il & 4, mid = il & 2, lo = il & 1;
  const int comp = mid ? (lo ? 3 : 2) : (lo ? 1 : 0);
  const long long nItems = counters[1];
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long *fcomp = facc + (size_t)(comp < 3 ? comp : 0) * fstride;
  const float two_a = c.two_a_sqrtpi;
  const unsigned lanebit = 1u << lane;
  esum[0][threadIdx.x] = 0;
  esum[1][threadIdx.x] = 0;
  esum[2][threadIdx.x] = 0;
  esum[3][threadIdx.x] = 0;
  int npair = 0;
  bool overflow = false;
  float vmax = 0.f;

  // items handed out by a counter (each warp takes the next one when it is
  // done, the following index fetched while the current item runs), so no
  // warp is left with a long tail of large items
  unsigned long long *work = reinterpret_cast<unsigned long long *>(acc + ACC_WORK);
  unsigned long long nxt = 0ull;
  if (lane == 0) nxt = atomicAdd(work, 1ull);
  long long it = (long long)__shfl_sync(0xffffffffu, nxt, 0);
  (void)gw;
  (void)nw;
  while (it < nItems) {
    if (lane == 0) nxt = atomicAdd(work, 1ull);
    const int4 item = items[it];
    const int ci = item.x, e0 = item.y, ne = item.z;
    const int nsteps = INNER ? (ne + 1) >> 1 : ne;
    const float4 xi = xq[ci * kClusterSize + il];
    const float2 li = lj[ci * kClusterSize + il];
    const float2 nx = f2(-xi.x), ny = f2(-xi.y), nz = f2(-xi.z);
    float2 fi_x = f2(0.f), fi_y = f2(0.f), fi_z = f2(0.f);
    float2 ec = f2(0.f), ev6 = f2(0.f), gs = f2(0.f), hs = f2(0.f);
    for (int s0 = 0; s0 < nsteps; s0 += kHIt) {
      const int nIt = min(kHIt, nsteps - s0);
      if (INNER) {
        const HalfEntry *__restrict__ hent = static_cast<const HalfEntry *>(entriesV);
        const unsigned *__restrict__ hmask = static_cast<const unsigned *>(masksV);
        const int nh = min(2 * kHIt, ne - 2 * s0);
        if (lane < nh) {
          const HalfEntry he = hent[e0 + 2 * s0 + lane];
          const unsigned m = hmask[e0 + 2 * s0 + lane];
          const int k = lane >> 1, side = lane & 1;
          float *sh = S.sh[k];
          int *js = reinterpret_cast<int *>(&S.js[k]);
          unsigned *mk = reinterpret_cast<unsigned *>(&S.mk[k]);
          sh[side] = he.sx;
          sh[2 + side] = he.sy;
          sh[4 + side] = he.sz;
          js[side] = he.jh * 4;
          mk[side] = m;
          if (side == 0 && lane == nh - 1) {  // a last half without a partner
            sh[1] = he.sx;
            sh[3] = he.sy;
            sh[5] = he.sz;
            js[1] = he.jh * 4;
            mk[1] = 0u;
          }
        }
      } else {
        // the full list: each entry supplies its own two halves
        const CPairEntry *__restrict__ ent = static_cast<const CPairEntry *>(entriesV);
        const uint2 *__restrict__ msk = static_cast<const uint2 *>(masksV);
        if (lane < nIt) {
          const CPairEntry en = ent[e0 + s0 + lane];
          *reinterpret_cast<float4 *>(S.sh[lane]) = make_float4(en.sx, en.sx, en.sy, en.sy);
          *reinterpret_cast<float2 *>(S.sh[lane] + 4) = make_float2(en.sz, en.sz);
          S.js[lane] = make_int2(en.j * kClusterSize, en.j * kClusterSize + 4);
          S.mk[lane] = msk[e0 + s0 + lane];
        }
      }
      __syncwarp();
      {
        const int k = lane >> 2, a = lane & 3;
        if (k < nIt) {
          const int2 js = S.js[k];
          const float4 sxy = *reinterpret_cast<const float4 *>(S.sh[k]);
          const float2 sz = *reinterpret_cast<const float2 *>(S.sh[k] + 4);
          const float4 xa = xq[js.x + a], xb = xq[js.y + a];
          const float2 la = lj[js.x + a], lb = lj[js.y + a];
          const float ax = xa.x + sxy.x, bx = xb.x + sxy.y, ay = xa.y + sxy.z, by = xb.y + sxy.w;
          const float az = xa.z + sz.x, bz = xb.z + sz.y;
          float4 *d = &S.jd[0][(k * 4 + a) * 3];
          d[0] = make_float4(ax, bx, ay, by);
          d[1] = make_float4(az, bz, xa.w, xb.w);
          d[2] = make_float4(la.x, lb.x, la.y, lb.y);
          float4 *e = &S.jd[1][(k * 4 + a) * 3];
          e[0] = make_float4(bx, ax, by, ay);
          e[1] = make_float4(bz, az, xb.w, xa.w);
          e[2] = make_float4(lb.x, la.x, lb.y, la.y);
          if (a == 0) {
            const uint2 mk = S.mk[k];
            S.mj[0][k] = make_int4((int)mk.x, (int)mk.y, js.x, js.y);
            S.mj[1][k] = make_int4((int)mk.y, (int)mk.x, js.y, js.x);
          }
        }
      }
      __syncwarp();
      const float4 *__restrict__ jdl = S.jd[up ? 1 : 0];
      const int4 *__restrict__ mjl = S.mj[up ? 1 : 0];
      for (int k = 0; k < nIt; ++k) {
        // this lane's two pairs: .x with the half it keeps in the reduction
        const float4 p0 = jdl[(k * 4 + jl) * 3], p1 = jdl[(k * 4 + jl) * 3 + 1];
        const int4 mj = mjl[k];
        const uint2 mk = make_uint2((unsigned)mj.x, (unsigned)mj.y);
        const float2 dx = __fadd2_rn(make_float2(p0.x, p0.y), nx);
        const float2 dy = __fadd2_rn(make_float2(p0.z, p0.w), ny);
        const float2 dz = __fadd2_rn(make_float2(p1.x, p1.y), nz);
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        // EXACT: the inner list was written by the search from these same
        // FP32 distances against this same rc^2, so its bits are the test
        const bool ina = (mk.x & lanebit) && (EXACT || r2.x <= c.rc2);
        const bool inb = (mk.y & lanebit) && (EXACT || r2.y <= c.rc2);
        // the full list: a step whose pairs all lie beyond the cut-off is skipped
        if (!INNER && !__any_sync(0xffffffffu, ina || inb)) continue;
        if (!EXACT) npair += (int)ina + (int)inb;
        const float2 r2s = make_float2(ina ? r2.x : kFar, inb ? r2.y : kFar);
        const float2 rinv = make_float2(rsqrt_approx(r2s.x), rsqrt_approx(r2s.y));
        const float2 rinv2 = __fmul2_rn(rinv, rinv);
        const float2 r = __fmul2_rn(r2s, rinv);
        const float2 qq = __fmul2_rn(f2(xi.w), make_float2(p1.z, p1.w));
        const float2 targ = __ffma2_rn(f2(c.p_alpha), r, f2(1.0f));
        const float2 t = make_float2(rcp_approx(targ.x), rcp_approx(targ.y));
        const float2 earg = __fmul2_rn(f2(-c.c_ex), r2s);
        const float2 ex = make_float2(ex2_approx(earg.x), ex2_approx(earg.y));
        float2 poly = __ffma2_rn(f2(kErfcC7), t, f2(kErfcC6));
        poly = __ffma2_rn(poly, t, f2(kErfcC5));
        poly = __ffma2_rn(poly, t, f2(kErfcC4));
        poly = __ffma2_rn(poly, t, f2(kErfcC3));
        poly = __ffma2_rn(poly, t, f2(kErfcC2));
        poly = __ffma2_rn(poly, t, f2(kErfcC1));
        poly = __ffma2_rn(poly, t, f2(kErfcC0));
        const float2 w = __ffma2_rn(__fmul2_rn(rinv, t), poly, f2(two_a));
        const float2 qe = __fmul2_rn(qq, ex);
        const float2 g = __fmul2_rn(qe, w);  // -r dE_c/dr
        ec = __fadd2_rn(ec, __ffma2_rn(qe, f2(-two_a), g));
        gs = __fadd2_rn(gs, g);
        float2 F = g;  // -(r dE/dr) while VDW adds to it below
        if (VDW) {
          const float4 lp = jdl[(k * 4 + jl) * 3 + 2];
          const float2 eps = __fmul2_rn(f2(li.x), make_float2(lp.x, lp.y));
          const float2 sg = __fadd2_rn(f2(li.y), make_float2(lp.z, lp.w));
          const float2 s2 = __fmul2_rn(__fmul2_rn(sg, sg), rinv2);
          const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
          const float2 s12 = __fmul2_rn(s6, s6);
          const float2 a = __ffma2_rn(s6, f2(-1.0f), s12);  // s12 - s6
          const float2 b = __fadd2_rn(a, s12);              // 2 s12 - s6
          const float2 u0 = __fadd2_rn(r2s, f2(-c.ron2));
          const float2 u = make_float2(fminf(fmaxf(u0.x, 0.f), c.sw_d),
                                       fminf(fmaxf(u0.y, 0.f), c.sw_d));
          const float2 m = __fmul2_rn(__fmul2_rn(u, u), __ffma2_rn(u, f2(-2.0f), f2(c.sw_3d)));
          const float2 S6 = __ffma2_rn(m, f2(c.sw_6), f2(-6.0f));  // -6 S
          const float2 dS = __fmul2_rn(__fmul2_rn(__ffma2_rn(u, f2(-1.0f), f2(c.sw_d)), u),
                                       __fmul2_rn(r2s, f2(c.sw_m12)));  // r dS/dr
          const float2 pv = __fmul2_rn(eps, a);
          ev6 = __ffma2_rn(pv, S6, ev6);
          const float2 hv = __fmul2_rn(eps, __ffma2_rn(a, dS, __fmul2_rn(b, S6)));  // r dE_v/dr
          hs = __fadd2_rn(hs, hv);
          F = __ffma2_rn(F, f2(-1.0f), hv);  // r dE/dr
        } else {
          F = __fmul2_rn(F, f2(-1.0f));
        }
        // F = r dE/dr: the force on i is F / r^2 (x_j - x_i)
        const float2 Fr = __fmul2_rn(F, rinv2);
        const float2 fx = __fmul2_rn(Fr, dx), fy = __fmul2_rn(Fr, dy), fz = __fmul2_rn(Fr, dz);
        fi_x = __fadd2_rn(fi_x, fx);
        fi_y = __fadd2_rn(fi_y, fy);
        fi_z = __fadd2_rn(fi_z, fz);
        // reduce-scatter of the two j atoms' forces over the 8 i lanes: every
        // lane keeps its .x atom (half A for i atoms 0-3, B for 4-7) and
        // passes its .y atom to the lane of i atom i ^ 4, which keeps it
        float k0 = fx.x + __shfl_xor_sync(0xffffffffu, fx.y, 4);
        float k1 = fy.x + __shfl_xor_sync(0xffffffffu, fy.y, 4);
        float k2 = fz.x + __shfl_xor_sync(0xffffffffu, fz.y, 4);
        const float t0 = mid ? k0 : k2, t1 = mid ? k1 : 0.f;
        float u0 = mid ? k2 : k0, u1 = mid ? 0.f : k1;
        u0 += __shfl_xor_sync(0xffffffffu, t0, 2);
        u1 += __shfl_xor_sync(0xffffffffu, t1, 2);
        const float wv = lo ? u0 : u1;
        float v = lo ? u1 : u0;
        v += __shfl_xor_sync(0xffffffffu, wv, 1);
        const bool put = comp < 3 && v != 0.f;
        vmax = fmaxf(vmax, fabsf(v));
        red_add_if(put, fcomp + mj.z + jl, fix_f(-v));
      }
      __syncwarp();
    }
    // i forces: the lane's two pairs, then the four j lanes of each i atom
    float fix = fi_x.x + fi_x.y, fiy = fi_y.x + fi_y.y, fiz = fi_z.x + fi_z.y;
    fix += __shfl_xor_sync(0xffffffffu, fix, 8);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 8);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 8);
    fix += __shfl_xor_sync(0xffffffffu, fix, 16);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 16);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 16);
    if (jl < 3) {
      const float v = (jl == 0) ? fix : (jl == 1 ? fiy : fiz);
      if (v != 0.f) {
        overflow |= !(fabsf(v) < kForceLimitF);
        red_add(facc + (size_t)jl * fstride + ci * kClusterSize + il, fix_f(v));
      }
    }
    // each lane's share of the item in fixed point on its own
    esum[0][threadIdx.x] += fix_e((double)ec.x + (double)ec.y);
    esum[1][threadIdx.x] += fix_e(((double)ev6.x + (double)ev6.y) * (-1.0 / 6.0));
    esum[2][threadIdx.x] += fix_e(-((double)gs.x + (double)gs.y));
    esum[3][threadIdx.x] += fix_e((double)hs.x + (double)hs.y);
    it = (long long)__shfl_sync(0xffffffffu, nxt, 0);
  }
  long long Ec = esum[0][threadIdx.x], Ev = esum[1][threadIdx.x], Vc = esum[2][threadIdx.x],
            Vv = esum[3][threadIdx.x];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Ec += __shfl_xor_sync(0xffffffffu, Ec, o);
    Ev += __shfl_xor_sync(0xffffffffu, Ev, o);
    Vc += __shfl_xor_sync(0xffffffffu, Vc, o);
    Vv += __shfl_xor_sync(0xffffffffu, Vv, o);
    if (!EXACT) npair += __shfl_xor_sync(0xffffffffu, npair, o);
  }
  overflow |= comp < 3 && !(vmax < kForceLimitF);
  if (__any_sync(0xffffffffu, overflow) && lane == 0) raise_flag(acc, FLAG_OVERFLOW);
  if (lane == 0) {
    red_add(acc + ACC_E_DIR, Ec);
    red_add(acc + ACC_E_VDW, Ev);
    red_add(acc + ACC_V_DIR, Vc);
    red_add(acc + ACC_V_VDW, Vv);
    // EXACT: the pairs were counted by the search (inner-list counter 4)
    if (EXACT) {
      if (gw == 0) red_add(acc + ACC_NPAIR, counters[4]);
    } else {
      red_add(acc + ACC_NPAIR, (long long)npair);
    }
  }
}

// ---------------------------------------------------------------------------
// Quarter-cluster kernel (kPairQuad).  Units of 4 x 4 atoms: an i-cluster
// half (i atoms 4 ih .. 4 ih + 3) against a j-cluster half.  The kernel reads
// the same inner list as k_pair_half (halves with 32-bit masks, bit i + 8 k)
// and splits each half's mask into its two i halves; a unit is kept when its
// 16 bits hold a pair, which drops the i half that lies out of reach (pair
// efficiency of water at rc = 12 A: ~0.57 against ~0.49 for 8 x 4).  One warp
// runs one work item in two passes, i half 0 then 1; per pass the item's
// halves are compacted (ballot) into the units of that i half, and each
// warp step computes four units: lane L owns i atom a = L % 4 of the pass's
// i half, j atom k = (L / 4) % 4 of units 2p and 2p + 1 (p = L / 16) in the
// .x and .y lanes of packed f32x2 arithmetic.  Same arithmetic as
// k_pair_half.  j forces: reduce-scatter over the four i lanes (xor 2 with
// the swapped staging order making it select-free, then xor 1), two
// fixed-point additions per lane and step; i forces once per pass.
// ---------------------------------------------------------------------------
constexpr int kQIt = 8;     // steps per staged chunk (32 units)
constexpr int kQWarps = 4;  // warps per block (6.9 KB of staging each)
struct QuadStage {
  float4 jd[2][kQIt * 2 * 4 * 3];  // [order][(step * 2 + p) * 4 + k][3]
  int4 mj[2][kQIt * 2];            // [order][step * 2 + p]: masks of units .x, .y; first slots
  HalfEntry ue[32];                // the pass's units: their half entries
  unsigned um[32];                 // their masks, bit a + 8 k
};

template <bool VDW, bool EXACT>
__global__ void __launch_bounds__(kQWarps * 32, 6)
k_pair_quad(const long long *__restrict__ counters, const int4 *__restrict__ items,
            const HalfEntry *__restrict__ hent, const unsigned *__restrict__ hmask,
            const float4 *__restrict__ xq, const float2 *__restrict__ lj, PairConstF c,
            long long *__restrict__ facc, int fstride, long long *__restrict__ acc) {
  __shared__ __align__(16) QuadStage stage[kQWarps];
  QuadStage &S = stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int a = lane & 3, k = (lane >> 2) & 3, p = lane >> 4;
  const int ord = a >> 1;          // lanes a >= 2 read the swapped order
  const bool odd = a & 1;
  const int sb = a + 8 * k;        // this lane's bit in a unit mask
  const long long nItems = counters[1];
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long *f0 = facc + (size_t)(odd ? 2 : 0) * fstride;  // first addition: x (even) or z (odd)
  long long *f1 = facc + (size_t)fstride;                  // second (even lanes): y
  const float two_a = c.two_a_sqrtpi;
  long long Ec = 0, Ev = 0, Vc = 0, Vv = 0;
  int npair = 0;
  bool overflow = false;

  for (long long it = gw; it < nItems; it += nw) {
    const int4 item = items[it];
    const int ci = item.x, e0 = item.y, ne = item.z;
    for (int ih = 0; ih < 2; ++ih) {
      const int islot = ci * kClusterSize + 4 * ih + a;
      const float4 xi = xq[islot];
      const float2 li = lj[islot];
      const float2 nx = f2(-xi.x), ny = f2(-xi.y), nz = f2(-xi.z);
      float2 fi_x = f2(0.f), fi_y = f2(0.f), fi_z = f2(0.f);
      float2 ec = f2(0.f), ev6 = f2(0.f), gs = f2(0.f), hs = f2(0.f);
      for (int h0 = 0; h0 < ne; h0 += 32) {
        // the units of this i half among the next 32 halves
        unsigned mu = 0u;
        HalfEntry he{};
        if (h0 + lane < ne) {
          he = hent[e0 + h0 + lane];
          mu = (hmask[e0 + h0 + lane] >> (4 * ih)) & 0x0f0f0f0fu;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, mu != 0u);
        const int nU = __popc(bal);
        if (mu != 0u) {
          const int pos = __popc(bal & ((1u << lane) - 1u));
          S.ue[pos] = he;
          S.um[pos] = mu;
        }
        __syncwarp();
        const int nSteps = (nU + 3) >> 2;
        // stage: tuple t = (step, p, k), two per lane
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int t = lane + 32 * r;
          const int st = t >> 3, pp = (t >> 2) & 1, kk = t & 3;
          const int ua = 4 * st + 2 * pp, ub = ua + 1;
          if (st < nSteps) {
            const bool va = ua < nU, vb = ub < nU;
            const HalfEntry ea = S.ue[va ? ua : 0];
            const HalfEntry eb = S.ue[vb ? ub : (va ? ua : 0)];
            const float4 xa = xq[ea.jh * 4 + kk], xb = xq[eb.jh * 4 + kk];
            const float2 la = lj[ea.jh * 4 + kk], lb = lj[eb.jh * 4 + kk];
            const float ax = xa.x + ea.sx, bx = xb.x + eb.sx, ay = xa.y + ea.sy,
                        by = xb.y + eb.sy, az = xa.z + ea.sz, bz = xb.z + eb.sz;
            const int q = ((st * 2 + pp) * 4 + kk) * 3;
            float4 *d = &S.jd[0][q];
            d[0] = make_float4(ax, bx, ay, by);
            d[1] = make_float4(az, bz, xa.w, xb.w);
            d[2] = make_float4(la.x, lb.x, la.y, lb.y);
            float4 *e = &S.jd[1][q];
            e[0] = make_float4(bx, ax, by, ay);
            e[1] = make_float4(bz, az, xb.w, xa.w);
            e[2] = make_float4(lb.x, la.x, lb.y, la.y);
            if (kk == 0) {
              const int ma = va ? (int)S.um[ua] : 0, mb = vb ? (int)S.um[ub] : 0;
              S.mj[0][st * 2 + pp] = make_int4(ma, mb, ea.jh * 4, eb.jh * 4);
              S.mj[1][st * 2 + pp] = make_int4(mb, ma, eb.jh * 4, ea.jh * 4);
            }
          }
        }
        __syncwarp();
        const float4 *__restrict__ jdl = S.jd[ord];
        const int4 *__restrict__ mjl = S.mj[ord];
        for (int st = 0; st < nSteps; ++st) {
          const int q = ((st * 2 + p) * 4 + k) * 3;
          const float4 p0 = jdl[q], p1 = jdl[q + 1];
          const int4 mj = mjl[st * 2 + p];
          const float2 dx = __fadd2_rn(make_float2(p0.x, p0.y), nx);
          const float2 dy = __fadd2_rn(make_float2(p0.z, p0.w), ny);
          const float2 dz = __fadd2_rn(make_float2(p1.x, p1.y), nz);
          const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
          const bool ina = ((unsigned)mj.x >> sb) & 1u && (EXACT || r2.x <= c.rc2);
          const bool inb = ((unsigned)mj.y >> sb) & 1u && (EXACT || r2.y <= c.rc2);
          if (!EXACT) {
            if (ina) ++npair;
            if (inb) ++npair;
          }
          const float2 r2s = make_float2(ina ? r2.x : 1.0f, inb ? r2.y : 1.0f);
          const float2 rinv = make_float2(rsqrt_approx(r2s.x), rsqrt_approx(r2s.y));
          const float2 rinv2 = __fmul2_rn(rinv, rinv);
          const float2 r = __fmul2_rn(r2s, rinv);
          const float2 qq0 = __fmul2_rn(f2(xi.w), make_float2(p1.z, p1.w));
          const float2 qq = make_float2(ina ? qq0.x : 0.f, inb ? qq0.y : 0.f);
          const float2 targ = __ffma2_rn(f2(c.p_alpha), r, f2(1.0f));
          const float2 t = make_float2(rcp_approx(targ.x), rcp_approx(targ.y));
          const float2 earg = __fmul2_rn(f2(-c.c_ex), r2s);
          const float2 ex = make_float2(ex2_approx(earg.x), ex2_approx(earg.y));
          float2 poly = __ffma2_rn(f2(kErfcC7), t, f2(kErfcC6));
          poly = __ffma2_rn(poly, t, f2(kErfcC5));
          poly = __ffma2_rn(poly, t, f2(kErfcC4));
          poly = __ffma2_rn(poly, t, f2(kErfcC3));
          poly = __ffma2_rn(poly, t, f2(kErfcC2));
          poly = __ffma2_rn(poly, t, f2(kErfcC1));
          poly = __ffma2_rn(poly, t, f2(kErfcC0));
          const float2 w = __ffma2_rn(__fmul2_rn(rinv, t), poly, f2(two_a));
          const float2 qe = __fmul2_rn(qq, ex);
          const float2 g = __fmul2_rn(qe, w);  // -r dE_c/dr
          ec = __fadd2_rn(ec, __ffma2_rn(qe, f2(-two_a), g));
          gs = __fadd2_rn(gs, g);
          float2 F = g;
          if (VDW) {
            const float4 lp = jdl[q + 2];
            const float2 eps0 = __fmul2_rn(f2(li.x), make_float2(lp.x, lp.y));
            const float2 eps = make_float2(ina ? eps0.x : 0.f, inb ? eps0.y : 0.f);
            const float2 sg = __fadd2_rn(f2(li.y), make_float2(lp.z, lp.w));
            const float2 s2 = __fmul2_rn(__fmul2_rn(sg, sg), rinv2);
            const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
            const float2 s12 = __fmul2_rn(s6, s6);
            const float2 av = __ffma2_rn(s6, f2(-1.0f), s12);  // s12 - s6
            const float2 bv = __fadd2_rn(av, s12);              // 2 s12 - s6
            const float2 u0 = __fadd2_rn(r2s, f2(-c.ron2));
            const float2 u = make_float2(fmaxf(u0.x, 0.f), fmaxf(u0.y, 0.f));
            const float2 m = __fmul2_rn(__fmul2_rn(u, u), __ffma2_rn(u, f2(-2.0f), f2(c.sw_3d)));
            const float2 S6 = __ffma2_rn(m, f2(c.sw_6), f2(-6.0f));  // -6 S
            const float2 dS = __fmul2_rn(__fmul2_rn(__ffma2_rn(u, f2(-1.0f), f2(c.sw_d)), u),
                                         __fmul2_rn(r2s, f2(c.sw_m12)));  // r dS/dr
            const float2 pv = __fmul2_rn(eps, av);
            ev6 = __ffma2_rn(pv, S6, ev6);
            const float2 hv = __fmul2_rn(eps, __ffma2_rn(av, dS, __fmul2_rn(bv, S6)));
            hs = __fadd2_rn(hs, hv);
            F = __ffma2_rn(F, f2(-1.0f), hv);  // r dE/dr
          } else {
            F = __fmul2_rn(F, f2(-1.0f));
          }
          const float2 Fr = __fmul2_rn(F, rinv2);
          const float2 fx = __fmul2_rn(Fr, dx), fy = __fmul2_rn(Fr, dy), fz = __fmul2_rn(Fr, dz);
          fi_x = __fadd2_rn(fi_x, fx);
          fi_y = __fadd2_rn(fi_y, fy);
          fi_z = __fadd2_rn(fi_z, fz);
          // j forces over the four i lanes: keep .x, pass .y to lane a ^ 2
          // (which keeps that unit), then x, y to the even and z to the odd
          // lane of each pair
          const float k0 = fx.x + __shfl_xor_sync(0xffffffffu, fx.y, 2);
          const float k1 = fy.x + __shfl_xor_sync(0xffffffffu, fy.y, 2);
          const float k2 = fz.x + __shfl_xor_sync(0xffffffffu, fz.y, 2);
          const float v0 = (odd ? k2 : k0) + __shfl_xor_sync(0xffffffffu, odd ? k0 : k2, 1);
          const float v1 = k1 + __shfl_xor_sync(0xffffffffu, k1, 1);
          const int js = mj.z + k;
          const bool put0 = v0 != 0.f, put1 = !odd && v1 != 0.f;
          overflow |= (put0 && !(fabsf(v0) < kForceLimitF)) || (put1 && !(fabsf(v1) < kForceLimitF));
          red_add_if(put0, f0 + js, fix_f(-v0));
          red_add_if(put1, f1 + js, fix_f(-v1));
        }
        __syncwarp();
      }
      // i forces of the pass: the lane's two units, then the eight lanes of
      // each i atom
      float fix = fi_x.x + fi_x.y, fiy = fi_y.x + fi_y.y, fiz = fi_z.x + fi_z.y;
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        fix += __shfl_xor_sync(0xffffffffu, fix, o);
        fiy += __shfl_xor_sync(0xffffffffu, fiy, o);
        fiz += __shfl_xor_sync(0xffffffffu, fiz, o);
      }
      if (p == 0 && k < 3) {
        const float v = (k == 0) ? fix : (k == 1 ? fiy : fiz);
        if (v != 0.f) {
          overflow |= !(fabsf(v) < kForceLimitF);
          red_add(facc + (size_t)k * fstride + islot, fix_f(v));
        }
      }
      Ec += fix_e((double)ec.x + (double)ec.y);
      Ev += fix_e(((double)ev6.x + (double)ev6.y) * (-1.0 / 6.0));
      Vc += fix_e(-((double)gs.x + (double)gs.y));
      Vv += fix_e((double)hs.x + (double)hs.y);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Ec += __shfl_xor_sync(0xffffffffu, Ec, o);
    Ev += __shfl_xor_sync(0xffffffffu, Ev, o);
    Vc += __shfl_xor_sync(0xffffffffu, Vc, o);
    Vv += __shfl_xor_sync(0xffffffffu, Vv, o);
    npair += __shfl_xor_sync(0xffffffffu, npair, o);
  }
  if (__any_sync(0xffffffffu, overflow) && lane == 0) raise_flag(acc, FLAG_OVERFLOW);
  if (lane == 0) {
    red_add(acc + ACC_E_DIR, Ec);
    red_add(acc + ACC_E_VDW, Ev);
    red_add(acc + ACC_V_DIR, Vc);
    red_add(acc + ACC_V_VDW, Vv);
    if (EXACT) {
      if (gw == 0) red_add(acc + ACC_NPAIR, counters[4]);
    } else {
      red_add(acc + ACC_NPAIR, (long long)npair);
    }
  }
}

constexpr int kChunk = 8;    // entries per filter/compute chunk
constexpr int kCWarps = 4;   // warps per block

struct CompactWarp {
  int ej[kChunk];
  uint2 em[kChunk];                                   // list masks per entry
  uint2 inm[kChunk];                                  // in-cut-off bits per entry
  float4 es[kChunk];                                  // FP32 shift per entry
  float4 xs[kChunk * kClusterSize];                   // staged j atoms
  float2 ls[kChunk * kClusterSize];                   // staged j LJ parameters
  unsigned char qlj[kClusterSize][kChunk * kClusterSize];  // per-i-atom queues
  unsigned char qn[kClusterSize][kChunk * kClusterSize];
  float4 fst[kChunk * kClusterSize][kClusterSize];    // force of pair (j key, i atom)
};

template <bool VDW>
__global__ void __launch_bounds__(kCWarps * 32, 5)
k_pair_fp32c(const long long *__restrict__ counters, const int4 *__restrict__ items,
             const CPairEntry *__restrict__ entries, const uint2 *__restrict__ masks,
             const float4 *__restrict__ xq, const float2 *__restrict__ lj, PairConstF c,
             long long *__restrict__ facc, int fstride, long long *__restrict__ acc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CompactWarp &W = reinterpret_cast<CompactWarp *>(smem_raw)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, q = lane >> 3;
  const unsigned gmask = 0x01010101u << il;
  const unsigned lt = (1u << lane) - 1u;
  const long long nItems = counters[1];
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long Ec = 0, Ev = 0, Vc = 0, Vv = 0, npair = 0;
  bool overflow = false;

  for (long long it = gw; it < nItems; it += nw) {
    const int4 item = items[it];
    const int ci = item.x, e0 = item.y, ne = item.z;
    const float4 xi = xq[ci * kClusterSize + il];
    const float2 li = lj[ci * kClusterSize + il];
    const bool iHasLJ = li.x != 0.f;
    float fix = 0.f, fiy = 0.f, fiz = 0.f;
    float ec = 0.f, ev = 0.f, vc = 0.f, vv = 0.f;
    for (int c0 = 0; c0 < ne; c0 += kChunk) {
      const int nEnt = min(kChunk, ne - c0);
      // ---- stage the chunk's entries and j atoms in shared memory ----------
      if (lane < nEnt) {
        const CPairEntry en = entries[e0 + c0 + lane];
        W.ej[lane] = en.j;
        W.es[lane] = make_float4(en.sx, en.sy, en.sz, 0.f);
        W.em[lane] = masks[e0 + c0 + lane];
      }
      __syncwarp();
      for (int a = lane; a < nEnt * kClusterSize; a += 32) {
        const int slot = W.ej[a >> 3] * kClusterSize + (a & 7);
        W.xs[a] = xq[slot];
        W.ls[a] = lj[slot];
      }
      __syncwarp();
      // ---- filter ---------------------------------------------------------
      int nLJ = 0, nN = 0;
      for (int e = 0; e < nEnt; ++e) {
        const float4 esh = W.es[e];
        const uint2 mk = W.em[e];
        const float4 xa = W.xs[e * kClusterSize + q];
        const float4 xb = W.xs[e * kClusterSize + q + 4];
        const float la = W.ls[e * kClusterSize + q].x;
        const float lb = W.ls[e * kClusterSize + q + 4].x;
        const float sx = esh.x - xi.x, sy = esh.y - xi.y, sz = esh.z - xi.z;
        const float ax = xa.x + sx, ay = xa.y + sy, az = xa.z + sz;
        const float bx = xb.x + sx, by = xb.y + sy, bz = xb.z + sz;
        const bool ina = ((mk.x >> lane) & 1u) && (fmaf(ax, ax, fmaf(ay, ay, az * az)) <= c.rc2);
        const bool inb = ((mk.y >> lane) & 1u) && (fmaf(bx, bx, fmaf(by, by, bz * bz)) <= c.rc2);
        const unsigned ba = __ballot_sync(0xffffffffu, ina);
        const unsigned bb = __ballot_sync(0xffffffffu, inb);
        if (lane == 0) W.inm[e] = make_uint2(ba, bb);
        const bool lja = VDW && iHasLJ && (la != 0.f);
        const bool ljb = VDW && iHasLJ && (lb != 0.f);
        const unsigned char ka = (unsigned char)(e * kClusterSize + q);
        const unsigned char kb = (unsigned char)(e * kClusterSize + q + 4);
        unsigned m = __ballot_sync(0xffffffffu, ina && lja) & gmask;
        if (ina && lja) W.qlj[il][nLJ + __popc(m & lt)] = ka;
        nLJ += __popc(m);
        m = __ballot_sync(0xffffffffu, inb && ljb) & gmask;
        if (inb && ljb) W.qlj[il][nLJ + __popc(m & lt)] = kb;
        nLJ += __popc(m);
        m = __ballot_sync(0xffffffffu, ina && !lja) & gmask;
        if (ina && !lja) W.qn[il][nN + __popc(m & lt)] = ka;
        nN += __popc(m);
        m = __ballot_sync(0xffffffffu, inb && !ljb) & gmask;
        if (inb && !ljb) W.qn[il][nN + __popc(m & lt)] = kb;
        nN += __popc(m);
      }
      __syncwarp();
      const int nTot = nLJ + nN;
      if (q == 0) npair += nTot;
      const int R = (int)__reduce_max_sync(0xffffffffu, (unsigned)((nTot + 3) >> 2));
      const int RL = (int)__reduce_max_sync(0xffffffffu, (unsigned)((nLJ + 3) >> 2));
      // ---- compute ----------------------------------------------------------
      for (int r = 0; r < R; ++r) {
        const int kq = 4 * r + q;
        const bool active = kq < nTot;
        int key = 0;
        if (active) key = (kq < nLJ) ? W.qlj[il][kq] : W.qn[il][kq - nLJ];
        const float4 sh = W.es[key >> 3];
        const float4 xj = W.xs[key];
        const float dx = xj.x + (sh.x - xi.x), dy = xj.y + (sh.y - xi.y),
                    dz = xj.z + (sh.z - xi.z);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float r2s = active ? r2 : 1.0f;
        const float rinv = rsqrt_approx(r2s);
        const float rr = r2s * rinv;
        const float qq = active ? xi.w * xj.w : 0.f;
        const float t = rcp_approx(fmaf(c.p_alpha, rr, 1.0f));
        const float ex = ex2_approx(-c.c_ex * r2s);
        float poly = fmaf(kErfcC7, t, kErfcC6);
        poly = fmaf(poly, t, kErfcC5);
        poly = fmaf(poly, t, kErfcC4);
        poly = fmaf(poly, t, kErfcC3);
        poly = fmaf(poly, t, kErfcC2);
        poly = fmaf(poly, t, kErfcC1);
        poly = fmaf(poly, t, kErfcC0);
        const float e_c = qq * rinv * (t * poly * ex);
        const float de_c = -fmaf(qq * c.two_a_sqrtpi, ex, e_c) * rinv;
        ec += e_c;
        vc = fmaf(de_c, rr, vc);
        float F = de_c;
        if (VDW && r < RL) {
          const float2 ljj = W.ls[key];
          const float eps = active ? li.x * ljj.x : 0.f;
          const float sg = (li.y + ljj.y) * rinv;
          const float s2 = sg * sg;
          const float s6 = s2 * s2 * s2;
          const float s12 = s6 * s6;
          const float pv = eps * (s12 - s6);
          const float dpv = eps * fmaf(-12.f, s12, 6.f * s6);
          const bool sw = r2s > c.ron2;
          const float s1 = c.rc2 - r2s;
          const float S = sw ? s1 * s1 * fmaf(c.sw_a, r2s, c.sw_b) : 1.f;
          const float dS = sw ? c.sw_c * r2s * s1 * (c.ron2 - r2s) : 0.f;
          const float de_v = fmaf(pv, dS, dpv * S) * rinv;
          ev = fmaf(pv, S, ev);
          vv = fmaf(de_v, rr, vv);
          F += de_v;
        }
        F *= rinv;
        const float fx = F * dx, fy = F * dy, fz = F * dz;
        fix += fx;
        fiy += fy;
        fiz += fz;
        if (active) W.fst[key][il] = make_float4(fx, fy, fz, 0.f);
      }
      __syncwarp();
      // ---- j forces: sum the stored pair forces of each j atom in i order ----
      for (int key = lane; key < nEnt * kClusterSize; key += 32) {
        const int e = key >> 3, jl = key & 7;
        const uint2 im = W.inm[e];
        const unsigned row = ((jl < 4) ? (im.x >> (8 * jl)) : (im.y >> (8 * (jl - 4)))) & 0xffu;
        if (row == 0u) continue;
        float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
        for (int ii = 0; ii < kClusterSize; ++ii) {
          if ((row >> ii) & 1u) {
            const float4 f = W.fst[key][ii];
            sx += f.x;
            sy += f.y;
            sz += f.z;
          }
        }
        overflow |= !(fabsf(sx) < kForceLimitF && fabsf(sy) < kForceLimitF &&
                      fabsf(sz) < kForceLimitF);
        const int slot = W.ej[e] * kClusterSize + jl;
        red_add(facc + slot, fix_f(-sx));
        red_add(facc + (size_t)fstride + slot, fix_f(-sy));
        red_add(facc + 2 * (size_t)fstride + slot, fix_f(-sz));
      }
      __syncwarp();
    }
    // i forces: sum over the four lanes of each i atom
    fix += __shfl_xor_sync(0xffffffffu, fix, 8);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 8);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 8);
    fix += __shfl_xor_sync(0xffffffffu, fix, 16);
    fiy += __shfl_xor_sync(0xffffffffu, fiy, 16);
    fiz += __shfl_xor_sync(0xffffffffu, fiz, 16);
    if (q < 3) {
      const float v = (q == 0) ? fix : (q == 1 ? fiy : fiz);
      if (v != 0.f) {
        overflow |= !(fabsf(v) < kForceLimitF);
        red_add(facc + (size_t)q * fstride + ci * kClusterSize + il, fix_f(v));
      }
    }
    Ec += fix_e(warp_sum_d((double)ec));
    Ev += fix_e(warp_sum_d((double)ev));
    Vc += fix_e(warp_sum_d((double)vc));
    Vv += fix_e(warp_sum_d((double)vv));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) npair += __shfl_xor_sync(0xffffffffu, npair, o);
  if (__any_sync(0xffffffffu, overflow) && lane == 0) raise_flag(acc, FLAG_OVERFLOW);
  if (lane == 0) {
    red_add(acc + ACC_E_DIR, Ec);
    red_add(acc + ACC_E_VDW, Ev);
    red_add(acc + ACC_V_DIR, Vc);
    red_add(acc + ACC_V_VDW, Vv);
    red_add(acc + ACC_NPAIR, npair);
  }
}

// Exclusion correction in FP64 (src/energy.c:567-621, ewald_corr
// src/ewald.c:371-384) into the fixed-point accumulators.
__global__ void __launch_bounds__(128)
k_excl_fix(int n, const DevBox *__restrict__ boxes, const int *__restrict__ atomRep,
           PairParams p, const int *__restrict__ exclStart,
           const int *__restrict__ exclFlat, const double *__restrict__ x,
           const double *__restrict__ y, const double *__restrict__ z,
           const double *__restrict__ q, const int *__restrict__ slotOf,
           long long *__restrict__ facc, int fstride, long long *__restrict__ acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  long long ecorr = 0, vcorr = 0;
  if (i < n) {
    const DevBox &b = boxes[atomRep ? atomRep[i] : 0];
    const int e = exclStart[i + 1];
    const int si = slotOf[i];
    for (int k = exclStart[i]; k < e; ++k) {
      const int j = exclFlat[k];
      if (j <= i) continue;
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      const double r2 = dist_d(b, dx, dy, dz);
      const double r = sqrt(r2);
      const double rt = 1. / r;
      const double qel = p.chargeConst * q[i] * q[j];
      const double alphar = p.alpha * r;
      const double eC = -qel * erf(alphar) * rt;
      double dE = 2.0 * qel * p.alpha * exp(-(alphar * alphar)) / kSqrtPi;
      dE = -(eC + dE) * rt;
      // every pair term goes to fixed point on its own (order independence)
      ecorr += fix_e(eC);
      vcorr += fix_e(dE * r);
      const long long fxj = fix_fd(dE * dx * rt), fyj = fix_fd(dE * dy * rt),
                      fzj = fix_fd(dE * dz * rt);
      const int sj = slotOf[j];
      red_add(facc + si, fxj);
      red_add(facc + (size_t)fstride + si, fyj);
      red_add(facc + 2 * (size_t)fstride + si, fzj);
      red_add(facc + sj, -fxj);
      red_add(facc + (size_t)fstride + sj, -fyj);
      red_add(facc + 2 * (size_t)fstride + sj, -fzj);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ecorr += __shfl_xor_sync(0xffffffffu, ecorr, o);
    vcorr += __shfl_xor_sync(0xffffffffu, vcorr, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red_add(acc + ACC_E_CORR, ecorr);
    red_add(acc + ACC_V_CORR, vcorr);
  }
}

// Fixed-point forces (slot order) -> FP64 forces (atom order); accumulate
// (+=) when add != 0, as MDBas's energy routines do.
__global__ void k_forces_out(int n, const int *__restrict__ slotOf,
                             const long long *__restrict__ facc, int fstride, int add,
                             double *__restrict__ fx, double *__restrict__ fy,
                             double *__restrict__ fz) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int s = slotOf[a];
  const double inv = 1.0 / kForceScale;
  const double vx = (double)facc[s] * inv;
  const double vy = (double)facc[(size_t)fstride + s] * inv;
  const double vz = (double)facc[2 * (size_t)fstride + s] * inv;
  if (add) {
    fx[a] += vx;
    fy[a] += vy;
    fz[a] += vz;
  } else {
    fx[a] = vx;
    fy[a] = vy;
    fz[a] = vz;
  }
}

}  // namespace

PairConstF make_pair_const(const PairParams &p) {
  PairConstF c;
  c.rc2 = (float)p.cutOff2;
  c.ron2 = (float)p.cutOn2;
  c.p_alpha = (float)(kErfcP * p.alpha);
  c.c_ex = (float)(p.alpha * p.alpha * 1.4426950408889634);
  c.two_a_sqrtpi = (float)(2.0 * p.alpha / kSqrtPi);
  c.sw_a = (float)(2.0 * p.switch2);
  c.sw_b = (float)((p.cutOff2 - 3.0 * p.cutOn2) * p.switch2);
  c.sw_c = (float)(12.0 * p.switch2);
  const double D = p.cutOff2 - p.cutOn2;
  c.sw_d = (float)D;
  c.sw_3d = (float)(3.0 * D);
  c.sw_6 = (float)(6.0 * p.switch2);
  c.sw_m12 = (float)(-12.0 * p.switch2);
  c.vdw = p.vdwSwitch;
  return c;
}

int pair_fp32_launch(ClusterWork &w, const PairParams &p, int grid, int block, cudaStream_t s,
                     int variant) {
  const PairConstF c = make_pair_const(p);
  // the list the kernel walks: the built list or, during dynamics, its
  // pruned inner copy
  if (variant == kPairQuad && w.useInner) {
    // the inner list written by the search at the kernel's own rc^2 (exact)
    // or a pruned one at rc + buffer; fixed blocks of kQWarps warps, the
    // same number of warps as grid x block
    const bool ex = w.innerRin2 == c.rc2 && w.rin2 == 0.f;
    auto kv = p.vdwSwitch ? (ex ? k_pair_quad<true, true> : k_pair_quad<true, false>)
                          : (ex ? k_pair_quad<false, true> : k_pair_quad<false, false>);
    const int qgrid = std::max(1, grid * block / (kQWarps * 32));
    MDB_LAUNCH(kv, qgrid, kQWarps * 32, 0, s, w.countersIn.as<long long>(),
               w.itemsIn.as<int4>(), w.entriesIn.as<HalfEntry>(), w.masksIn.as<unsigned>(),
               w.xq.as<float4>(), w.lj.as<float2>(), c, w.facc.as<long long>(), w.slotCap,
               w.acc.as<long long>());
    return MDBAS_NB_OK;
  }
  if (variant == kPairHalf || variant == kPairHalf3 || variant == kPairQuad ||
      variant == kPairHalfLean) {
    const bool in = w.useInner;
    // the inner list written by the search at the kernel's own rc^2
    const bool ex = in && w.innerRin2 == make_pair_const(p).rc2 && w.rin2 == 0.f;
    auto kv = p.vdwSwitch ? k_pair_half<true, false, 4, false> : k_pair_half<false, false, 4, false>;
    if (variant == kPairHalf3) {
      if (in && ex)
        kv = p.vdwSwitch ? k_pair_half<true, true, 3, true> : k_pair_half<false, true, 3, true>;
      else if (in)
        kv = p.vdwSwitch ? k_pair_half<true, true, 3, false> : k_pair_half<false, true, 3, false>;
      else
        kv = p.vdwSwitch ? k_pair_half<true, false, 3, false> : k_pair_half<false, false, 3, false>;
    } else if (variant == kPairHalfLean) {
      kv = !in ? (p.vdwSwitch ? k_pair_half_lean<true, false, false> : k_pair_half_lean<false, false, false>)
         : ex  ? (p.vdwSwitch ? k_pair_half_lean<true, true, true> : k_pair_half_lean<false, true, true>)
               : (p.vdwSwitch ? k_pair_half_lean<true, true, false> : k_pair_half_lean<false, true, false>);
    } else if (in && ex) {
      kv = p.vdwSwitch ? k_pair_half<true, true, 4, true> : k_pair_half<false, true, 4, true>;
    } else if (in) {
      kv = p.vdwSwitch ? k_pair_half<true, true, 4, false> : k_pair_half<false, true, 4, false>;
    }
    const DBuf &counters = in ? w.countersIn : w.counters;
    const DBuf &items = in ? w.itemsIn : w.items;
    const DBuf &entries = in ? w.entriesIn : w.entries;
    const DBuf &masks = in ? w.masksIn : w.masks;
    MDB_LAUNCH(kv, grid, block, 0, s, counters.as<long long>(), items.as<int4>(), entries.p,
               masks.p, w.xq.as<float4>(), w.lj.as<float2>(), c, w.facc.as<long long>(),
               w.slotCap, w.acc.as<long long>());
    return MDBAS_NB_OK;
  }
  // the 8 x 8 kernels read the full list
  DBuf &counters = w.counters;
  DBuf &items = w.items;
  DBuf &entries = w.entries;
  DBuf &masks = w.masks;
  if (variant == kPairPacked) {
    auto kv = p.vdwSwitch ? k_pair_fp32x2<true> : k_pair_fp32x2<false>;
    MDB_LAUNCH(kv, grid, block, 0, s, counters.as<long long>(), items.as<int4>(),
               entries.as<CPairEntry>(), masks.as<uint2>(), w.xq.as<float4>(),
               w.lj.as<float2>(), w.xp.as<float4>(), w.ljp.as<float4>(), c,
               w.facc.as<long long>(), w.slotCap, w.acc.as<long long>());
    return MDBAS_NB_OK;
  }
  if (variant == kPairBulk) {
    auto kv = p.vdwSwitch ? k_pair_fp32x2_bulk<true> : k_pair_fp32x2_bulk<false>;
    MDB_LAUNCH(kv, grid, block, 0, s, counters.as<long long>(), items.as<int4>(),
               entries.as<CPairEntry>(), masks.as<uint2>(), w.xq.as<float4>(),
               w.lj.as<float2>(), w.xp.as<float4>(), w.ljp.as<float4>(), c,
               w.facc.as<long long>(), w.slotCap, w.acc.as<long long>());
    return MDBAS_NB_OK;
  }
  if (variant == kPairDense) {
    if (p.vdwSwitch)
      MDB_LAUNCH(k_pair_fp32<true>, grid, block, 0, s, counters.as<long long>(),
                 items.as<int4>(), entries.as<CPairEntry>(), masks.as<uint2>(),
                 w.xq.as<float4>(), w.lj.as<float2>(), c, w.facc.as<long long>(), w.slotCap,
                 w.acc.as<long long>());
    else
      MDB_LAUNCH(k_pair_fp32<false>, grid, block, 0, s, counters.as<long long>(),
                 items.as<int4>(), entries.as<CPairEntry>(), masks.as<uint2>(),
                 w.xq.as<float4>(), w.lj.as<float2>(), c, w.facc.as<long long>(), w.slotCap,
                 w.acc.as<long long>());
    return MDBAS_NB_OK;
  }
  // compacted variant: fixed block of kCWarps warps, dynamic shared memory
  const size_t smem = sizeof(CompactWarp) * kCWarps;
  static bool attr_set[64][2];
  int dev = 0;
  MDB_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !attr_set[dev][p.vdwSwitch ? 1 : 0]) {
    if (p.vdwSwitch)
      MDB_CUDA(cudaFuncSetAttribute(k_pair_fp32c<true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
      MDB_CUDA(cudaFuncSetAttribute(k_pair_fp32c<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set[dev][p.vdwSwitch ? 1 : 0] = true;
  }
  const int cgrid = grid * block / (kCWarps * 32);
  if (p.vdwSwitch)
    MDB_LAUNCH(k_pair_fp32c<true>, cgrid, kCWarps * 32, smem, s, counters.as<long long>(),
               items.as<int4>(), entries.as<CPairEntry>(), masks.as<uint2>(),
               w.xq.as<float4>(), w.lj.as<float2>(), c, w.facc.as<long long>(), w.slotCap,
               w.acc.as<long long>());
  else
    MDB_LAUNCH(k_pair_fp32c<false>, cgrid, kCWarps * 32, smem, s, counters.as<long long>(),
               items.as<int4>(), entries.as<CPairEntry>(), masks.as<uint2>(),
               w.xq.as<float4>(), w.lj.as<float2>(), c, w.facc.as<long long>(), w.slotCap,
               w.acc.as<long long>());
  return MDBAS_NB_OK;
}

int excl_fix_launch(ClusterWork &w, int n, const PairParams &p, const int *exclStart,
                    const int *exclFlat, const double *x, const double *y, const double *z,
                    const double *q, cudaStream_t s) {
  if (n <= 0) return MDBAS_NB_OK;
  MDB_LAUNCH(k_excl_fix, grid_for(n, 128), 128, 0, s, n, w.boxes.as<DevBox>(), w.atomRepDev(),
             p, exclStart, exclFlat, x, y, z, q,
             w.slotOf.as<int>(), w.facc.as<long long>(), w.slotCap, w.acc.as<long long>());
  return MDBAS_NB_OK;
}

int forces_out_launch(ClusterWork &w, int n, int add, double *fx, double *fy, double *fz,
                      cudaStream_t s) {
  if (n <= 0) return MDBAS_NB_OK;
  MDB_LAUNCH(k_forces_out, grid_for(n, 256), 256, 0, s, n, w.slotOf.as<int>(),
             w.facc.as<long long>(), w.slotCap, add, fx, fy, fz);
  return MDBAS_NB_OK;
}

}  // namespace mdbas
