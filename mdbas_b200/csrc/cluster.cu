// cluster.cu -- cell-sorted cluster layout and the cluster-pair list.
//
// Layout.  The box is cut into an x-y grid of cells ("columns") whose width
// makes 8 atoms at the system's density fill a roughly cubic volume.  Cells
// are numbered in Morton (Z-curve) order of their (cx, cy) indices, atoms are
// counting-sorted into cells and sorted by z inside each cell, and every run
// of 8 consecutive atoms of a cell is one cluster (a cell's last cluster is
// padded).  Each cluster keeps an FP64 origin (its bounding-box centre) and
// FP32 half extents; each atom slot keeps float4 (x,y,z relative to the
// cluster origin, q*sqrt(C)) and float2 (2*eps_i, sig_i).  Relative FP32
// coordinates keep ~1e-6 A resolution in any box size; the large part of
// every displacement (origin to origin, periodic shift included) is formed
// in FP64 once per cluster pair.
//
// Cluster-pair search ("cell sweep").  One warp per i cluster walks the
// cells within reach in x-y (periodic images as explicit shifts), lanes test
// 32 candidate j clusters at a time against the i bounding box for each
// z image, and a ballot + prefix count compacts the survivors into a
// per-warp buffer.  Newton's third law: each unordered cluster pair is kept
// once (j > i, or j == i with a positive or zero shift, the latter with only
// the upper triangle of atom pairs).  Buffers are flushed as work items of
// 32 entries; at flush the warp builds each entry's 64-bit interaction mask
// (pairs within the list radius at build time, padding, exclusions, frozen
// pairs, self-pair triangle) with two ballots and drops entries whose mask
// is empty.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cluster.cuh"
#include "list_ref.cuh"

namespace mdbas {

namespace {

constexpr int kSearchThreads = 128;
constexpr int kBufCap = 64;

__device__ __forceinline__ double wrap_pos(double v, double L, double invL) {
  return v - L * floor(v * invL + 0.5);
}

__global__ void k_col_bin(int n, const ClusterGeom *__restrict__ geoms,
                          const int *__restrict__ atomRep, const int *__restrict__ colOff,
                          const int *__restrict__ colRank, const double *__restrict__ x,
                          const double *__restrict__ y, const double *__restrict__ z,
                          int *__restrict__ atomCol, double *__restrict__ atomZ,
                          int *__restrict__ colCount, long long *__restrict__ counters) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned act = __ballot_sync(0xffffffffu, i < n);  // lanes that go on
  if (i >= n) return;
  const int rep = atomRep ? atomRep[i] : 0;
  const ClusterGeom &g = geoms[rep];
  double sx = x[i] / g.Lx + 0.5, sy = y[i] / g.Ly + 0.5, sz = z[i] / g.Lz + 0.5;
  if (!(isfinite(sx) && isfinite(sy) && isfinite(sz))) {
    atomicOr(reinterpret_cast<unsigned long long *>(counters + 2), (unsigned long long)CL_NONFINITE);
    sx = sy = sz = 0.5;
  }
  sx -= floor(sx);
  sy -= floor(sy);
  sz -= floor(sz);
  const int cx = min((int)(sx * g.ncx), g.ncx - 1);
  const int cy = min((int)(sy * g.ncy), g.ncy - 1);
  const int col = colRank[colOff[rep] + cy * g.ncx + cx];
  atomCol[i] = col;
  atomZ[i] = sz;
  // one atomic per column among the warp's atoms (neighbouring atoms of a
  // molecule-ordered system mostly share a column)
  const unsigned same = __match_any_sync(act, col);
  if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(colCount + col, __popc(same));
}

// Column offsets in one block of 1,024 threads (the grid has at most a few
// tens of thousands of columns): colStart = exclusive scan of the atom
// counts, colPadStart = exclusive scan of the counts padded to whole
// clusters, colClStart = colPadStart / 8, each with its total at index nCols.
// One launch instead of two multi-kernel scans and two small kernels.
__global__ void __launch_bounds__(1024)
k_col_scan(int nCols, const int *__restrict__ colCount, int *__restrict__ colStart,
           int *__restrict__ colPadStart, int *__restrict__ colClStart) {
  __shared__ int wsum[2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int run0 = 0, run1 = 0;  // totals of the chunks before this one
  for (int c0 = 0; c0 < nCols; c0 += 1024) {
    const int c = c0 + threadIdx.x;
    const int v0 = c < nCols ? colCount[c] : 0;
    const int v1 = (v0 + kClusterSize - 1) & ~(kClusterSize - 1);
    int x0 = v0, x1 = v1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y0 = __shfl_up_sync(0xffffffffu, x0, o);
      const int y1 = __shfl_up_sync(0xffffffffu, x1, o);
      if (lane >= o) {
        x0 += y0;
        x1 += y1;
      }
    }
    if (lane == 31) {
      wsum[0][warp] = x0;
      wsum[1][warp] = x1;
    }
    __syncthreads();
    if (warp == 0) {
      int t0 = wsum[0][lane], t1 = wsum[1][lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y0 = __shfl_up_sync(0xffffffffu, t0, o);
        const int y1 = __shfl_up_sync(0xffffffffu, t1, o);
        if (lane >= o) {
          t0 += y0;
          t1 += y1;
        }
      }
      wsum[0][lane] = t0;
      wsum[1][lane] = t1;
    }
    __syncthreads();
    const int e0 = run0 + x0 - v0 + (warp > 0 ? wsum[0][warp - 1] : 0);
    const int e1 = run1 + x1 - v1 + (warp > 0 ? wsum[1][warp - 1] : 0);
    if (c < nCols) {
      colStart[c] = e0;
      colPadStart[c] = e1;
      colClStart[c] = e1 / kClusterSize;
    }
    run0 += wsum[0][31];
    run1 += wsum[1][31];
    __syncthreads();  // wsum is rewritten by the next chunk
  }
  if (threadIdx.x == 0) {
    colStart[nCols] = run0;
    colPadStart[nCols] = run1;
    colClStart[nCols] = run1 / kClusterSize;
  }
}

// The build's counters and per-column tallies cleared in one launch (instead
// of a memset each): column atom counts and fill cursors, the search's
// counters of both lists, the largest half extents per replica.
__global__ void __launch_bounds__(256)
k_build_reset(int nCols, int nRep, int *__restrict__ colCount, int *__restrict__ colFill,
              long long *__restrict__ counters, long long *__restrict__ countersIn,
              int *__restrict__ hmax) {
  for (int i = threadIdx.x; i <= nCols; i += blockDim.x) {
    colCount[i] = 0;
    colFill[i] = 0;
  }
  if (threadIdx.x < 8) {
    counters[threadIdx.x] = 0;
    countersIn[threadIdx.x] = 0;
  }
  for (int i = threadIdx.x; i < 4 * nRep; i += blockDim.x) hmax[i] = 0;
}

__global__ void k_col_scatter(int n, const int *__restrict__ atomCol,
                              const int *__restrict__ colStart, int *__restrict__ colFill,
                              int *__restrict__ tmpIdx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned act = __ballot_sync(0xffffffffu, i < n);  // lanes that go on
  if (i >= n) return;
  const int c = atomCol[i];
  // one atomic per column among the warp's atoms; lanes take consecutive
  // places in lane order (the column sort fixes the final order anyway)
  const unsigned same = __match_any_sync(act, c);
  const int lane = threadIdx.x & 31, leader = __ffs(same) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(colFill + c, __popc(same));
  base = __shfl_sync(same, base, leader);
  tmpIdx[colStart[c] + base + __popc(same & ((1u << lane) - 1u))] = i;
}

// One column per block: its atoms in ascending (z, atom index) order into
// the column's slots, padding slots set to -1.  Columns of up to 1,024 atoms
// are sorted by a bitonic network over 256, 512 or 1,024 keys (padded with
// +inf) held in registers, R = 1, 2 or 4 per thread (element t + 256 r):
// partners within a warp are exchanged by shuffles, partners in another warp
// through shared memory, partners in the same thread directly.  Longer
// columns are sorted by rank counting.  Both give the same total order, so
// the same slots.
__device__ __forceinline__ bool key_less(double za, int ia, double zb, int ib) {
  return za < zb || (za == zb && ia < ib);
}
template <int R>
__device__ __forceinline__ void col_bitonic(double (&key)[R], int (&idx)[R], double *xz, int *xi) {
  constexpr int P = 256 * R;
  const int t = threadIdx.x;
  // fully unrolled: every partner index below is a constant, so the keys stay
  // in registers
#pragma unroll
  for (int k = 2; k <= P; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 256) {
        const int rj = j >> 8;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int rp = r ^ rj;
          if (rp > r) {
            // element t + 256 r is the lower of the pair
            const bool asc = ((t + 256 * r) & k) == 0;
            if (key_less(key[rp], idx[rp], key[r], idx[r]) == asc) {
              const double kz = key[r];
              const int ki = idx[r];
              key[r] = key[rp];
              idx[r] = idx[rp];
              key[rp] = kz;
              idx[rp] = ki;
            }
          }
        }
      } else {
        double pz[R];
        int pi[R];
        if (j >= 32) {
          __syncthreads();  // the previous exchange's reads are done
#pragma unroll
          for (int r = 0; r < R; ++r) {
            xz[t + 256 * r] = key[r];
            xi[t + 256 * r] = idx[r];
          }
          __syncthreads();
#pragma unroll
          for (int r = 0; r < R; ++r) {
            pz[r] = xz[(t + 256 * r) ^ j];
            pi[r] = xi[(t + 256 * r) ^ j];
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            pz[r] = __shfl_xor_sync(0xffffffffu, key[r], j);
            pi[r] = __shfl_xor_sync(0xffffffffu, idx[r], j);
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int e = t + 256 * r;
          // the lower element of an ascending pair keeps the smaller key, the
          // upper one the larger; a descending pair the other way round
          const bool wantMin = ((e & j) == 0) == ((e & k) == 0);
          const bool take = wantMin ? key_less(pz[r], pi[r], key[r], idx[r])
                                    : key_less(key[r], idx[r], pz[r], pi[r]);
          if (take) {
            key[r] = pz[r];
            idx[r] = pi[r];
          }
        }
      }
    }
  }
}
template <int R>
__device__ __forceinline__ void col_sort_small(int n, int s, int ps, const int *__restrict__ tmpIdx,
                                               const double *__restrict__ atomZ,
                                               int *__restrict__ slotAtom, double *xz, int *xi) {
  double key[R];
  int idx[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int e = threadIdx.x + 256 * r;
    if (e < n) {
      idx[r] = tmpIdx[s + e];
      key[r] = atomZ[idx[r]];
    } else {
      idx[r] = 0x7fffffff;
      key[r] = __longlong_as_double(0x7ff0000000000000LL);  // +inf
    }
  }
  col_bitonic<R>(key, idx, xz, xi);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int e = threadIdx.x + 256 * r;
    if (e < n) slotAtom[ps + e] = idx[r];
  }
}

__global__ void __launch_bounds__(256)
k_col_sort(int nCols, const int *__restrict__ colStart,
           const int *__restrict__ colPadStart, const int *__restrict__ tmpIdx,
           const double *__restrict__ atomZ, int *__restrict__ slotAtom) {
  constexpr int kMax = 1024;
  __shared__ double sz[kMax];
  __shared__ int si[kMax];
  const int c = blockIdx.x;
  if (c >= nCols) return;
  const int s = colStart[c], e = colStart[c + 1];
  const int ps = colPadStart[c], pe = colPadStart[c + 1];
  const int n = e - s;
  if (n <= 256) {
    col_sort_small<1>(n, s, ps, tmpIdx, atomZ, slotAtom, sz, si);
  } else if (n <= 512) {
    col_sort_small<2>(n, s, ps, tmpIdx, atomZ, slotAtom, sz, si);
  } else if (n <= kMax) {
    col_sort_small<4>(n, s, ps, tmpIdx, atomZ, slotAtom, sz, si);
  } else {
    for (int base = s; base < e; base += blockDim.x) {
      const int m = base + threadIdx.x;
      const int mi = (m < e) ? tmpIdx[m] : 0;
      const double mz = (m < e) ? atomZ[mi] : 0.0;
      int rank = 0;
      for (int cb = s; cb < e; cb += kMax) {
        const int cnt = min(kMax, e - cb);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
          const int a = tmpIdx[cb + t];
          si[t] = a;
          sz[t] = atomZ[a];
        }
        __syncthreads();
        if (m < e) {
          // four independent counts: the comparisons do not wait on each other
          int r0 = 0, r1 = 0, r2 = 0, r3 = 0, t = 0;
          for (; t + 3 < cnt; t += 4) {
            r0 += (sz[t] < mz) || (sz[t] == mz && si[t] < mi);
            r1 += (sz[t + 1] < mz) || (sz[t + 1] == mz && si[t + 1] < mi);
            r2 += (sz[t + 2] < mz) || (sz[t + 2] == mz && si[t + 2] < mi);
            r3 += (sz[t + 3] < mz) || (sz[t + 3] == mz && si[t + 3] < mi);
          }
          for (; t < cnt; ++t) r0 += (sz[t] < mz) || (sz[t] == mz && si[t] < mi);
          rank += (r0 + r1) + (r2 + r3);
        }
      }
      if (m < e) slotAtom[ps + rank] = mi;
    }
  }
  for (int p = ps + n + threadIdx.x; p < pe; p += blockDim.x) slotAtom[p] = -1;
}

// One thread per slot, 8 consecutive lanes per cluster: FP64 origin and half
// extents (min/max over the cluster's lanes by shuffles), slot data.
__device__ __forceinline__ double grp_min8(double v) {
#pragma unroll
  for (int o = 1; o < kClusterSize; o <<= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double grp_max8(double v) {
#pragma unroll
  for (int o = 1; o < kClusterSize; o <<= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void k_clusters(const int *__restrict__ nSlotsDev,
                           const ClusterGeom *__restrict__ geoms,
                           const int *__restrict__ atomRep, int *__restrict__ clusterRep,
                           const int *__restrict__ slotAtom,
                           const int *__restrict__ atomCol, const int *__restrict__ colXY,
                           const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, const double *__restrict__ q,
                           const double *__restrict__ eps, const double *__restrict__ sig,
                           double sqrtC, double4 *__restrict__ origin,
                           float4 *__restrict__ originF, float4 *__restrict__ half,
                           float4 *__restrict__ xq, float2 *__restrict__ lj,
                           float *__restrict__ xp, float *__restrict__ ljp,
                           int *__restrict__ slotOf, int *__restrict__ clusterXY,
                           int *__restrict__ hmaxBits) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // slot
  const int c = t / kClusterSize, k = t % kClusterSize;
  // every lane takes part in the shuffles; lanes past the last cluster only
  // do that (8-lane groups are whole clusters: blockDim is a multiple of 32)
  // the slot loads do not wait for the slot count: the grid covers slotCap
  // slots, all allocated (those past the count are not used)
  const bool active = c < (*nSlotsDev >> 3);
  // a cluster's first slot always holds an atom (columns are padded at the end)
  const int a0s = slotAtom[c * kClusterSize], as = slotAtom[t];
  const int a0 = active ? a0s : 0;
  const int rep = (active && atomRep) ? atomRep[a0] : 0;
  const ClusterGeom &g = geoms[rep];
  const int a = active ? as : -1;
  double px = 0., py = 0., pz = 0.;
  double lx = 1e300, ly = 1e300, lz = 1e300, hx = -1e300, hy = -1e300, hz = -1e300;
  if (a >= 0) {
    px = wrap_pos(x[a], g.Lx, g.invLx);
    py = wrap_pos(y[a], g.Ly, g.invLy);
    pz = wrap_pos(z[a], g.Lz, g.invLz);
    lx = hx = px;
    ly = hy = py;
    lz = hz = pz;
  }
  lx = grp_min8(lx);
  ly = grp_min8(ly);
  lz = grp_min8(lz);
  hx = grp_max8(hx);
  hy = grp_max8(hy);
  hz = grp_max8(hz);
  const int nreal = __popc(__ballot_sync(0xffffffffu, a >= 0) >> (threadIdx.x & 24) & 0xffu);
  const double ox = 0.5 * (lx + hx), oy = 0.5 * (ly + hy), oz = 0.5 * (lz + hz);
  // Half extents rounded up so that the FP32 box always contains its atoms;
  // w holds the number of real (non-padding) atoms.
  const float4 h = make_float4(__double2float_ru(0.5 * (hx - lx) * (1.0 + 1e-6) + 1e-6),
                               __double2float_ru(0.5 * (hy - ly) * (1.0 + 1e-6) + 1e-6),
                               __double2float_ru(0.5 * (hz - lz) * (1.0 + 1e-6) + 1e-6),
                               (float)nreal);
  // The largest half extents per box, one atomic per warp and dimension
  // when the warp's clusters share a box (non-negative floats order like
  // their bits); every lane is still present here.
  {
    const bool mine = active && k == 0;
    const int bx = mine ? __float_as_int(h.x) : 0, by = mine ? __float_as_int(h.y) : 0,
              bz = mine ? __float_as_int(h.z) : 0;
    const int rep0 = __shfl_sync(0xffffffffu, rep, 0);
    if (__all_sync(0xffffffffu, !active || rep == rep0)) {
      const int mx = __reduce_max_sync(0xffffffffu, bx), my = __reduce_max_sync(0xffffffffu, by),
                mz = __reduce_max_sync(0xffffffffu, bz);
      if ((threadIdx.x & 31) == 0 && active) {
        atomicMax(hmaxBits + 4 * rep0 + 0, mx);
        atomicMax(hmaxBits + 4 * rep0 + 1, my);
        atomicMax(hmaxBits + 4 * rep0 + 2, mz);
      }
    } else if (mine) {
      atomicMax(hmaxBits + 4 * rep + 0, bx);
      atomicMax(hmaxBits + 4 * rep + 1, by);
      atomicMax(hmaxBits + 4 * rep + 2, bz);
    }
  }
  if (!active) return;
  if (k == 0) {
    if (clusterRep) clusterRep[c] = rep;
    origin[c] = make_double4(ox, oy, oz, 0.0);
    originF[c] = make_float4((float)ox, (float)oy, (float)oz, (float)nreal);
    half[c] = h;
    clusterXY[c] = colXY[atomCol[a0]];
  }
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  float2 l = make_float2(0.f, 0.f);
  if (a >= 0) {
    v = make_float4((float)(px - ox), (float)(py - oy), (float)(pz - oz), (float)(q[a] * sqrtC));
    l = make_float2((float)(2.0 * eps[a]), (float)sig[a]);
    slotOf[a] = t;
  }
  xq[t] = v;
  lj[t] = l;
  float *p = xp + (size_t)(c * 4 + (k & 3)) * 8 + (k >> 2);
  p[0] = v.x;
  p[2] = v.y;
  p[4] = v.z;
  p[6] = v.w;
  float *m = ljp + (size_t)(c * 4 + (k & 3)) * 4 + (k >> 2);
  m[0] = l.x;
  m[2] = l.y;
}

constexpr int kExclRegs = 8;  // exclusion partners per atom kept in registers
constexpr int kSearchCols = 192;  // z-windowed ranges listed per warp before a candidate scan

// Per warp: the i cluster, the candidates found so far (with their FP32
// shifts) and the z-windowed column ranges of the current candidate scan.
struct WarpBuf {
  int j[kBufCap];
  int code[kBufCap];                   // image index (0..26) | real j atoms << 8
  uint2 mask[kItemMax];
  float4 sj[kClusterSize * kItemMax];  // staged j atoms (xq), sj[j * kItemMax + entry]
  float4 sn[kClusterSize];             // the i cluster's atoms, negated and paired:
  float2 snz[kClusterSize];            // (-x, -x, -y, -y) and (-z, -z)
  int ps[kClusterSize][kExclRegs];     // per i atom: its first exclusion partners' slots
  int es[kClusterSize], ee[kClusterSize];  // per i atom: its range of exclFlat
  int rstart[kSearchCols];             // first cluster of a z-windowed range
  int rcount[kSearchCols];
  int rcode[kSearchCols];              // (sx + 1) | (sy + 1) << 2 | (sz + 1) << 4
  int rpre[kSearchCols + 1];
  int tally[4];  // entries kept, inner halves, warp steps and pairs of the inner items
};

// Outputs of the search: the list (entries with 64-bit masks at the list
// radius, exactly MDBas's pairs) and the inner list (j-cluster halves with a
// pair within sqrt(rin2), 32-bit masks).
// Both lists take their room with one 64-bit atomic per flush on a packed
// counter (items << 40 | entries taken): counters[4]; the inner list uses the
// same item index and twice the entry index.  The search's last warp writes
// the readers' counts into counters[0..1] / hcounters[0..1].
constexpr int kPackShift = 40;
struct SearchOut {
  CPairEntry *entries;
  uint2 *masks;
  int4 *items;
  long long *counters;
  long long entryCap, itemCap;
  HalfEntry *hent;
  unsigned *hmask;
  int4 *hitems;
  long long *hcounters;
  float rin2;
  long long *sticky;  // a build that does not wait: the word the error bits are latched into
};

// MDBas's FP64 squared distance of atoms a and c, the expression of the list
// builder it would run (either order of the two atoms gives the same bits).
// listMode 1: link cells (src/list.c:1932-1936, 2051-2055): fractional
// coordinates + 0.5, their difference plus the cell wrap's shift (the one
// image within the list radius: the box holds at least three cells of that
// width), mapped back by the box rows.  listMode 0: dist() (src/utils.c:
// 38-80) of x[c] - x[a].
__device__ __noinline__ double mdbas_pair_r2(const DevBox &b, int listMode,
                                             const double *__restrict__ x,
                                             const double *__restrict__ y,
                                             const double *__restrict__ z, int a, int c) {
  if (listMode) {
    const double xa = dadd(dadd(dadd(dmul(x[a], b.u1), dmul(y[a], b.u2)), dmul(z[a], b.u3)), 0.5);
    const double ya = dadd(dadd(dadd(dmul(x[a], b.v1), dmul(y[a], b.v2)), dmul(z[a], b.v3)), 0.5);
    const double za = dadd(dadd(dadd(dmul(x[a], b.w1), dmul(y[a], b.w2)), dmul(z[a], b.w3)), 0.5);
    const double xc = dadd(dadd(dadd(dmul(x[c], b.u1), dmul(y[c], b.u2)), dmul(z[c], b.u3)), 0.5);
    const double yc = dadd(dadd(dadd(dmul(x[c], b.v1), dmul(y[c], b.v2)), dmul(z[c], b.v3)), 0.5);
    const double zc = dadd(dadd(dadd(dmul(x[c], b.w1), dmul(y[c], b.w2)), dmul(z[c], b.w3)), 0.5);
    double xt = dsub(xc, xa), yt = dsub(yc, ya), zt = dsub(zc, za);
    xt = dadd(xt, -rint(xt));
    yt = dadd(yt, -rint(yt));
    zt = dadd(zt, -rint(zt));
    const double xd = dadd(dadd(dmul(xt, b.a1), dmul(yt, b.b1)), dmul(zt, b.c1));
    const double yd = dadd(dadd(dmul(xt, b.a2), dmul(yt, b.b2)), dmul(zt, b.c2));
    const double zd = dadd(dadd(dmul(xt, b.a3), dmul(yt, b.b3)), dmul(zt, b.c3));
    return dadd(dadd(dmul(xd, xd), dmul(yd, yd)), dmul(zd, zd));
  }
  double dx = dsub(x[c], x[a]), dy = dsub(y[c], y[a]), dz = dsub(z[c], z[a]);
  return dist_d(b, dx, dy, dz);
}

// An asynchronous 16-byte copy from global into shared memory (completed by
// cp.async.wait_all).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}

// Shared-memory loads the compiler keeps where they are written (not hoisted
// out of a loop into registers that the loop would then hold throughout).
__device__ __forceinline__ float4 lds_keep(const float4 *p) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"((unsigned)__cvta_generic_to_shared(p))
               : "memory");
  return v;
}
__device__ __forceinline__ float2 lds_keep(const float2 *p) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];"
               : "=f"(v.x), "=f"(v.y)
               : "r"((unsigned)__cvta_generic_to_shared(p))
               : "memory");
  return v;
}

// Flush the first cnt (<= kItemMax) buffered candidates as one work item.
// Lane k builds candidate k's 64-bit interaction mask on its own: bit i + 8 j
// (j < 4 in .x, j >= 4 in .y at i + 8 (j - 4)) for the pair (i atom i, j atom
// j) within the list radius, both slots real, j > i on the cluster's own
// entry, not an exclusion (checked only when the j cluster lies in the range
// of clusters holding a partner of the i cluster's atoms: [pcLo, pcHi]) and
// not both frozen.  The FP32 distances are formed exactly as the pair kernel
// forms them (j atoms plus the entry's shift, minus the i atom), so the
// inner mask at the cut-off (rin2 = the kernel's FP32 rc^2) holds exactly the
// pairs the kernel would find inside it.  Pairs in the band around the list
// radius are settled by MDBas's FP64 expression, so the list's pairs are
// MDBas's.  The halves of the entries holding inner pairs become the item's
// inner-list entries, halves 0 first.
// Room: one 64-bit atomic per flush takes an item and cnt entries (an upper
// bound of the entries kept) before the mask pass, so its round trip overlaps
// the pass; the inner list's item has the same index and its halves sit at
// twice the entry index.  Entries not kept leave gaps, which no reader
// visits: every reader goes through the items.
__device__ void flush_item(WarpBuf &B, int cnt, int ci, int lane,
                           const float4 *__restrict__ xq, const ClusterGeom &g,
                           const DevBox &box, int nreal_i, int pcLo, int pcHi, unsigned fimask,
                           const int *__restrict__ exclFlat, const int *__restrict__ slotOf,
                           const int *__restrict__ slotAtom, const int *__restrict__ frozen,
                           const double *__restrict__ px, const double *__restrict__ py,
                           const double *__restrict__ pz,
                           const double4 *__restrict__ origin, const SearchOut &o) {
  unsigned long long pk = 0ull;
  if (lane == 0)
    pk = atomicAdd(reinterpret_cast<unsigned long long *>(o.counters + 4),
                   (1ull << kPackShift) | (unsigned long long)cnt);
  // the origins for this lane's entry shift, loaded with the staged atoms
  const double4 oi = origin[ci];
  double4 oj = make_double4(0., 0., 0., 0.);
  if (lane < cnt) oj = origin[B.j[lane]];
  // the j atoms straight into shared memory (asynchronous 16-byte copies:
  // no registers hold them in flight)
#pragma unroll
  for (int r = 0; r < kClusterSize; ++r) {
    const int idx = lane + 32 * r, k = idx >> 3, j = idx & 7;
    if (k < cnt)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(
                       (unsigned)__cvta_generic_to_shared(&B.sj[j * kItemMax + k])),
                   "l"(xq + (size_t)B.j[k] * kClusterSize + j)
                   : "memory");
  }
  // while the copies land: the entry's shift and its masks of padding slots,
  // the cluster's own triangle, exclusions and frozen pairs
  uint2 inner = make_uint2(0u, 0u);
  CPairEntry en{};
  int npin = 0, cj = 0, sidx = 0;
  unsigned m0 = 0u, m1 = 0u;
  if (lane < cnt) {
    const int code = B.code[lane];
    cj = B.j[lane];
    sidx = code & 31;
    const int nrj = code >> 8;
    // the entry's shift, formed in FP64 and rounded once: the value the pair
    // kernel adds to the j atoms
    const int sx = sidx % 3 - 1, sy = (sidx / 3) % 3 - 1, sz = sidx / 9 - 1;
    en.j = cj;
    en.sx = (float)(oj.x + sx * g.Lx - oi.x);
    en.sy = (float)(oj.y + sy * g.Ly - oi.y);
    en.sz = (float)(oj.z + sz * g.Lz - oi.z);
    // padding slots of either cluster
    const unsigned irow = (nreal_i >= 8 ? 0xffu : ((1u << nreal_i) - 1u)) * 0x01010101u;
    m0 = irow & (nrj >= 4 ? 0xffffffffu : ((1u << (8 * nrj)) - 1u));
    m1 = irow & (nrj >= 8 ? 0xffffffffu : (nrj <= 4 ? 0u : ((1u << (8 * (nrj - 4))) - 1u)));
    if (cj == ci && sidx == 13) {  // the cluster with itself: j > i
      m0 &= 0x07030100u;
      m1 &= 0x7f3f1f0fu;
    }
    if (cj >= pcLo && cj <= pcHi) {
      for (int i = 0; i < kClusterSize; ++i) {
        const int e0 = B.es[i], n = B.ee[i] - e0;
        for (int r = 0; r < n; ++r) {
          const int p = r < kExclRegs ? B.ps[i][r] : slotOf[__ldg(exclFlat + e0 + r)];
          if ((p >> 3) == cj) {
            const int j = p & 7;
            if (j < 4) m0 &= ~(1u << (i + 8 * j));
            else m1 &= ~(1u << (i + 8 * (j - 4)));
          }
        }
      }
    }
    if (frozen && fimask) {
      for (int j = 0; j < kClusterSize; ++j) {
        const int ja = slotAtom[cj * kClusterSize + j];
        if (ja >= 0 && frozen[ja]) {
          const unsigned m = fimask << (8 * (j & 3));
          if (j < 4) m0 &= ~m;
          else m1 &= ~m;
        }
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncwarp();
  if (lane < cnt) {
    const int k = lane;
    // Per pair the sign of (radius^2 - r^2), exact for the FP32 distance the
    // pair kernel forms (j atom plus the shift, minus the i atom), is shifted
    // into a word per radius and half: h from 3 down to 0, i from 7 down to
    // 0 leaves pair (i, h) at bit i + 8 h.  A set bit is a pair beyond the
    // radius; the words are inverted at the end.  Per radius: beyond the
    // band's lower edge (lo), beyond its upper edge (ca), beyond the inner
    // radius (in).
    const float2 rlo = make_float2(g.rlo2, g.rlo2), rhi = make_float2(g.rhi2, g.rhi2),
                 rin = make_float2(o.rin2, o.rin2);
    unsigned lo0 = 0u, lo1 = 0u, ca0 = 0u, ca1 = 0u, in0 = 0u, in1 = 0u;
#pragma unroll 1
    for (int h = 3; h >= 0; --h) {
      // the j atoms h and h + 4 side by side, shifted as the pair kernel does
      const float4 a = B.sj[h * kItemMax + k], b = B.sj[(h + 4) * kItemMax + k];
      const float2 jx = make_float2(a.x + en.sx, b.x + en.sx);
      const float2 jy = make_float2(a.y + en.sy, b.y + en.sy);
      const float2 jz = make_float2(a.z + en.sz, b.z + en.sz);
#pragma unroll
      for (int i = kClusterSize - 1; i >= 0; --i) {
        const float4 nxy = lds_keep(&B.sn[i]);
        const float2 dx = __fadd2_rn(jx, make_float2(nxy.x, nxy.y));
        const float2 dy = __fadd2_rn(jy, make_float2(nxy.z, nxy.w));
        const float2 dz = __fadd2_rn(jz, lds_keep(&B.snz[i]));
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        const float2 dl = __ffma2_rn(r2, make_float2(-1.f, -1.f), rlo);
        const float2 dc = __ffma2_rn(r2, make_float2(-1.f, -1.f), rhi);
        const float2 di = __ffma2_rn(r2, make_float2(-1.f, -1.f), rin);
        lo0 = __funnelshift_l(__float_as_uint(dl.x), lo0, 1);
        lo1 = __funnelshift_l(__float_as_uint(dl.y), lo1, 1);
        ca0 = __funnelshift_l(__float_as_uint(dc.x), ca0, 1);
        ca1 = __funnelshift_l(__float_as_uint(dc.y), ca1, 1);
        in0 = __funnelshift_l(__float_as_uint(di.x), in0, 1);
        in1 = __funnelshift_l(__float_as_uint(di.y), in1, 1);
      }
    }
    lo0 = ~lo0;
    lo1 = ~lo1;
    ca0 = ~ca0;
    ca1 = ~ca1;
    in0 = ~in0;
    in1 = ~in1;
    // pairs in the band: MDBas's own FP64 distance decides
    unsigned amb0 = ca0 & ~lo0 & m0, amb1 = ca1 & ~lo1 & m1;
    unsigned fin0 = lo0 & m0, fin1 = lo1 & m1;
    while (amb0 | amb1) {
      const bool second = amb0 == 0u;
      const unsigned v = second ? amb1 : amb0;
      const int b = __ffs(v) - 1;
      if (second) amb1 &= amb1 - 1u; else amb0 &= amb0 - 1u;
      const int i = b & 7, j = (b >> 3) + (second ? 4 : 0);
      const int a = slotAtom[ci * kClusterSize + i], c = slotAtom[cj * kClusterSize + j];
      if (mdbas_pair_r2(box, g.listMode, px, py, pz, a, c) <= g.cutnb2) {
        if (second) fin1 |= 1u << b; else fin0 |= 1u << b;
      }
    }
    B.mask[k] = make_uint2(fin0, fin1);
    inner = make_uint2(in0 & fin0, in1 & fin1);
    npin = __popc(inner.x) + __popc(inner.y);
  }
  __syncwarp();
  // keep the entries with at least one pair within the list radius
  const bool keep = lane < cnt && (B.mask[lane].x | B.mask[lane].y) != 0u;
  const unsigned km = __ballot_sync(0xffffffffu, keep);
  const int nkeep = __popc(km);
  const unsigned hA = __ballot_sync(0xffffffffu, inner.x != 0u);
  const unsigned hB = __ballot_sync(0xffffffffu, inner.y != 0u);
  const int nA = __popc(hA), nin = nA + __popc(hB);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) npin += __shfl_xor_sync(0xffffffffu, npin, off);
  pk = __shfl_sync(0xffffffffu, pk, 0);
  const long long e0 = (long long)(pk & ((1ull << kPackShift) - 1ull));
  const long long it = (long long)(pk >> kPackShift);
  if (e0 + cnt > o.entryCap || it >= o.itemCap) {
    if (lane == 0)
      atomicOr(reinterpret_cast<unsigned long long *>(o.counters + 2),
               (unsigned long long)CL_OVERFLOW);
    return;
  }
  if (lane == 0) {
    B.tally[0] += nkeep;
    B.tally[1] += nin;
    B.tally[2] += (nin + 1) >> 1;
    B.tally[3] += npin;
  }
  if (keep) {
    const int pos = __popc(km & ((1u << lane) - 1u));
    o.entries[e0 + pos] = en;
    o.masks[e0 + pos] = B.mask[lane];
    const unsigned lt = (1u << lane) - 1u;
    if (inner.x != 0u) {
      const long long q = 2 * e0 + __popc(hA & lt);
      HalfEntry he;
      he.jh = 2 * en.j;
      he.sx = en.sx;
      he.sy = en.sy;
      he.sz = en.sz;
      o.hent[q] = he;
      o.hmask[q] = inner.x;
    }
    if (inner.y != 0u) {
      const long long q = 2 * e0 + nA + __popc(hB & lt);
      HalfEntry he;
      he.jh = 2 * en.j + 1;
      he.sx = en.sx;
      he.sy = en.sy;
      he.sz = en.sz;
      o.hent[q] = he;
      o.hmask[q] = inner.y;
    }
  }
  // an item whose entries all fell out stays in the list, empty
  if (lane == 0) {
    o.items[it] = make_int4(ci, (int)e0, nkeep, 0);
    o.hitems[it] = make_int4(ci, (int)(2 * e0), nin, 0);
  }
}

// Per column, the first cluster (clusters are z-sorted in their column)
// whose FP32 origin z is at least -Lz/2 + b Lz / kZBins, for b = 0..kZBins
// (b = 0: the column's first cluster, b = kZBins: one past its last).  The
// search reads a z window's range from two entries of this table instead of
// two binary searches over the column; a conservative bin on either side
// keeps the range a superset, and the bounding-box test that follows drops
// the extra clusters.  The table is indexed by grid cell (colOff[r] + cy *
// ncx + cx, the index of colRank), so the search reads it without going
// through the column numbering.  One block per cell, one thread per bin,
// binary searches over the column's origins staged in shared memory.
__global__ void __launch_bounds__((kZBins + 32) & ~31)
k_col_ztab(int nCols, const ClusterGeom *__restrict__ geoms, const int *__restrict__ clusterRep,
           const int *__restrict__ colRank, const int *__restrict__ colClStart,
           const float4 *__restrict__ originF, int *__restrict__ zTab) {
  // the column's origin z in shared memory (one load each) when they fit
  constexpr int kStaged = 512;
  __shared__ float oz[kStaged];
  const int cell = blockIdx.x, b = threadIdx.x;
  if (cell >= nCols) return;
  const int col = colRank[cell];
  const int cs = colClStart[col], ce = colClStart[col + 1];
  const bool staged = ce - cs <= kStaged;
  if (staged)
    for (int k = threadIdx.x; k < ce - cs; k += blockDim.x) oz[k] = originF[cs + k].z;
  __syncthreads();
  if (b > kZBins) return;
  int a = cs;
  if (b == kZBins) {
    a = ce;
  } else if (b > 0 && ce > cs) {
    const float Lz = (float)geoms[clusterRep ? clusterRep[cs] : 0].Lz;
    const float zb = -0.5f * Lz + (float)b * (Lz / (float)kZBins);
    int hi = ce;
    while (a < hi) {  // first origin z >= zb
      const int mid = (a + hi) >> 1;
      if ((staged ? oz[mid - cs] : originF[mid].z) < zb) a = mid + 1; else hi = mid;
    }
  }
  zTab[(size_t)cell * (kZBins + 1) + b] = a;
}

// Cluster-pair search ("cell sweep"): one warp per i cluster.  The columns
// within reach in x-y (periodic images as explicit shifts) are listed, 32 at
// a time, with per z image within reach the clusters (z-sorted in their
// column) whose origin lies within the z reach left over the column's x-y
// gap, read from the column's z table (k_col_ztab); then all candidates of
// the listed ranges are tested against the i bounding box as one flat index
// space, 32 per round, so every lane has work and all loads of a round are
// independent.  Survivors are compacted by ballot into the warp's buffer
// with their image and flushed as work items of up to 32 entries (the flush
// forms each entry's FP32 shift: the FP64 origin difference plus the image,
// rounded once).  Newton's third law: each unordered cluster pair is kept
// once (j > i, or j == i with a positive or zero shift, the latter with only
// the upper triangle of atom pairs).
// (at most 96 registers and ~34 KB of shared memory per block: five blocks
// of four warps per SM)
__global__ void __launch_bounds__(kSearchThreads, 5)
k_search(const int *__restrict__ nSlotsDev, const ClusterGeom *__restrict__ geoms,
         const DevBox *__restrict__ boxes, const int *__restrict__ clusterRep,
         const int *__restrict__ colOff, const int *__restrict__ zTab,
         const int *__restrict__ clusterXY,
         const double4 *__restrict__ origin, const float4 *__restrict__ originF,
         const float4 *__restrict__ half, const int *__restrict__ slotAtom,
         const int *__restrict__ slotOf, const int *__restrict__ frozen,
         const int *__restrict__ exclStart, const int *__restrict__ exclFlat,
         const int *__restrict__ hmaxBits, const float4 *__restrict__ xq,
         const double *__restrict__ px, const double *__restrict__ py,
         const double *__restrict__ pz, const SearchOut o) {
  __shared__ WarpBuf bufs[kSearchThreads / 32];
  const int lane = threadIdx.x & 31;
  const int ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nClusters = *nSlotsDev >> 3;
  if (ci >= nClusters) return;
  WarpBuf &B = bufs[threadIdx.x >> 5];
  const int rep = clusterRep ? clusterRep[ci] : 0;
  const ClusterGeom &g = geoms[rep];
  const DevBox &box = boxes[rep];
  const int colBase = colOff[rep];
  hmaxBits += 4 * rep;

  const float4 oif = originF[ci];
  const float4 hi = half[ci];
  const int nreal_i = (int)hi.w;
  const int xy = clusterXY[ci];
  const int cx = xy & 0xffff, cy = xy >> 16;
  // this lane's i atom, its exclusion partners as slots
  const int ia = slotAtom[ci * kClusterSize + (lane & 7)];
  int es = 0, ee = 0;
  if (ia >= 0) {
    es = exclStart[ia];
    ee = exclStart[ia + 1];
  }
  const int nps = ee - es;
  int ps[kExclRegs];
#pragma unroll
  for (int r = 0; r < kExclRegs; ++r) ps[r] = (r < nps) ? slotOf[__ldg(exclFlat + es + r)] : -1;
  // the clusters holding any exclusion partner of the i cluster's atoms
  int pcLo = 0x7fffffff, pcHi = -1;
  for (int e = es; e < ee; ++e) {
    const int pc = (e - es < kExclRegs ? ps[min(e - es, kExclRegs - 1)]
                                       : slotOf[__ldg(exclFlat + e)]) / kClusterSize;
    pcLo = min(pcLo, pc);
    pcHi = max(pcHi, pc);
  }
  pcLo = __reduce_min_sync(0xffffffffu, pcLo);
  pcHi = __reduce_max_sync(0xffffffffu, pcHi);
  const int fi = (ia >= 0 && frozen) ? frozen[ia] : 0;
  const unsigned fimask = __ballot_sync(0xffffffffu, lane < kClusterSize && fi) & 0xffu;
  if (lane < 4) B.tally[lane] = 0;
  if (lane < kClusterSize) {
    const float4 xi = xq[ci * kClusterSize + lane];
    B.sn[lane] = make_float4(-xi.x, -xi.x, -xi.y, -xi.y);
    B.snz[lane] = make_float2(-xi.z, -xi.z);
#pragma unroll
    for (int r = 0; r < kExclRegs; ++r) B.ps[lane][r] = ps[r];
    B.es[lane] = es;
    B.ee[lane] = ee;
  }
  __syncwarp();

  const float rlist2 = g.rlist2;
  const float Lx = (float)g.Lx, Ly = (float)g.Ly, Lz = (float)g.Lz;
  const float wx = (float)g.wx, wy = (float)g.wy;
  // no cluster extends more than hmax[2] from its centre in z
  const float hzmax = __int_as_float(hmaxBits[2]);
  int cnt = 0, cand = 0;

  const int nx = 2 * g.Dx + 1, ncomb = nx * (2 * g.Dy + 1);
  int ncol = 0;
  for (int c0 = 0; c0 < ncomb; c0 += 32) {
    const int cb = c0 + lane;
    bool pass = false, zm = false, zp = false;
    int code = 0, tab = 0, zbl = 0, zbh = 0;  // tab: the cell's row of zTab
    if (cb < ncomb) {
      const int dy = cb / nx - g.Dy, dx = cb % nx - g.Dx;
      int jy = cy + dy, sy = 0;
      if (jy < 0) { jy += g.ncy; sy = -1; } else if (jy >= g.ncy) { jy -= g.ncy; sy = 1; }
      int jx = cx + dx, sx = 0;
      if (jx < 0) { jx += g.ncx; sx = -1; } else if (jx >= g.ncx) { jx -= g.ncx; sx = 1; }
      const float ylo = -0.5f * Ly + jy * wy + sy * Ly, yhi = ylo + wy;
      const float gy = fmaxf(fmaxf(ylo - (oif.y + hi.y), (oif.y - hi.y) - yhi), 0.f);
      const float xlo = -0.5f * Lx + jx * wx + sx * Lx, xhi = xlo + wx;
      const float gx = fmaxf(fmaxf(xlo - (oif.x + hi.x), (oif.x - hi.x) - xhi), 0.f);
      const float gxy2 = gx * gx + gy * gy;
      if (gxy2 <= rlist2) {
        tab = (colBase + jy * g.ncx + jx) * (kZBins + 1);
        code = (sx + 1) | ((sy + 1) << 2);
        pass = true;
        // the z reach left over the column's x-y gap (a cluster's x-y extent
        // lies inside its column: the gaps less 0.01 A, which covers the
        // rounding of both), the window of j origins it allows, and whether
        // the images below and above can be within reach (cluster centres
        // lie in [-Lz/2, Lz/2))
        const float gxm = fmaxf(gx - 0.01f, 0.f), gym = fmaxf(gy - 0.01f, 0.f);
        const float zr = sqrtf(fmaxf(rlist2 - (gxm * gxm + gym * gym), 0.f)) + 0.01f + hi.z + hzmax;
        const float zwlo = oif.z - zr, zwhi = oif.z + zr;
        zm = zwlo < -0.5f * Lz;
        zp = zwhi > 0.5f * Lz;
        // z-table bins of the window's ends (image sz: minus sz * kZBins),
        // widened by one bin below and two above since the bin of a
        // coordinate is rounded (the table's bin b starts at
        // -Lz/2 + b Lz / kZBins)
        zbl = __float2int_rd((zwlo + 0.5f * Lz) * ((float)kZBins / Lz)) - 1;
        zbh = __float2int_rd((zwhi + 0.5f * Lz) * ((float)kZBins / Lz)) + 2;
      }
    }
    // Per z image within reach, the column's clusters (z-sorted) whose
    // origin lies within the i box's reach: one listed range each.
#pragma unroll
    for (int sz = -1; sz <= 1; ++sz) {
      int first = 0, n = 0;
      if (pass && !((sz < 0 && !zm) || (sz > 0 && !zp))) {
        // the clusters with origin z in the window (a superset)
        const int bl = min(max(zbl - sz * kZBins, 0), kZBins);
        const int bh = min(max(zbh - sz * kZBins, 0), kZBins);
        first = __ldg(zTab + tab + bl);
        n = max(__ldg(zTab + tab + bh) - first, 0);
        // half list: a pair with cj < ci is listed from cj's side, so the
        // range starts at ci at the earliest (cluster indices ascend within
        // a column)
        if (first < ci) {
          n = max(0, first + n - ci);
          first = ci;
        }
      }
      const bool has = n > 0;
      const unsigned pm = __ballot_sync(0xffffffffu, has);
      if (has) {
        const int k = ncol + __popc(pm & ((1u << lane) - 1u));
        B.rstart[k] = first;
        B.rcount[k] = n;
        B.rcode[k] = code | ((sz + 1) << 4);
      }
      ncol += __popc(pm);
    }
    if (ncol <= kSearchCols - 96 && c0 + 32 < ncomb) continue;
    __syncwarp();
    // prefix of the listed ranges' cluster counts (kPer ranges per lane)
    constexpr int kPer = kSearchCols / 32;
    int v[kPer], tot = 0;
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const int k = kPer * lane + r;
      v[r] = k < ncol ? B.rcount[k] : 0;
      tot += v[r];
    }
    int incl = tot;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += t;
    }
    int run = incl - tot;
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const int k = kPer * lane + r;
      if (k <= ncol) B.rpre[k] = run;  // rpre[ncol] = total
      run += v[r];
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();
    int k0 = 0;  // the listed range holding flat index b0
    for (int b0 = 0; b0 < total; b0 += 32) {
      const int t = b0 + lane;
      const bool valid = t < total;
      int cj = 0, sx = 0, sy = 0, sz = 0;
      float4 oj = make_float4(0.f, 0.f, 1e30f, 0.f);
      float4 hj = make_float4(0.f, 0.f, 0.f, 0.f);
      // The range holding flat index t: lane j reads where range k0 + j ends,
      // relative to b0 (at least 1: range k0 holds b0), and marks that bit;
      // t's range is k0 plus the ranges that end at or before t.  At most 32
      // ranges end within a round (ranges are not empty).
      const int kj = k0 + lane + 1;
      const int ej = kj <= ncol ? B.rpre[kj] - b0 : 64;
      const unsigned ends = __reduce_or_sync(0xffffffffu, (ej > 0 && ej < 32) ? 1u << ej : 0u);
      const int rk = k0 + __popc(ends & ((2u << lane) - 1u));
      k0 += __popc(__ballot_sync(0xffffffffu, ej <= 32));
      if (valid) {
        cj = B.rstart[rk] + (t - B.rpre[rk]);
        const int rc = B.rcode[rk];
        sx = (rc & 3) - 1;
        sy = ((rc >> 2) & 3) - 1;
        sz = ((rc >> 4) & 3) - 1;
        oj = originF[cj];
        hj = half[cj];
      }
      const float fx = oj.x + sx * Lx - oif.x;
      const float fy = oj.y + sy * Ly - oif.y;
      const float fz = oj.z + sz * Lz - oif.z;
      const float gxx = fmaxf(fabsf(fx) - hi.x - hj.x, 0.f);
      const float gyy = fmaxf(fabsf(fy) - hi.y - hj.y, 0.f);
      const float gzz = fmaxf(fabsf(fz) - hi.z - hj.z, 0.f);
      cand += valid;
      const int sidx = (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
      const bool positive = sz > 0 || (sz == 0 && (sy > 0 || (sy == 0 && sx > 0)));
      const bool half_ok = (cj > ci) || (cj == ci && (sidx == 13 || positive));
      const bool ok = valid && half_ok && (gxx * gxx + gyy * gyy + gzz * gzz <= rlist2);
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const int pos = cnt + __popc(m & ((1u << lane) - 1u));
        B.j[pos] = cj;
        B.code[pos] = sidx | ((int)hj.w << 8);
      }
      cnt += __popc(m);
      __syncwarp();
      if (cnt >= kItemMax) {
        flush_item(B, kItemMax, ci, lane, xq, g, box, nreal_i, pcLo, pcHi, fimask, exclFlat,
                   slotOf, slotAtom, frozen, px, py, pz, origin, o);
        __syncwarp();
        const int rem = cnt - kItemMax;
        if (lane < rem) {
          B.j[lane] = B.j[kItemMax + lane];
          B.code[lane] = B.code[kItemMax + lane];
        }
        cnt = rem;
        __syncwarp();
      }
    }
    ncol = 0;
    __syncwarp();
  }
  if (cnt > 0)
    flush_item(B, cnt, ci, lane, xq, g, box, nreal_i, pcLo, pcHi, fimask, exclFlat, slotOf,
               slotAtom, frozen, px, py, pz, origin, o);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) cand += __shfl_xor_sync(0xffffffffu, cand, off);
  if (lane == 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(o.counters + 3), (unsigned long long)cand);
    // entries kept and inner halves written (the counts of the two lists),
    // warp steps of the half-cluster kernel over this i cluster's inner
    // items, and its inner pairs
    if (B.tally[0] > 0)
      atomicAdd(reinterpret_cast<unsigned long long *>(o.counters + 5),
                (unsigned long long)B.tally[0]);
    if (B.tally[1] > 0) {
      atomicAdd(reinterpret_cast<unsigned long long *>(o.hcounters + 6),
                (unsigned long long)B.tally[1]);
      atomicAdd(reinterpret_cast<unsigned long long *>(o.hcounters + 3),
                (unsigned long long)B.tally[2]);
      atomicAdd(reinterpret_cast<unsigned long long *>(o.hcounters + 4),
                (unsigned long long)B.tally[3]);
    }
    // The warp that finishes last (counters[7] counts the finished ones)
    // writes the readers' counts: entries kept (counters[5]) and inner halves
    // written (hcounters[6]); both lists have the packed counter's item count
    // (items << 40 | entries taken, counters[4]).  For a build that does not
    // wait it also latches the error bits into the sticky word: a list that
    // overflowed is unusable (its item count may point past the item buffer
    // and some items were never written), so the counts of both lists are
    // zeroed and the pair kernels that follow in the same stream (or graph)
    // see an empty list until the host rebuilds with room.
    __threadfence();
    const unsigned long long done =
        atomicAdd(reinterpret_cast<unsigned long long *>(o.counters + 7), 1ull);
    if (done + 1ull == (unsigned long long)nClusters) {
      __threadfence();
      auto rd = [](long long *p) {  // the value in L2, after every warp's atomics
        return (long long)atomicAdd(reinterpret_cast<unsigned long long *>(p), 0ull);
      };
      const unsigned long long a = (unsigned long long)rd(o.counters + 4);
      long long nEnt = rd(o.counters + 5), nIt = (long long)(a >> kPackShift);
      long long nHalf = rd(o.hcounters + 6);
      if (o.sticky) {
        const long long f = rd(o.counters + 2) | rd(o.hcounters + 2);
        o.sticky[0] |= f;
        if (f & CL_OVERFLOW) nEnt = nIt = nHalf = 0;
      }
      o.counters[0] = nEnt;
      o.counters[1] = nIt;
      o.hcounters[0] = nHalf;
      o.hcounters[1] = nIt;
    }
  }
}

__global__ void k_refresh(const int *__restrict__ nSlotsDev,
                          const ClusterGeom *__restrict__ geoms,
                          const int *__restrict__ clusterRep,
                          const int *__restrict__ slotAtom, const double4 *__restrict__ origin,
                          const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ z, const double *__restrict__ q, double sqrtC,
                          float4 *__restrict__ xq, float *__restrict__ xp) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= *nSlotsDev) return;
  const int a = slotAtom[s];
  if (a < 0) return;
  const ClusterGeom &g = geoms[clusterRep ? clusterRep[s / kClusterSize] : 0];
  const double4 o = origin[s / kClusterSize];
  double dx = x[a] - o.x, dy = y[a] - o.y, dz = z[a] - o.z;
  dx -= g.Lx * rint(dx / g.Lx);
  dy -= g.Ly * rint(dy / g.Ly);
  dz -= g.Lz * rint(dz / g.Lz);
  const float4 v = make_float4((float)dx, (float)dy, (float)dz, (float)(q[a] * sqrtC));
  xq[s] = v;
  const int k = s & (kClusterSize - 1);
  float *p = xp + (size_t)((s / kClusterSize) * 4 + (k & 3)) * 8 + (k >> 2);
  p[0] = v.x;
  p[2] = v.y;
  p[4] = v.z;
  p[6] = v.w;
}

// Per warp of the prune: the item's j atoms and its i atoms (negated and
// paired, as the search stages them).
struct PruneBuf {
  float4 sj[kClusterSize * kItemMax];  // sj[a * kItemMax + entry]
  float4 sn[kClusterSize];
  float2 snz[kClusterSize];
};
constexpr int kPruneThreads = 128;

// Rewrite the inner list at the current layout: one warp per item of the
// list and one lane per entry, as in the search's flush.  The item's j atoms
// are staged in shared memory, each lane forms its entry's 64 FP32 distances
// (j atom plus the shift, minus the i atom, as the pair kernel does), shifts
// the sign bits of (rin2 - r^2) into a word per half (bit i + 8 h) and keeps
// the pairs the list mask holds.  The entry halves with a pair become the
// item's inner entries, halves A first, at twice the entry index, and the
// inner item takes the item's index: no room is taken and nothing can
// overflow.  hcounters: [0] halves written, [1] items, [3] warp steps.
__global__ void __launch_bounds__(kPruneThreads)
k_prune(const long long *__restrict__ counters, const int4 *__restrict__ items,
        const CPairEntry *__restrict__ entries, const uint2 *__restrict__ masks,
        const float4 *__restrict__ xq, float rin2, HalfEntry *__restrict__ hent,
        unsigned *__restrict__ hmask, int4 *__restrict__ hitems,
        long long *__restrict__ hcounters) {
  __shared__ PruneBuf bufs[kPruneThreads / 32];
  PruneBuf &B = bufs[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const long long nItems = counters[1];
  if (blockIdx.x == 0 && threadIdx.x == 0) hcounters[1] = nItems;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const float2 rin = make_float2(rin2, rin2);
  long long halves = 0, steps = 0;
  for (long long it = gw; it < nItems; it += nw) {
    const int4 item = items[it];
    const int ci = item.x, e0 = item.y, ne = item.z;
    CPairEntry en{};
    uint2 mk = make_uint2(0u, 0u);
    if (lane < ne) {
      en = entries[e0 + lane];
      mk = masks[e0 + lane];
    }
    if (lane < kClusterSize) {
      const float4 xi = xq[ci * kClusterSize + lane];
      B.sn[lane] = make_float4(-xi.x, -xi.x, -xi.y, -xi.y);
      B.snz[lane] = make_float2(-xi.z, -xi.z);
    }
#pragma unroll
    for (int r = 0; r < kClusterSize; ++r) {
      const int idx = lane + 32 * r, k = idx >> 3, a = idx & 7;
      const int jk = __shfl_sync(0xffffffffu, en.j, k);
      if (k < ne) cp_async16(&B.sj[a * kItemMax + k], xq + (size_t)jk * kClusterSize + a);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncwarp();
    unsigned in0 = 0u, in1 = 0u;  // set bits: beyond the inner radius
    if (lane < ne) {
#pragma unroll 1
      for (int h = 3; h >= 0; --h) {
        const float4 pa = B.sj[h * kItemMax + lane], pb = B.sj[(h + 4) * kItemMax + lane];
        const float2 jx = make_float2(pa.x + en.sx, pb.x + en.sx);
        const float2 jy = make_float2(pa.y + en.sy, pb.y + en.sy);
        const float2 jz = make_float2(pa.z + en.sz, pb.z + en.sz);
#pragma unroll
        for (int i = kClusterSize - 1; i >= 0; --i) {
          const float4 nxy = lds_keep(&B.sn[i]);
          const float2 dx = __fadd2_rn(jx, make_float2(nxy.x, nxy.y));
          const float2 dy = __fadd2_rn(jy, make_float2(nxy.z, nxy.w));
          const float2 dz = __fadd2_rn(jz, lds_keep(&B.snz[i]));
          const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
          const float2 d = __ffma2_rn(r2, make_float2(-1.f, -1.f), rin);
          in0 = __funnelshift_l(__float_as_uint(d.x), in0, 1);
          in1 = __funnelshift_l(__float_as_uint(d.y), in1, 1);
        }
      }
      in0 = ~in0 & mk.x;
      in1 = ~in1 & mk.y;
    }
    __syncwarp();  // every lane is done with B before the next item's staging
    const unsigned hA = __ballot_sync(0xffffffffu, in0 != 0u);
    const unsigned hB = __ballot_sync(0xffffffffu, in1 != 0u);
    const int nA = __popc(hA), nin = nA + __popc(hB);
    const unsigned lt = (1u << lane) - 1u;
    if (in0 != 0u) {
      const long long q = 2 * (long long)e0 + __popc(hA & lt);
      HalfEntry he;
      he.jh = 2 * en.j;
      he.sx = en.sx;
      he.sy = en.sy;
      he.sz = en.sz;
      hent[q] = he;
      hmask[q] = in0;
    }
    if (in1 != 0u) {
      const long long q = 2 * (long long)e0 + nA + __popc(hB & lt);
      HalfEntry he;
      he.jh = 2 * en.j + 1;
      he.sx = en.sx;
      he.sy = en.sy;
      he.sz = en.sz;
      hent[q] = he;
      hmask[q] = in1;
    }
    if (lane == 0) {
      hitems[it] = make_int4(ci, 2 * e0, nin, 0);
      halves += nin;
      steps += (nin + 1) >> 1;
    }
  }
  if (lane == 0 && halves > 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(hcounters + 0), (unsigned long long)halves);
    atomicAdd(reinterpret_cast<unsigned long long *>(hcounters + 3), (unsigned long long)steps);
  }
}

// Latch a prune's error bits into the sticky word (the search latches its
// own in its last warp).  A list
// that overflowed is unusable: its item count may point past the item buffer
// and some items were never written, so the counts of both lists are zeroed
// and the pair kernels that follow in the same stream (or graph) see an
// empty list until the host rebuilds with room.
__global__ void k_latch(long long *__restrict__ counters, long long *__restrict__ hcounters,
                        long long *__restrict__ sticky) {
  if (threadIdx.x == 0) {
    const long long f = counters[2] | hcounters[2];
    sticky[0] |= f;
    if (f & CL_OVERFLOW) {
      counters[0] = 0;
      counters[1] = 0;
      hcounters[0] = 0;
      hcounters[1] = 0;
    }
  }
}

unsigned morton2(unsigned x, unsigned y) {
  auto spread = [](unsigned v) {
    v &= 0xffff;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
  };
  return spread(x) | (spread(y) << 1);
}

}  // namespace

namespace {

// Column grid of one box (orthorhombic), or an error status.
int make_geom(const DevBox &b, int n, double cutOff, double delr, int listRule, ClusterGeom &g) {
  if (b.type != CUBIC && b.type != ORBIC) return MDBAS_NB_ERR_UNSUPPORTED;
  if (n <= 0) return MDBAS_NB_ERR_ARG;
  g = ClusterGeom{};
  g.Lx = b.a1;
  g.Ly = (b.type == CUBIC) ? b.a1 : b.b2;
  g.Lz = (b.type == CUBIC) ? b.a1 : b.c3;
  g.invLx = 1.0 / g.Lx;
  g.invLy = 1.0 / g.Ly;
  g.invLz = 1.0 / g.Lz;
  const double rlist = cutOff + delr;
  // The pair kernel relies on a unique image within the cut-off.
  if (std::min(g.Lx, std::min(g.Ly, g.Lz)) <= 2.0 * cutOff) return MDBAS_NB_ERR_BOX;
  const double vol = g.Lx * g.Ly * g.Lz;
  // cells hold ~8 atoms each, but are wide enough that the search reaches at
  // most 7 cells to each side ((2 D + 1)^2 columns within the block table)
  const double w0 = std::max(std::cbrt((double)kClusterSize * vol / (double)n), rlist / 6.5);
  g.ncx = std::max(1, (int)std::lround(g.Lx / w0));
  g.ncy = std::max(1, (int)std::lround(g.Ly / w0));
  g.wx = g.Lx / g.ncx;
  g.wy = g.Ly / g.ncy;
  g.Dx = (int)std::floor(rlist / g.wx) + 1;
  g.Dy = (int)std::floor(rlist / g.wy) + 1;
  if (g.Dx >= g.ncx || g.Dy >= g.ncy) {
    // Fewer cells than the search reaches: use one cell column fewer than
    // the reach in that direction so shifts stay within one image.
    if (rlist + g.wx >= g.Lx || rlist + g.wy >= g.Ly) return MDBAS_NB_ERR_BOX;
    if (g.Dx >= g.ncx) g.Dx = g.ncx - 1;
    if (g.Dy >= g.ncy) g.Dy = g.ncy - 1;
  }
  // MDBas's list radius (src/list.c: cutnb = cutOff + delr, compared with its
  // square) and the FP32 band around it
  g.cutnb2 = rlist * rlist;
  g.rlo2 = (float)(g.cutnb2 * (1.0 - 2e-5));
  g.rhi2 = (float)(g.cutnb2 * (1.0 + 2e-5));
  g.rlist2 = g.rhi2;
  g.listMode = makelist_uses_link_cells(b, cutOff, delr, listRule & 7, (listRule >> 3) & 1);
  return MDBAS_NB_OK;
}

bool same_geom(const ClusterGeom &a, const ClusterGeom &b) {
  return a.ncx == b.ncx && a.ncy == b.ncy && a.Dx == b.Dx && a.Dy == b.Dy && a.Lx == b.Lx &&
         a.Ly == b.Ly && a.Lz == b.Lz && a.rlist2 == b.rlist2 && a.listMode == b.listMode;
}

}  // namespace

int cluster_build(ClusterWork &w, int n, int nRep, const DevBox *boxes, const int *atomOff,
                  double cutOff, double delr, int listRule, double sqrtC, const double *x,
                  const double *y, const double *z, const double *q, const double *eps,
                  const double *sig, const int *frozen, const int *exclStart,
                  const int *exclFlat, cudaStream_t s, bool sync) {
  if (nRep <= 0 || n <= 0 || atomOff[0] != 0 || atomOff[nRep] != n) return MDBAS_NB_ERR_ARG;
  std::vector<ClusterGeom> geoms(nRep);
  std::vector<int> colOff(nRep + 1, 0);
  for (int r = 0; r < nRep; ++r) {
    const int nr = atomOff[r + 1] - atomOff[r];
    MDB_TRY(make_geom(boxes[r], nr, cutOff, delr, listRule, geoms[r]));
    colOff[r + 1] = colOff[r] + geoms[r].ncx * geoms[r].ncy;
  }
  const int nCols = colOff[nRep];
  const int slotCap = (n + (kClusterSize - 1) * nCols + kClusterSize - 1) & ~(kClusterSize - 1);
  bool sameGrid = nRep == w.nRep && w.atomOffH.size() == (size_t)nRep + 1;
  for (int r = 0; sameGrid && r < nRep; ++r)
    sameGrid = same_geom(geoms[r], w.geomH[r]) && atomOff[r + 1] == w.atomOffH[r + 1];
  // The captured form cannot upload tables or grow buffers.
  if (!sync && (!sameGrid || slotCap > w.slotCap || w.entryCap == 0)) return MDBAS_NB_ERR_STATE;

  // Per-replica tables, rebuilt when any grid changes: Morton rank of each
  // (cx, cy) cell as a global column, and each column's (cx, cy).
  if (!sameGrid) {
    std::vector<int> rank(nCols), xyOf(nCols);
    for (int r = 0; r < nRep; ++r) {
      const ClusterGeom &g = geoms[r];
      const int nc = g.ncx * g.ncy;
      std::vector<std::pair<unsigned, int>> keys(nc);
      for (int cy = 0; cy < g.ncy; ++cy)
        for (int cx = 0; cx < g.ncx; ++cx)
          keys[cy * g.ncx + cx] = {morton2(cx, cy), cy * g.ncx + cx};
      std::sort(keys.begin(), keys.end());
      for (int k = 0; k < nc; ++k) {
        const int cell = keys[k].second;
        rank[colOff[r] + cell] = colOff[r] + k;
        xyOf[colOff[r] + k] = (cell % g.ncx) | ((cell / g.ncx) << 16);
      }
    }
    MDB_TRY(w.colRank.ensure(sizeof(int) * nCols));
    MDB_TRY(w.colXY.ensure(sizeof(int) * nCols));
    MDB_TRY(w.geoms.ensure(sizeof(ClusterGeom) * nRep));
    MDB_TRY(w.colOff.ensure(sizeof(int) * (nRep + 1)));
    MDB_TRY(w.boxes.ensure(sizeof(DevBox) * nRep));
    MDB_CUDA(cudaMemcpyAsync(w.colRank.p, rank.data(), sizeof(int) * nCols,
                             cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaMemcpyAsync(w.colXY.p, xyOf.data(), sizeof(int) * nCols,
                             cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaMemcpyAsync(w.geoms.p, geoms.data(), sizeof(ClusterGeom) * nRep,
                             cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaMemcpyAsync(w.colOff.p, colOff.data(), sizeof(int) * (nRep + 1),
                             cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaMemcpyAsync(w.boxes.p, boxes, sizeof(DevBox) * nRep, cudaMemcpyHostToDevice, s));
    if (nRep > 1) {
      std::vector<int> rep(n);
      for (int r = 0; r < nRep; ++r)
        for (int i = atomOff[r]; i < atomOff[r + 1]; ++i) rep[i] = r;
      MDB_TRY(w.atomRep.ensure(sizeof(int) * n));
      MDB_CUDA(cudaMemcpyAsync(w.atomRep.p, rep.data(), sizeof(int) * n, cudaMemcpyHostToDevice,
                               s));
    }
    MDB_CUDA(cudaStreamSynchronize(s));
    w.geomH = geoms;
    w.colOffH = colOff;
    w.atomOffH.assign(atomOff, atomOff + nRep + 1);
    w.nRep = nRep;
  }
  w.geom = geoms[0];
  w.nCols = nCols;

  if (sync) {
    MDB_TRY(w.colCount.ensure(sizeof(int) * (nCols + 1)));
    MDB_TRY(w.colFill.ensure(sizeof(int) * (nCols + 1)));
    MDB_TRY(w.colStart.ensure(sizeof(int) * (nCols + 2)));
    MDB_TRY(w.colPadStart.ensure(sizeof(int) * (nCols + 2)));
    MDB_TRY(w.colClStart.ensure(sizeof(int) * (nCols + 2)));
    MDB_TRY(w.zTab.ensure(sizeof(int) * (size_t)nCols * (kZBins + 1)));
    MDB_TRY(w.atomCol.ensure(sizeof(int) * n));
    MDB_TRY(w.atomZ.ensure(sizeof(double) * n));
    MDB_TRY(w.tmpIdx.ensure(sizeof(int) * n));
    MDB_TRY(w.slotOf.ensure(sizeof(int) * n));
    MDB_TRY(w.counters.ensure(sizeof(long long) * 8));
    MDB_TRY(w.countersIn.ensure(sizeof(long long) * 8));
    MDB_TRY(w.acc.ensure(sizeof(long long) * ACC_COUNT));
    if (!w.sticky.p) {
      MDB_TRY(w.sticky.ensure(sizeof(long long)));
      MDB_CUDA(cudaMemsetAsync(w.sticky.p, 0, sizeof(long long), s));
    }
    if (slotCap > w.slotCap) {
      w.slotCap = slotCap;
      w.clCap = slotCap / kClusterSize;
    }
    MDB_TRY(w.slotAtom.ensure(sizeof(int) * w.slotCap));
    MDB_TRY(w.clusterXY.ensure(sizeof(int) * w.clCap));
    if (nRep > 1) MDB_TRY(w.clusterRep.ensure(sizeof(int) * w.clCap));
    MDB_TRY(w.origin.ensure(sizeof(double4) * w.clCap));
    MDB_TRY(w.half.ensure(sizeof(float4) * w.clCap));
    MDB_TRY(w.originF.ensure(sizeof(float4) * w.clCap));
    MDB_TRY(w.hmax.ensure(sizeof(int) * 4 * nRep));
    MDB_TRY(w.xq.ensure(sizeof(float4) * w.slotCap));
    MDB_TRY(w.lj.ensure(sizeof(float2) * w.slotCap));
    MDB_TRY(w.xp.ensure(sizeof(float4) * 8 * (size_t)w.clCap));
    MDB_TRY(w.ljp.ensure(sizeof(float4) * 4 * (size_t)w.clCap));
    MDB_TRY(w.facc.ensure(sizeof(long long) * 3 * (size_t)w.slotCap));
  }
  const ClusterGeom *gd = w.geoms.as<ClusterGeom>();

  MDB_LAUNCH(k_build_reset, 1, 256, 0, s, nCols, nRep, w.colCount.as<int>(),
             w.colFill.as<int>(), w.counters.as<long long>(), w.countersIn.as<long long>(),
             w.hmax.as<int>());
  if (w.timeStages) MDB_CUDA(cudaEventRecord(w.stageEv[0], s));
  MDB_LAUNCH(k_col_bin, grid_for(n, 256), 256, 0, s, n, gd, w.atomRepDev(), w.colOff.as<int>(),
             w.colRank.as<int>(), x, y, z, w.atomCol.as<int>(), w.atomZ.as<double>(),
             w.colCount.as<int>(), w.counters.as<long long>());
  if (w.timeStages) MDB_CUDA(cudaEventRecord(w.stageEv[1], s));
  MDB_LAUNCH(k_col_scan, 1, 1024, 0, s, nCols, w.colCount.as<int>(), w.colStart.as<int>(),
             w.colPadStart.as<int>(), w.colClStart.as<int>());
  if (w.timeStages) MDB_CUDA(cudaEventRecord(w.stageEv[2], s));
  MDB_LAUNCH(k_col_scatter, grid_for(n, 256), 256, 0, s, n, w.atomCol.as<int>(),
             w.colStart.as<int>(), w.colFill.as<int>(), w.tmpIdx.as<int>());
  if (w.timeStages) MDB_CUDA(cudaEventRecord(w.stageEv[3], s));
  MDB_LAUNCH(k_col_sort, nCols, 256, 0, s, nCols, w.colStart.as<int>(), w.colPadStart.as<int>(),
             w.tmpIdx.as<int>(), w.atomZ.as<double>(), w.slotAtom.as<int>());
  if (w.timeStages) MDB_CUDA(cudaEventRecord(w.stageEv[4], s));
  MDB_LAUNCH(k_clusters, grid_for(w.slotCap, 256), 256, 0, s, w.nSlotsDev(), gd, w.atomRepDev(),
             nRep > 1 ? w.clusterRep.as<int>() : nullptr, w.slotAtom.as<int>(), w.atomCol.as<int>(), w.colXY.as<int>(), x,
             y, z, q, eps, sig, sqrtC, w.origin.as<double4>(), w.originF.as<float4>(),
             w.half.as<float4>(), w.xq.as<float4>(), w.lj.as<float2>(), w.xp.as<float>(),
             w.ljp.as<float>(), w.slotOf.as<int>(), w.clusterXY.as<int>(), w.hmax.as<int>());
  MDB_LAUNCH(k_col_ztab, nCols, (kZBins + 32) & ~31, 0, s, nCols, gd, w.clusterRepDev(),
             w.colRank.as<int>(), w.colClStart.as<int>(), w.originF.as<float4>(),
             w.zTab.as<int>());

  // Cluster-pair search; in the synchronising form grow the list and search
  // again if it overflowed.  The inner list holds at most two halves per
  // entry, so it never overflows on its own.
  if (w.entryCap == 0) {
    w.entryCap = (long long)w.clCap * 192 + 4096;
    w.itemCap = w.entryCap / kItemMax + w.clCap + 1024;
  }
  // 0: the pair kernel's own FP32 rc^2 (PairConstF::rc2), whose test on the
  // kernel's own FP32 distances the search repeats bit for bit
  const float rin2 = w.rin2 > 0.f ? w.rin2 : (float)(cutOff * cutOff);
  for (int attempt = 0; attempt < 4; ++attempt) {
    w.inEntryCap = 2 * w.entryCap;
    w.inItemCap = w.itemCap;
    if (sync) {
      MDB_TRY(w.entries.ensure(sizeof(CPairEntry) * (size_t)w.entryCap));
      MDB_TRY(w.masks.ensure(sizeof(uint2) * (size_t)w.entryCap));
      MDB_TRY(w.items.ensure(sizeof(int4) * (size_t)w.itemCap));
      MDB_TRY(w.entriesIn.ensure(sizeof(HalfEntry) * (size_t)w.inEntryCap));
      MDB_TRY(w.masksIn.ensure(sizeof(unsigned) * (size_t)w.inEntryCap));
      MDB_TRY(w.itemsIn.ensure(sizeof(int4) * (size_t)w.inItemCap));
    }
    if (attempt > 0) {  // the first attempt's counters were cleared by k_build_reset
      MDB_CUDA(cudaMemsetAsync(w.counters.p, 0, sizeof(long long) * 2, s));
      MDB_CUDA(cudaMemsetAsync(w.counters.as<long long>() + 3, 0, sizeof(long long) * 5, s));
      MDB_CUDA(cudaMemsetAsync(w.countersIn.p, 0, sizeof(long long) * 8, s));
    }
    SearchOut o;
    o.entries = w.entries.as<CPairEntry>();
    o.masks = w.masks.as<uint2>();
    o.items = w.items.as<int4>();
    o.counters = w.counters.as<long long>();
    o.entryCap = w.entryCap;
    o.itemCap = w.itemCap;
    o.hent = w.entriesIn.as<HalfEntry>();
    o.hmask = w.masksIn.as<unsigned>();
    o.hitems = w.itemsIn.as<int4>();
    o.hcounters = w.countersIn.as<long long>();
    o.rin2 = rin2;
    o.sticky = sync ? nullptr : w.sticky.as<long long>();
  if (w.timeStages) MDB_CUDA(cudaEventRecord(w.stageEv[5], s));
    MDB_LAUNCH(k_search, grid_for((long long)w.clCap * 32, kSearchThreads), kSearchThreads, 0, s,
               w.nSlotsDev(), gd, w.boxes.as<DevBox>(), w.clusterRepDev(), w.colOff.as<int>(),
               w.zTab.as<int>(), w.clusterXY.as<int>(),
               w.origin.as<double4>(), w.originF.as<float4>(), w.half.as<float4>(),
               w.slotAtom.as<int>(), w.slotOf.as<int>(), frozen, exclStart, exclFlat,
               w.hmax.as<int>(), w.xq.as<float4>(), x, y, z, o);
  if (w.timeStages) MDB_CUDA(cudaEventRecord(w.stageEv[6], s));
    w.innerRin2 = rin2;
    if (!sync) {
      w.useInner = true;
      return MDBAS_NB_OK;
    }
    long long flags[8], hflags[4];
    int nSlots = 0;
    MDB_CUDA(cudaMemcpyAsync(flags, w.counters.p, sizeof(flags), cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaMemcpyAsync(hflags, w.countersIn.p, sizeof(hflags), cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaMemcpyAsync(&nSlots, w.nSlotsDev(), sizeof(int), cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaStreamSynchronize(s));
    if (flags[2] & CL_NONFINITE) return MDBAS_NB_ERR_NONFINITE;
    w.nSlots = nSlots;
    w.nClusters = nSlots / kClusterSize;
    w.nEntries = flags[0];
    w.nItems = flags[1];
    w.nInEntries = hflags[0];
    w.nInItems = hflags[1];
    w.nInSteps = hflags[3];
    if (!(flags[2] & CL_OVERFLOW)) {
      w.useInner = true;
      return MDBAS_NB_OK;
    }
    // the search does not clear the overflow bit; the next attempt starts clean
    MDB_CUDA(cudaMemsetAsync(w.counters.as<long long>() + 2, 0, sizeof(long long), s));
    // room for the entries the search took (kept or not)
    const long long taken = (long long)((unsigned long long)flags[4] & ((1ull << kPackShift) - 1ull));
    w.entryCap = (long long)(taken * 1.25) + 4096;
    w.itemCap = (long long)(flags[1] * 1.25) + 1024;
  }
  return MDBAS_NB_ERR_CAPACITY;
}

int cluster_build(ClusterWork &w, int n, const DevBox &b, double cutOff, double delr,
                  int listRule, double sqrtC, const double *x, const double *y,
                  const double *z, const double *q, const double *eps, const double *sig,
                  const int *frozen, const int *exclStart, const int *exclFlat, cudaStream_t s,
                  bool sync) {
  const int off[2] = {0, n};
  return cluster_build(w, n, 1, &b, off, cutOff, delr, listRule, sqrtC, x, y, z, q, eps, sig,
                       frozen, exclStart, exclFlat, s, sync);
}

void cluster_symmetric_excl(int n, const int *start, const int *flat, std::vector<int> &outStart,
                            std::vector<int> &outFlat) {
  std::vector<std::vector<int>> rows(n);
  for (int i = 0; i < n; ++i)
    for (int k = start[i]; k < start[i + 1]; ++k) {
      const int j = flat[k];
      if (j == i) continue;
      rows[i].push_back(j);
      rows[j].push_back(i);
    }
  outStart.assign(n + 1, 0);
  outFlat.clear();
  for (int i = 0; i < n; ++i) {
    std::vector<int> &r = rows[i];
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    outFlat.insert(outFlat.end(), r.begin(), r.end());
    outStart[i + 1] = (int)outFlat.size();
  }
}

int cluster_prune(ClusterWork &w, float rin2, cudaStream_t s) {
  if (w.entryCap <= 0 || !w.countersIn.p) return MDBAS_NB_ERR_STATE;
  int dev = 0, sms = 148;
  MDB_CUDA(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  MDB_CUDA(cudaMemsetAsync(w.countersIn.p, 0, sizeof(long long) * 8, s));
  MDB_LAUNCH(k_prune, sms * 16, kPruneThreads, 0, s, w.counters.as<long long>(),
             w.items.as<int4>(), w.entries.as<CPairEntry>(), w.masks.as<uint2>(),
             w.xq.as<float4>(), rin2, w.entriesIn.as<HalfEntry>(), w.masksIn.as<unsigned>(),
             w.itemsIn.as<int4>(), w.countersIn.as<long long>());
  MDB_LAUNCH(k_latch, 1, 32, 0, s, w.counters.as<long long>(), w.countersIn.as<long long>(),
             w.sticky.as<long long>());
  w.innerRin2 = rin2;
  w.useInner = true;
  return MDBAS_NB_OK;
}

int cluster_build_stages(ClusterWork &w, int n, int nRep, const DevBox *boxes,
                         const int *atomOff, double cutOff, double delr, int listRule,
                         double sqrtC, const double *x, const double *y, const double *z,
                         const double *q, const double *eps, const double *sig,
                         const int *frozen, const int *exclStart, const int *exclFlat,
                         cudaStream_t s, double ms[6]) {
  for (cudaEvent_t &ev : w.stageEv)
    if (!ev) MDB_CUDA(cudaEventCreate(&ev));
  w.timeStages = true;
  const int st = cluster_build(w, n, nRep, boxes, atomOff, cutOff, delr, listRule, sqrtC, x, y,
                               z, q, eps, sig, frozen, exclStart, exclFlat, s, true);
  w.timeStages = false;
  MDB_TRY(st);
  MDB_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < 6; ++k) {
    float t = 0.f;
    MDB_CUDA(cudaEventElapsedTime(&t, w.stageEv[k], w.stageEv[k + 1]));
    ms[k] = t;
  }
  return MDBAS_NB_OK;
}

int cluster_read_counts(ClusterWork &w, cudaStream_t s) {
  if (!w.counters.p || w.nCols <= 0) return MDBAS_NB_ERR_STATE;
  long long flags[4], hflags[4] = {0, 0, 0, 0};
  int nSlots = 0;
  MDB_CUDA(cudaMemcpyAsync(flags, w.counters.p, sizeof(flags), cudaMemcpyDeviceToHost, s));
  if (w.countersIn.p)
    MDB_CUDA(cudaMemcpyAsync(hflags, w.countersIn.p, sizeof(hflags), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaMemcpyAsync(&nSlots, w.nSlotsDev(), sizeof(int), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  w.nSlots = nSlots;
  w.nClusters = nSlots / kClusterSize;
  w.nEntries = flags[0];
  w.nItems = flags[1];
  w.nInEntries = hflags[0];
  w.nInItems = hflags[1];
  w.nInSteps = hflags[3];
  return MDBAS_NB_OK;
}

int cluster_refresh(ClusterWork &w, const double *x, const double *y, const double *z,
                    const double *q, double sqrtC, cudaStream_t s) {
  if (w.slotCap <= 0) return MDBAS_NB_ERR_STATE;
  // an inner list at the plain cut-off holds the pairs of the build's
  // positions only
  if (w.rin2 == 0.f) w.useInner = false;
  MDB_LAUNCH(k_refresh, grid_for(w.slotCap, 256), 256, 0, s, w.nSlotsDev(),
             w.geoms.as<ClusterGeom>(), w.clusterRepDev(), w.slotAtom.as<int>(),
             w.origin.as<double4>(), x, y, z, q, sqrtC, w.xq.as<float4>(), w.xp.as<float>());
  return MDBAS_NB_OK;
}

}  // namespace mdbas
