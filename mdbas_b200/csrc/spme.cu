// spme.cu -- smooth particle-mesh Ewald on the GPU: MDBas's init_spme,
// spme_energy and spme_free (include/spme.h:28-40; src/spme.c) and a
// status-returning entry point.
//
// The algorithm is MDBas's (src/spme.c:357-700): per atom the cardinal
// B-splines of order nbsp and their derivatives in each dimension
// (bspgen's recursion), charges spread onto the m1 x m2 x m3 grid, an
// unnormalised e^{+i} 3-D transform (FFTW_BACKWARD), the influence function
// B(m) exp(-k^2 / 4 alpha^2) / k^2 inside the reciprocal cut-off with the
// virial, an e^{-i} transform back (FFTW_FORWARD), force interpolation with
// the mean force removed, and the energy sum(Q * (theta conv Q)) with the
// self and non-neutral terms.  The transforms are cuFFT Z2Z plans in the
// same row-major layout as fftw_plan_dft_3d(m1, m2, m3); spreading, the
// influence function and the interpolation are the kernels below (FP64).
// Spreading is deterministic when every grid dimension is a multiple of 8
// (atoms binned by 8^3 grid tile, one block per tile, no atomics); other
// grids spread with FP64 atomics.
#include <cufft.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <complex>
#include <vector>

#include "kspace.cuh"

using namespace mdbas;

namespace {

constexpr int kMaxOrder = 16;  // B-spline orders 2..16

struct SpmeBox {
  double u1, u2, u3, v1, v2, v3, w1, w2, w3;  // reciprocal vectors
  double u, v, w;                             // 1 / perpendicular widths
  double vol;
};

// B-splines and derivatives of one atom in one dimension (bspgen,
// src/spme.c:269-355): s is the scaled fractional coordinate.
template <int P>  // the order, or 0: nbspRun
__device__ __forceinline__ void bspline(double s, int nbspRun, double *bsp, double *bsd) {
  const int nbsp = P > 0 ? P : nbspRun;
  const double fr = s - trunc(s);
#pragma unroll
  for (int k = 0; k < nbsp; ++k) bsp[k] = bsd[k] = 0.;
  bsd[0] = 1.0;
  bsd[1] = -1.0;
  bsp[0] = fr;
  bsp[1] = 1.0 - fr;
#pragma unroll
  for (int k = 2; k < nbsp; ++k) {
    bsp[k] = 0.0;
#pragma unroll
    for (int j = k; j > 0; --j) {
      if (k == nbsp - 1) bsd[j] = bsp[j] - bsp[j - 1];
      const double ts = s + (double)j - trunc(s);
      bsp[j] = (ts * bsp[j] + ((double)(k + 1) - ts) * bsp[j - 1]) / (double)k;
    }
    if (k == nbsp - 1) bsd[0] = bsp[0];
    bsp[0] = fr * bsp[0] / (double)k;
  }
}

// grid index of the stencil point base cell - offset; base cells are stored
// in [0, m), so one wrap brings it into [0, m) as MDBas's does for atoms in
// the box (src/spme.c:453-481)
__device__ __forceinline__ int wrap_index(int i, int m) { return i < 0 ? i + m : i; }

// base cell in [0, m).  MDBas's (int)s lies in [0, m] for atoms in the box
// (image_update wraps them there before every energy call) and its indices
// (int)s - a wrap to the same grid points; for atoms further out the
// periodic image is used, which keeps every grid access in bounds (MDBas
// folds indices >= m onto plane 0 and leaves the array below -(m - p + 1)).
__device__ __forceinline__ int cell_mod(int c, int m) {
  c %= m;
  return c < 0 ? c + m : c;
}

// Per atom and dimension (one thread each): the grid coordinate, B-splines
// (bsp[3][nbsp], bsd[3][nbsp] per atom) and the integer grid cell.
template <int P>  // the order, or 0: nbspRun
__global__ void k_spme_splines(int n, SpmeBox b, int m1, int m2, int m3, int nbspRun,
                               const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, double *__restrict__ spl,
                               int *__restrict__ cell) {
  const int nbsp = P > 0 ? P : nbspRun;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n) return;
  const int i = t / 3, d = t - 3 * (t / 3);
  double s;
  if (d == 0) s = (double)m1 * (x[i] * b.u1 + y[i] * b.u2 + z[i] * b.u3 + 0.5);
  else if (d == 1) s = (double)m2 * (x[i] * b.v1 + y[i] * b.v2 + z[i] * b.v3 + 0.5);
  else s = (double)m3 * (x[i] * b.w1 + y[i] * b.w2 + z[i] * b.w3 + 0.5);
  double *o = spl + (size_t)i * 6 * nbsp;
  double bp[P > 0 ? P : kMaxOrder], bd[P > 0 ? P : kMaxOrder];
  bspline<P>(s, nbsp, bp, bd);
#pragma unroll
  for (int k = 0; k < (P > 0 ? P : nbsp); ++k) {
    o[d * nbsp + k] = bp[k];
    o[(3 + d) * nbsp + k] = bd[k];
  }
  cell[3 * i + d] = cell_mod((int)s, d == 0 ? m1 : (d == 1 ? m2 : m3));
}

// Charge spreading: one thread per (atom, first-dimension offset).
__global__ void k_spme_spread(int n, int m1, int m2, int m3, int nbsp,
                              const double *__restrict__ q, const double *__restrict__ spl,
                              const int *__restrict__ cell, double *__restrict__ qsp) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * nbsp) return;
  const int l = (int)(t / nbsp), a = (int)(t % nbsp);
  const double *o = spl + (size_t)l * 6 * nbsp;
  const int ii = wrap_index(cell[3 * l] - a, m1);
  const double qa = q[l] * o[a];
  for (int bb = 0; bb < nbsp; ++bb) {
    const int jj = wrap_index(cell[3 * l + 1] - bb, m2);
    const double qab = qa * o[nbsp + bb];
    const size_t base = (size_t)m3 * (jj + (size_t)m2 * ii);
    for (int c = 0; c < nbsp; ++c) {
      const int kk = wrap_index(cell[3 * l + 2] - c, m3);
      atomicAdd(qsp + base + kk, qab * o[2 * nbsp + c]);
    }
  }
}

// Deterministic spreading.  The grid is cut into 8^3 tiles (every grid
// dimension a multiple of 8); atoms are binned by the tile of their base
// cell and each bin is put in ascending atom order.  Phase one, one block per
// tile: the bin's atoms, one after the other, scatter their p^3 stencils
// into a shared-memory copy of the tile plus its halo ((8 + p - 1)^3 points:
// a stencil reaches p - 1 cells below its base cell), one thread per stencil
// point; the halo boxes go to global memory.  Phase two, one thread per grid
// point: the sum over the halo boxes that cover the point (its own tile and
// the next ones upward, as far as the order reaches) in a fixed order.  No
// atomics: the same sums in the same order on every run.
constexpr int kSpTile = 8;
constexpr int kSpBatch = 32;
constexpr int kSpPts = (kMaxOrder * kMaxOrder * kMaxOrder + 511) / 512;  // per thread

__global__ void k_spme_tile_count(int n, int m1, int m2, int m3, int nt2, int nt3,
                                  const int *__restrict__ cell, int *__restrict__ tileOf,
                                  int *__restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int t = ((cell[3 * i] / kSpTile) * nt2 + cell[3 * i + 1] / kSpTile) * nt3 +
                cell[3 * i + 2] / kSpTile;
  tileOf[i] = t;
  atomicAdd(count + t, 1);
}

__global__ void k_spme_tile_fill(int n, const int *__restrict__ tileOf,
                                 const int *__restrict__ start, int *__restrict__ fill,
                                 int *__restrict__ list) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int t = tileOf[i];
  list[start[t] + atomicAdd(fill + t, 1)] = i;
}

// one block per bin: its atoms in ascending index order (rank sort)
__global__ void k_spme_tile_sort(const int *__restrict__ start, const int *__restrict__ list,
                                 int *__restrict__ sorted) {
  const int s0 = start[blockIdx.x], s1 = start[blockIdx.x + 1];
  for (int u = s0 + threadIdx.x; u < s1; u += blockDim.x) {
    const int a = list[u];
    int rank = 0;
    for (int v = s0; v < s1; ++v) rank += list[v] < a;
    sorted[s0 + rank] = a;
  }
}

template <int PTS>  // stencil points per thread: 1 when p^3 <= 512
__global__ void __launch_bounds__(512, PTS == 1 ? 3 : 2)
    k_spme_spread_halo(int nbsp, int nt2, int nt3, const double *__restrict__ q,
                       const double *__restrict__ spl, const int *__restrict__ cell,
                       const int *__restrict__ start, const int *__restrict__ sorted,
                       double *__restrict__ halo) {
  extern __shared__ double hb[];  // (8 + p - 1)^3 halo box
  __shared__ double sq[kSpBatch];
  __shared__ int sc[kSpBatch];
  __shared__ double sb[kSpBatch][3 * kMaxOrder];
  const int tile = blockIdx.x;
  const int t3 = tile % nt3, t2 = (tile / nt3) % nt2, t1 = tile / (nt2 * nt3);
  const int H = kSpTile + nbsp - 1, H3 = H * H * H, p3 = nbsp * nbsp * nbsp;
  const int th = threadIdx.x;
  // this thread's stencil points (a, b, c), at most PTS of them
  int abc[PTS];
#pragma unroll
  for (int k = 0; k < PTS; ++k) {
    const int idx = th + k * 512;
    abc[k] = idx / (nbsp * nbsp) | ((idx / nbsp) % nbsp) << 8 | (idx % nbsp) << 16;
  }
  for (int u = th; u < H3; u += blockDim.x) hb[u] = 0.;
  const int s0 = start[tile], s1 = start[tile + 1];
  for (int base = s0; base < s1; base += kSpBatch) {
    const int cnt = min(kSpBatch, s1 - base);
    __syncthreads();
    if (th < cnt) {
      const int a = sorted[base + th];
      sq[th] = q[a];
      // the stencil's top corner in the halo box: base cell - tile origin + p - 1
      sc[th] = ((cell[3 * a] - kSpTile * t1 + nbsp - 1) * H +
                (cell[3 * a + 1] - kSpTile * t2 + nbsp - 1)) * H +
               (cell[3 * a + 2] - kSpTile * t3 + nbsp - 1);
    }
    for (int idx = th; idx < cnt * 3 * nbsp; idx += blockDim.x) {
      const int u = idx / (3 * nbsp), r = idx - u * 3 * nbsp;
      sb[u][r] = spl[(size_t)sorted[base + u] * 6 * nbsp + r];
    }
    __syncthreads();
    for (int u = 0; u < cnt; ++u) {
      const double qu = sq[u];
      const int su = sc[u];
#pragma unroll
      for (int k = 0; k < PTS; ++k)
        if (th + k * 512 < p3) {
          const int a = abc[k] & 0xff, bb = (abc[k] >> 8) & 0xff, c = abc[k] >> 16;
          hb[su - (a * H + bb) * H - c] +=
              ((qu * sb[u][a]) * sb[u][nbsp + bb]) * sb[u][2 * nbsp + c];
        }
      __syncthreads();  // the next atom may hit the same points
    }
  }
  __syncthreads();
  double *out = halo + (size_t)tile * H3;
  for (int u = th; u < H3; u += blockDim.x) out[u] = hb[u];
}

// Phase one for a B-spline order P known at compile time (P <= 9, so the
// (8 + P - 1)^2 rows of the halo box fit one block): each thread owns one
// row (l1, l2) of the box, kept in shared memory; an atom covers the row
// when its stencil planes reach l1 and l2, and then adds ((q b1_a) b2_b) b3_c
// to the row's points -- the same products, summed over the bin's atoms in
// the same ascending order, as k_spme_spread_halo, but no thread ever
// touches another's row: no barrier per atom.
template <int P>
__global__ void __launch_bounds__(256)
    k_spme_spread_rows(int nt2, int nt3, const double *__restrict__ q,
                       const double *__restrict__ spl, const int *__restrict__ cell,
                       const int *__restrict__ start, const int *__restrict__ sorted,
                       double *__restrict__ halo) {
  constexpr int H = kSpTile + P - 1, H3 = H * H * H;
  static_assert(H * H <= 256, "one row per thread");
  __shared__ double hb[H3];
  __shared__ double sq[kSpBatch];
  __shared__ int sx[kSpBatch], sy[kSpBatch], sz[kSpBatch];
  __shared__ double sb[kSpBatch][3 * P];
  const int tile = blockIdx.x;
  const int t3 = tile % nt3, t2 = (tile / nt3) % nt2, t1 = tile / (nt2 * nt3);
  const int th = threadIdx.x;
  const bool mine = th < H * H;
  const int l1 = th / H, l2 = th - (th / H) * H;
  if (mine) {
#pragma unroll
    for (int k = 0; k < H; ++k) hb[th * H + k] = 0.;
  }
  const int s0 = start[tile], s1 = start[tile + 1];
  for (int base = s0; base < s1; base += kSpBatch) {
    const int cnt = min(kSpBatch, s1 - base);
    __syncthreads();
    if (th < cnt) {
      const int a = sorted[base + th];
      sq[th] = q[a];
      // the stencil's top corner in the halo box: base cell - tile origin + P - 1
      sx[th] = cell[3 * a] - kSpTile * t1 + P - 1;
      sy[th] = cell[3 * a + 1] - kSpTile * t2 + P - 1;
      sz[th] = cell[3 * a + 2] - kSpTile * t3 + P - 1;
    }
    for (int idx = th; idx < cnt * 3 * P; idx += blockDim.x) {
      const int u = idx / (3 * P), r = idx - u * 3 * P;
      sb[u][r] = spl[(size_t)sorted[base + u] * 6 * P + r];
    }
    __syncthreads();
    if (mine)
      for (int u = 0; u < cnt; ++u) {
        const int a = sx[u] - l1, bb = sy[u] - l2;
        if ((unsigned)a < (unsigned)P && (unsigned)bb < (unsigned)P) {
          const double w = (sq[u] * sb[u][a]) * sb[u][P + bb];
          double *row = hb + th * H + sz[u];  // row[-c], c < P, stays in the row
#pragma unroll
          for (int c = 0; c < P; ++c) row[-c] += w * sb[u][2 * P + c];
        }
      }
  }
  __syncthreads();
  double *out = halo + (size_t)tile * H3;
  for (int u = th; u < H3; u += blockDim.x) out[u] = hb[u];
}

// Phase two: grid point g takes, per dimension, the halo boxes of tiles
// tg + d (d = 0 .. reach - 1, modulo the tile count) at the local coordinate
// g - 8 (tg + d) + p - 1 when that is >= 0.  Writes the real grid and its
// complex copy for the FFT.  Grid (ceil(m2 m3 / blockDim), m1), plane i =
// blockIdx.y.
__global__ void k_spme_halo_gather(int m1, int m2, int m3, int nbsp, int reach, int nt1,
                                   int nt2, int nt3, const double *__restrict__ halo,
                                   double *__restrict__ qsp, cufftDoubleComplex *__restrict__ ft) {
  const int i = blockIdx.y;
  const int t2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (t2 >= m2 * m3) return;
  const long long t = (long long)i * m2 * m3 + t2;
  const int j = t2 / m3, k = t2 - j * m3;
  const int H = kSpTile + nbsp - 1, H3 = H * H * H;
  const int ti = i / kSpTile, tj = j / kSpTile, tk = k / kSpTile;
  double acc = 0.;
  for (int d1 = 0; d1 < reach; ++d1) {
    const int l1 = i - kSpTile * (ti + d1) + nbsp - 1;
    if (l1 < 0) break;
    const int s1 = (ti + d1) % nt1;
    for (int d2 = 0; d2 < reach; ++d2) {
      const int l2 = j - kSpTile * (tj + d2) + nbsp - 1;
      if (l2 < 0) break;
      const int s2 = (tj + d2) % nt2;
      for (int d3 = 0; d3 < reach; ++d3) {
        const int l3 = k - kSpTile * (tk + d3) + nbsp - 1;
        if (l3 < 0) break;
        const int s3 = (tk + d3) % nt3;
        const size_t src = ((size_t)s1 * nt2 + s2) * nt3 + s3;
        acc += halo[src * H3 + ((size_t)l1 * H + l2) * H + l3];
      }
    }
  }
  qsp[t] = acc;
  ft[t] = make_cuDoubleComplex(acc, 0.0);
}

// The same for orders P <= 9 (two halo boxes per dimension at most), fully
// unrolled: same terms, same order.
template <int P>
__global__ void k_spme_halo_gather2(int m2, int m3, int nt1, int nt2, int nt3,
                                    const double *__restrict__ halo, double *__restrict__ qsp,
                                    cufftDoubleComplex *__restrict__ ft) {
  constexpr int H = kSpTile + P - 1, H3 = H * H * H;
  static_assert(P <= 9, "two halo boxes per dimension");
  const int i = blockIdx.y;
  const int t2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (t2 >= m2 * m3) return;
  const long long t = (long long)i * m2 * m3 + t2;
  const int j = t2 / m3, k = t2 - j * m3;
  const int ti = i / kSpTile, tj = j / kSpTile, tk = k / kSpTile;
  // local coordinates in the own tile's box (d = 0) and the next one (d = 1)
  const int l1 = i - kSpTile * ti + P - 1, l2 = j - kSpTile * tj + P - 1,
            l3 = k - kSpTile * tk + P - 1;
  const int u1 = ti + 1 == nt1 ? 0 : ti + 1, u2 = tj + 1 == nt2 ? 0 : tj + 1,
            u3 = tk + 1 == nt3 ? 0 : tk + 1;
  const bool n1 = l1 >= kSpTile, n2 = l2 >= kSpTile, n3 = l3 >= kSpTile;
  double acc = 0.;
#pragma unroll
  for (int d1 = 0; d1 < 2; ++d1) {
    if (d1 == 1 && !n1) break;
    const int s1 = d1 ? u1 : ti, m1l = l1 - kSpTile * d1;
#pragma unroll
    for (int d2 = 0; d2 < 2; ++d2) {
      if (d2 == 1 && !n2) break;
      const int s2 = d2 ? u2 : tj, m2l = l2 - kSpTile * d2;
#pragma unroll
      for (int d3 = 0; d3 < 2; ++d3) {
        if (d3 == 1 && !n3) break;
        const int s3 = d3 ? u3 : tk, m3l = l3 - kSpTile * d3;
        const size_t src = ((size_t)s1 * nt2 + s2) * nt3 + s3;
        acc += halo[src * H3 + (m1l * H + m2l) * H + m3l];
      }
    }
  }
  qsp[t] = acc;
  ft[t] = make_cuDoubleComplex(acc, 0.0);
}

__global__ void k_spme_pack(long long mm, const double *__restrict__ qsp,
                            cufftDoubleComplex *__restrict__ ft) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < mm) ft[t] = make_cuDoubleComplex(qsp[t], 0.0);
}

// The block's sum of v into part[id] (id: the block's linear index; fixed
// reduction order); k_spme_sum adds the blocks' partials in block order:
// run-to-run identical.
__device__ __forceinline__ void block_add(double v, double *part, int id) {
  __shared__ double red[32];
  v = warp_sum_d(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    v = warp_sum_d(v);
    if (lane == 0) part[id] = v;
  }
  __syncthreads();
}

// dst[q] = sum over b of part[q * nb + b], one block per q: thread t adds
// the partials t, t + blockDim, ... in order, then a fixed tree.
__global__ void __launch_bounds__(1024) k_spme_sum(const double *__restrict__ part, int nb,
                                                   double *__restrict__ dst) {
  __shared__ double red[32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double *p = part + (size_t)blockIdx.x * nb;
  double v = 0.;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) v += p[b];
  v = warp_sum_d(v);
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    v = warp_sum_d(v);
    if (lane == 0) dst[blockIdx.x] = v;
  }
}

// Influence function and virial (src/spme.c:460-530); stress[6] += ...
// Grid (ceil(m2 m3 / blockDim), m1): plane i = blockIdx.y, no 64-bit division.
__global__ void k_spme_influence(int m1, int m2, int m3, SpmeBox b, double ralpha2, double rc2,
                                 const double *__restrict__ bmod,  // m1 + m2 + m3
                                 cufftDoubleComplex *__restrict__ ft, double *__restrict__ part) {
  const int i = blockIdx.y;
  const int t2 = blockIdx.x * blockDim.x + threadIdx.x;
  const long long t = (long long)i * m2 * m3 + t2;
  double s[6] = {0., 0., 0., 0., 0., 0.};
  if (t2 < m2 * m3) {
    const int j = t2 / m3, k = t2 - j * m3;
    const int ii = i > m1 / 2 ? i - m1 : i, jj = j > m2 / 2 ? j - m2 : j,
              kk = k > m3 / 2 ? k - m3 : k;
    const double tw = 6.283185307179586;
    const double ti = tw * (double)ii, tj = tw * (double)jj, tk = tw * (double)kk;
    const double rmx = ti * b.u1 + tj * b.v1 + tk * b.w1;
    const double rmy = ti * b.u2 + tj * b.v2 + tk * b.w2;
    const double rmz = ti * b.u3 + tj * b.v3 + tk * b.w3;
    const double rm = rmx * rmx + rmy * rmy + rmz * rmz;
    const double bm = bmod[i] * bmod[m1 + j] * bmod[m1 + m2 + k];
    cufftDoubleComplex f = ft[t];
    if (rm > 2.220446049250313e-16 && rm <= rc2) {
      const double rrm = 1.0 / rm;
      const double a = bm * exp(ralpha2 * rm) * rrm;
      const cufftDoubleComplex cam = make_cuDoubleComplex(a * f.x, a * f.y);
      // creal(cam * conj(f)) = a |f|^2
      const double vam = 2.0 * (rrm - ralpha2) * (cam.x * f.x + cam.y * f.y);
      s[0] = -vam * rmx * rmx;
      s[1] = -vam * rmx * rmy;
      s[2] = -vam * rmx * rmz;
      s[3] = -vam * rmy * rmy;
      s[4] = -vam * rmy * rmz;
      s[5] = -vam * rmz * rmz;
      f = cam;
    } else {
      f = make_cuDoubleComplex(0.0, 0.0);
    }
    ft[t] = f;
  }
  const int nb = gridDim.x * gridDim.y, id = blockIdx.y * gridDim.x + blockIdx.x;
  for (int c = 0; c < 6; ++c) block_add(s[c], part + (size_t)c * nb, id);
}

// Force interpolation (src/spme.c:532-575) into fr[3][n]; sums for the mean.
// MDBas's triple sum over the p^3 grid points of an atom factorises:
//   sum_abc Q(a,b,c) d1_a b2_b b3_c = sum_a d1_a sum_b b2_b sum_c Q b3_c
// (likewise for the y and z parts), so per (a, b) row only the two sums
// over c of Q b3_c and Q d3_c are needed.  `group` lanes (the next power of
// two >= p) share one atom, lane a taking the plane a; the group's three
// partial forces are summed with shuffles.
__global__ void k_spme_forces(int n, int m1, int m2, int m3, int nbsp, int group, SpmeBox b,
                              double fact1, const double *__restrict__ q,
                              const double *__restrict__ spl, const int *__restrict__ cell,
                              const cufftDoubleComplex *__restrict__ ft, double *__restrict__ fr,
                              double *__restrict__ fsum) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int l = (int)(t / group), a = (int)(t % group);
  double px = 0., py = 0., pz = 0.;
  if (l < n && a < nbsp) {
    const double *o = spl + (size_t)l * 6 * nbsp;
    const double *b2 = o + nbsp, *b3 = o + 2 * nbsp;
    const double *d2 = o + 4 * nbsp, *d3 = o + 5 * nbsp;
    const int ii = wrap_index(cell[3 * l] - a, m1);
    const int cy = cell[3 * l + 1], cz = cell[3 * l + 2];
    double t1 = 0., t2 = 0., t3 = 0.;
    for (int bb = 0; bb < nbsp; ++bb) {
      const int jj = wrap_index(cy - bb, m2);
      const size_t base = (size_t)m3 * (jj + (size_t)m2 * ii);
      double sb = 0., sd = 0.;
      for (int c = 0; c < nbsp; ++c) {
        const double qt = ft[base + wrap_index(cz - c, m3)].x;
        sb += qt * __ldg(b3 + c);
        sd += qt * __ldg(d3 + c);
      }
      const double wb = __ldg(b2 + bb);
      t1 += wb * sb;
      t2 += __ldg(d2 + bb) * sb;
      t3 += wb * sd;
    }
    px = __ldg(o + 3 * nbsp + a) * t1;  // d1_a
    const double b1a = __ldg(o + a);
    py = b1a * t2;
    pz = b1a * t3;
  }
  for (int off = group >> 1; off > 0; off >>= 1) {
    px += __shfl_xor_sync(0xffffffffu, px, off);
    py += __shfl_xor_sync(0xffffffffu, py, off);
    pz += __shfl_xor_sync(0xffffffffu, pz, off);
  }
  double fx = 0., fy = 0., fz = 0.;
  if (l < n && a == 0) {
    const double fbx = px * (double)m1, fby = py * (double)m2, fbz = pz * (double)m3;
    const double fq = fact1 * q[l];
    fx = fq * (fbx * b.u1 + fby * b.v1 + fbz * b.w1);
    fy = fq * (fbx * b.u2 + fby * b.v2 + fbz * b.w2);
    fz = fq * (fbx * b.u3 + fby * b.v3 + fbz * b.w3);
    fr[l] = fx;
    fr[n + l] = fy;
    fr[2 * (size_t)n + l] = fz;
  }
  block_add(fx, fsum, blockIdx.x);
  block_add(fy, fsum + gridDim.x, blockIdx.x);
  block_add(fz, fsum + 2 * (size_t)gridDim.x, blockIdx.x);
}

// sum over the grid of Re(theta conv Q) * Q
__global__ void k_spme_energy(long long mm, const cufftDoubleComplex *__restrict__ ft,
                              const double *__restrict__ qsp, double *__restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  block_add(t < mm ? ft[t].x * qsp[t] : 0.0, out, blockIdx.x);
}

// Force interpolation per grid tile (same arithmetic per atom as
// k_spme_forces): the block loads the tile's halo box of the convolved grid
// (real part; local l is grid point 8 t - (p - 1) + l modulo m) into shared
// memory, one warp per row, then takes the bin's atoms, `group` lanes per
// atom.  fsum gets one partial per tile, accumulated in atom order.
template <int P>  // the B-spline order, or 0: given at run time
__global__ void __launch_bounds__(256, 4)  // four blocks per SM (64 registers)
    k_spme_forces_tiled(int n, int m1, int m2, int m3, int nbspRun, int group, int nt2, int nt3,
                        SpmeBox b, double fact1, const double *__restrict__ q,
                        const double *__restrict__ spl, const int *__restrict__ cell,
                        const int *__restrict__ start, const int *__restrict__ sorted,
                        const cufftDoubleComplex *__restrict__ ft, double *__restrict__ fr,
                        double *__restrict__ fsum) {
  extern __shared__ double hb[];
  const int nbsp = P > 0 ? P : nbspRun;
  const int tile = blockIdx.x;
  const int t3 = tile % nt3, t2 = (tile / nt3) % nt2, t1 = tile / (nt2 * nt3);
  const int H = kSpTile + nbsp - 1;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  int g3 = kSpTile * t3 - (nbsp - 1) + lane;
  if (g3 < 0) g3 += m3;
  // four rows per warp in flight
  for (int r0 = w; r0 < H * H; r0 += 4 * nw) {
    double v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = r0 + k * nw;
      v[k] = 0.;
      if (r < H * H && lane < H) {
        const int l1 = r / H, l2 = r - l1 * H;
        int g1 = kSpTile * t1 - (nbsp - 1) + l1, g2 = kSpTile * t2 - (nbsp - 1) + l2;
        if (g1 < 0) g1 += m1;
        if (g2 < 0) g2 += m2;
        v[k] = ft[((size_t)g1 * m2 + g2) * m3 + g3].x;
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = r0 + k * nw;
      if (r < H * H && lane < H) hb[r * H + lane] = v[k];
    }
  }
  __syncthreads();
  const int s0 = start[tile], s1 = start[tile + 1];
  const int per = blockDim.x / group, a = threadIdx.x % group;
  double sx = 0., sy = 0., sz = 0.;
  for (int base = s0; base < s1; base += per) {  // same trip count in the whole block
    const int u = base + (int)threadIdx.x / group;
    const int l = u < s1 ? sorted[u] : -1;
    double px = 0., py = 0., pz = 0.;
    if (l >= 0 && a < nbsp) {
      const double *o = spl + (size_t)l * 6 * nbsp;
      const double *b2 = o + nbsp, *b3 = o + 2 * nbsp;
      const double *d2 = o + 4 * nbsp, *d3 = o + 5 * nbsp;
      const int c1 = cell[3 * l] - kSpTile * t1 + nbsp - 1 - a;  // plane a, local
      const int cy = cell[3 * l + 1] - kSpTile * t2 + nbsp - 1;
      const int cz = cell[3 * l + 2] - kSpTile * t3 + nbsp - 1;
      double t1s = 0., t2s = 0., t3s = 0.;
      if constexpr (P > 0) {
        double rb3[P], rd3[P];
#pragma unroll
        for (int c = 0; c < P; ++c) {
          rb3[c] = __ldg(b3 + c);
          rd3[c] = __ldg(d3 + c);
        }
#pragma unroll
        for (int bb = 0; bb < P; ++bb) {
          const double *row = hb + (c1 * H + cy - bb) * H + cz;
          double sb = 0., sd = 0.;
#pragma unroll
          for (int c = 0; c < P; ++c) {
            const double qt = row[-c];
            sb += qt * rb3[c];
            sd += qt * rd3[c];
          }
          const double wb = __ldg(b2 + bb);
          t1s += wb * sb;
          t2s += __ldg(d2 + bb) * sb;
          t3s += wb * sd;
        }
      } else {
        for (int bb = 0; bb < nbsp; ++bb) {
          const double *row = hb + (c1 * H + cy - bb) * H + cz;
          double sb = 0., sd = 0.;
          for (int c = 0; c < nbsp; ++c) {
            const double qt = row[-c];
            sb += qt * __ldg(b3 + c);
            sd += qt * __ldg(d3 + c);
          }
          const double wb = __ldg(b2 + bb);
          t1s += wb * sb;
          t2s += __ldg(d2 + bb) * sb;
          t3s += wb * sd;
        }
      }
      px = __ldg(o + 3 * nbsp + a) * t1s;  // d1_a
      const double b1a = __ldg(o + a);
      py = b1a * t2s;
      pz = b1a * t3s;
    }
    for (int o = group >> 1; o > 0; o >>= 1) {
      px += __shfl_xor_sync(0xffffffffu, px, o);
      py += __shfl_xor_sync(0xffffffffu, py, o);
      pz += __shfl_xor_sync(0xffffffffu, pz, o);
    }
    if (l >= 0 && a == 0) {
      const double fbx = px * (double)m1, fby = py * (double)m2, fbz = pz * (double)m3;
      const double fq = fact1 * q[l];
      const double fx = fq * (fbx * b.u1 + fby * b.v1 + fbz * b.w1);
      const double fy = fq * (fbx * b.u2 + fby * b.v2 + fbz * b.w2);
      const double fz = fq * (fbx * b.u3 + fby * b.v3 + fbz * b.w3);
      fr[l] = fx;
      fr[n + l] = fy;
      fr[2 * (size_t)n + l] = fz;
      sx += fx;
      sy += fy;
      sz += fz;
    }
  }
  block_add(sx, fsum, blockIdx.x);
  block_add(sy, fsum + gridDim.x, blockIdx.x);
  block_add(sz, fsum + 2 * (size_t)gridDim.x, blockIdx.x);
}

// f += fr - mean (device arrays)
__global__ void k_spme_add(int n, const double *__restrict__ fr, const double *__restrict__ fsum,
                           double *__restrict__ fx, double *__restrict__ fy,
                           double *__restrict__ fz) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const double inv = 1.0 / (double)n;
  fx[l] += fr[l] - fsum[0] * inv;
  fy[l] += fr[n + l] - fsum[1] * inv;
  fz[l] += fr[2 * (size_t)n + l] - fsum[2] * inv;
}

// |bspc|^2 of one dimension (epl_cplx/bspcoef, src/spme.c:170-267).
void bsp_moduli(int m, int nbsp, double *out) {
  std::vector<double> bsp(nbsp, 0.0);
  bsp[1] = 1.0;
  for (int k = 2; k < nbsp; ++k) {
    bsp[k] = 0.0;
    for (int j = k; j > 0; --j) bsp[j] = ((double)j * bsp[j] + (double)(k + 1 - j) * bsp[j - 1]) / k;
  }
  std::vector<std::complex<double>> epl(m);
  epl[0] = 1.0;
  for (int i = 1; i <= m / 2; ++i) {
    epl[i] = std::exp(std::complex<double>(0.0, 6.283185307179586 * (double)i / (double)m));
    epl[m - i] = std::conj(epl[i]);
  }
  for (int i = 0; i < m; ++i) {
    std::complex<double> coeff(0.0, 0.0);
    for (int k = 0; k < nbsp - 1; ++k) coeff += bsp[k + 1] * epl[(size_t)((long long)i * k % m)];
    const std::complex<double> c = epl[(size_t)((long long)i * (nbsp - 1) % m)] / coeff;
    out[i] = std::real(c * std::conj(c));
  }
}

// The standalone calls' state (the engine keeps its own).
SpmeWork &spme_ctx() {
  static SpmeWork c;
  return c;
}

SpmeBox make_spme_box(const PBC *p) {
  SpmeBox b;
  b.u1 = p->u1; b.u2 = p->u2; b.u3 = p->u3;
  b.v1 = p->v1; b.v2 = p->v2; b.v3 = p->v3;
  b.w1 = p->w1; b.w2 = p->w2; b.w3 = p->w3;
  b.u = p->u; b.v = p->v; b.w = p->w;
  b.vol = p->vol;
  return b;
}

int cufft_check(cufftResult r, const char *what) {
  if (r == CUFFT_SUCCESS) return MDBAS_NB_OK;
  char buf[128];
  snprintf(buf, sizeof(buf), "%s failed (cufftResult %d)", what, (int)r);
  set_last_status(MDBAS_NB_ERR_CUDA, buf);
  return MDBAS_NB_ERR_CUDA;
}

// Grid-size dependent state: plan, moduli, grid buffers.
int spme_setup(SpmeWork &c, int n, int m1, int m2, int m3, int nbsp, cudaStream_t s) {
  // planes on the y grid dimension, 32-bit plane and atom indices
  if (m1 > 65535 || (long long)m2 * m3 > (1LL << 30) || n > (1 << 28)) return MDBAS_NB_ERR_ARG;
  int dev = 0;
  MDB_CUDA(cudaGetDevice(&dev));
  const long long mm = (long long)m1 * m2 * m3;
  if (!c.planValid || c.m1 != m1 || c.m2 != m2 || c.m3 != m3 || c.device != dev) {
    if (c.planValid) cufftDestroy(c.plan);
    c.planValid = false;
    MDB_TRY(cufft_check(cufftPlan3d(&c.plan, m1, m2, m3, CUFFT_Z2Z), "cufftPlan3d"));
    c.planValid = true;
    c.m1 = m1;
    c.m2 = m2;
    c.m3 = m3;
    c.device = dev;
    c.nbsp = 0;
    c.haloSmem = 0;  // a function attribute is per device
  }
  MDB_TRY(cufft_check(cufftSetStream(c.plan, s), "cufftSetStream"));
  if (c.nbsp != nbsp) {
    std::vector<double> bm(m1 + m2 + m3);
    bsp_moduli(m1, nbsp, bm.data());
    bsp_moduli(m2, nbsp, bm.data() + m1);
    bsp_moduli(m3, nbsp, bm.data() + m1 + m2);
    MDB_TRY(c.bmod.ensure(sizeof(double) * bm.size()));
    MDB_CUDA(cudaMemcpy(c.bmod.p, bm.data(), sizeof(double) * bm.size(), cudaMemcpyHostToDevice));
    c.nbsp = nbsp;
  }
  MDB_TRY(c.qsp.ensure(sizeof(double) * mm));
  MDB_TRY(c.ft.ensure(sizeof(cufftDoubleComplex) * mm));
  MDB_TRY(c.spl.ensure(sizeof(double) * 6 * (size_t)nbsp * n));
  MDB_TRY(c.cell.ensure(sizeof(int) * 3 * (size_t)n));
  MDB_TRY(c.fr.ensure(sizeof(double) * 3 * (size_t)n));
  MDB_TRY(c.sums.ensure(sizeof(double) * 16));
  {
    // per-block partial sums: influence (6 x blocks), forces (3 x blocks),
    // energy (1 x blocks)
    const long long gI = ((long long)m2 * m3 + 255) / 256 * m1, gF = ((long long)n * 16 + 127) / 128;
    const long long nt = (long long)(m1 / 8) * (m2 / 8) * (m3 / 8);
    MDB_TRY(c.part.ensure(sizeof(double) * (size_t)std::max(6 * gI, 3 * std::max(gF, nt))));
  }
  {
    const int nt = (m1 / 8) * (m2 / 8) * (m3 / 8);
    MDB_TRY(c.tileOf.ensure(sizeof(int) * (size_t)n));
    MDB_TRY(c.tileList.ensure(sizeof(int) * (size_t)n));
    MDB_TRY(c.tileSorted.ensure(sizeof(int) * (size_t)n));
    MDB_TRY(c.tileCount.ensure(sizeof(int) * (size_t)(nt + 1)));
    MDB_TRY(c.tileStart.ensure(sizeof(int) * (size_t)(nt + 1)));
    MDB_TRY(c.tileFill.ensure(sizeof(int) * (size_t)(nt + 1)));
    MDB_TRY(c.scanTmp.ensure(scan_tmp_bytes(nt > 0 ? nt : 1)));
    if (nt > 0) {
      const int H = kSpTile + nbsp - 1;
      const int smem = (int)sizeof(double) * H * H * H;
      MDB_TRY(c.halo.ensure(sizeof(double) * (size_t)nt * H * H * H));
      if (smem > c.haloSmem) {  // set once, before any capture of these launches
        MDB_CUDA(cudaFuncSetAttribute(k_spme_spread_halo<1>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        MDB_CUDA(cudaFuncSetAttribute(k_spme_spread_halo<kSpPts>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        MDB_CUDA(cudaFuncSetAttribute(k_spme_forces_tiled<0>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        c.haloSmem = smem;
      }
    }
  }
  c.n = n;
  return MDBAS_NB_OK;
}

// The whole computation on device arrays; forces (minus their mean) are added
// to fx/fy/fz; out[0] = reciprocal energy + self + non-neutral, out[1] =
// virial, out[2..7] = stress (MDBas's 6-component layout).
int spme_launch_impl(SpmeWork &c, int n, const PBC *box, double alpha, double chargeConst,
                     int m1, int m2, int m3, int nbsp, const double *x, const double *y,
                     const double *z, const double *q, double *fx, double *fy, double *fz,
                     cudaStream_t s) {
  MDB_TRY(spme_setup(c, n, m1, m2, m3, nbsp, s));
  const SpmeBox b = make_spme_box(box);
  const long long mm = (long long)m1 * m2 * m3;
  double *sums = c.sums.as<double>();  // 0-5 stress, 6-8 force sums, 9 energy
  MDB_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * 16, s));
  {
    const int g = grid_for(3LL * n, 128);
    double *spl = c.spl.as<double>();
    int *cel = c.cell.as<int>();
    if (nbsp == 8)
      MDB_LAUNCH(k_spme_splines<8>, g, 128, 0, s, n, b, m1, m2, m3, nbsp, x, y, z, spl, cel);
    else if (nbsp == 6)
      MDB_LAUNCH(k_spme_splines<6>, g, 128, 0, s, n, b, m1, m2, m3, nbsp, x, y, z, spl, cel);
    else if (nbsp == 4)
      MDB_LAUNCH(k_spme_splines<4>, g, 128, 0, s, n, b, m1, m2, m3, nbsp, x, y, z, spl, cel);
    else
      MDB_LAUNCH(k_spme_splines<0>, g, 128, 0, s, n, b, m1, m2, m3, nbsp, x, y, z, spl, cel);
  }
  const bool tiled = m1 % kSpTile == 0 && m2 % kSpTile == 0 && m3 % kSpTile == 0;
  const int nt1 = m1 / kSpTile, nt2 = m2 / kSpTile, nt3 = m3 / kSpTile;
  const int nt = nt1 * nt2 * nt3;
  if (tiled) {
    // deterministic: bins of atoms per 8^3 tile, one block per tile
    const int reach = 1 + (nbsp + kSpTile - 2) / kSpTile;  // halo boxes covering a point, per dim
    int *cnt = c.tileCount.as<int>();
    MDB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(nt + 1), s));
    MDB_CUDA(cudaMemsetAsync(c.tileFill.p, 0, sizeof(int) * (size_t)nt, s));
    MDB_LAUNCH(k_spme_tile_count, grid_for(n, 256), 256, 0, s, n, m1, m2, m3, nt2, nt3,
               c.cell.as<int>(),
               c.tileOf.as<int>(), cnt);
    MDB_TRY(exclusive_scan32(cnt, c.tileStart.as<int>(), nt, c.scanTmp.p, s));
    MDB_LAUNCH(k_spme_tile_fill, grid_for(n, 256), 256, 0, s, n, c.tileOf.as<int>(),
               c.tileStart.as<int>(), c.tileFill.as<int>(), c.tileList.as<int>());
    MDB_LAUNCH(k_spme_tile_sort, nt, 64, 0, s, c.tileStart.as<int>(), c.tileList.as<int>(),
               c.tileSorted.as<int>());
    const int H = kSpTile + nbsp - 1;
    const int *tst = c.tileStart.as<int>(), *tso = c.tileSorted.as<int>();
    const double *spl = c.spl.as<double>();
    const int *cel = c.cell.as<int>();
    double *hal = c.halo.as<double>();
    if (nbsp == 8)
      MDB_LAUNCH(k_spme_spread_rows<8>, nt, 256, 0, s, nt2, nt3, q, spl, cel, tst, tso, hal);
    else if (nbsp == 6)
      MDB_LAUNCH(k_spme_spread_rows<6>, nt, 256, 0, s, nt2, nt3, q, spl, cel, tst, tso, hal);
    else if (nbsp == 4)
      MDB_LAUNCH(k_spme_spread_rows<4>, nt, 256, 0, s, nt2, nt3, q, spl, cel, tst, tso, hal);
    else if (nbsp <= 8)
      MDB_LAUNCH(k_spme_spread_halo<1>, nt, 512, sizeof(double) * H * H * H, s, nbsp, nt2, nt3,
                 q, c.spl.as<double>(), c.cell.as<int>(), c.tileStart.as<int>(),
                 c.tileSorted.as<int>(), c.halo.as<double>());
    else
      MDB_LAUNCH(k_spme_spread_halo<kSpPts>, nt, 512, sizeof(double) * H * H * H, s, nbsp, nt2,
                 nt3, q, c.spl.as<double>(), c.cell.as<int>(), c.tileStart.as<int>(),
                 c.tileSorted.as<int>(), c.halo.as<double>());
    const dim3 gg(grid_for((long long)m2 * m3, 256), m1);
    double *qs = c.qsp.as<double>();
    cufftDoubleComplex *fc = c.ft.as<cufftDoubleComplex>();
    if (nbsp == 8)
      MDB_LAUNCH(k_spme_halo_gather2<8>, gg, 256, 0, s, m2, m3, nt1, nt2, nt3, hal, qs, fc);
    else if (nbsp == 6)
      MDB_LAUNCH(k_spme_halo_gather2<6>, gg, 256, 0, s, m2, m3, nt1, nt2, nt3, hal, qs, fc);
    else if (nbsp == 4)
      MDB_LAUNCH(k_spme_halo_gather2<4>, gg, 256, 0, s, m2, m3, nt1, nt2, nt3, hal, qs, fc);
    else
      MDB_LAUNCH(k_spme_halo_gather, gg, 256, 0, s, m1, m2, m3, nbsp, reach, nt1, nt2, nt3, hal,
                 qs, fc);
  } else {
    MDB_CUDA(cudaMemsetAsync(c.qsp.p, 0, sizeof(double) * mm, s));
    MDB_LAUNCH(k_spme_spread, grid_for((long long)n * nbsp, 128), 128, 0, s, n, m1, m2, m3,
               nbsp, q, c.spl.as<double>(), c.cell.as<int>(), c.qsp.as<double>());
    MDB_LAUNCH(k_spme_pack, grid_for(mm, 256), 256, 0, s, mm, c.qsp.as<double>(),
               c.ft.as<cufftDoubleComplex>());
  }
  cufftDoubleComplex *ft = c.ft.as<cufftDoubleComplex>();
  MDB_TRY(cufft_check(cufftExecZ2Z(c.plan, ft, ft, CUFFT_INVERSE), "cufftExecZ2Z"));
  const double rvol = 6.283185307179586 / b.vol;
  const double ralpha2 = -0.25 / (alpha * alpha);
  double rc = fmin((double)m1 * b.u, (double)m2 * b.v);
  rc = fmin(rc, (double)m3 * b.w) * 1.05 * 6.283185307179586;
  const int gx = grid_for((long long)m2 * m3, 256), gI = gx * m1, gE = grid_for(mm, 256);
  double *part = c.part.as<double>();
  MDB_LAUNCH(k_spme_influence, dim3(gx, m1), 256, 0, s, m1, m2, m3, b, ralpha2, rc * rc,
             c.bmod.as<double>(), ft, part);
  MDB_LAUNCH(k_spme_sum, 6, 1024, 0, s, part, gI, sums);
  MDB_TRY(cufft_check(cufftExecZ2Z(c.plan, ft, ft, CUFFT_FORWARD), "cufftExecZ2Z"));
  int group = 1;
  while (group < nbsp) group <<= 1;
  if (tiled) {
    const int H = kSpTile + nbsp - 1;
    const size_t smem = sizeof(double) * H * H * H;
    const double f2 = -2.0 * rvol * chargeConst;
    const int *tst = c.tileStart.as<int>(), *tso = c.tileSorted.as<int>();
    const double *spl = c.spl.as<double>();
    const int *cel = c.cell.as<int>();
    double *frr = c.fr.as<double>();
    if (nbsp == 8)
      MDB_LAUNCH(k_spme_forces_tiled<8>, nt, 256, smem, s, n, m1, m2, m3, nbsp, group, nt2, nt3,
                 b, f2, q, spl, cel, tst, tso, ft, frr, part);
    else if (nbsp == 6)
      MDB_LAUNCH(k_spme_forces_tiled<6>, nt, 256, smem, s, n, m1, m2, m3, nbsp, group, nt2, nt3,
                 b, f2, q, spl, cel, tst, tso, ft, frr, part);
    else if (nbsp == 4)
      MDB_LAUNCH(k_spme_forces_tiled<4>, nt, 256, smem, s, n, m1, m2, m3, nbsp, group, nt2, nt3,
                 b, f2, q, spl, cel, tst, tso, ft, frr, part);
    else
      MDB_LAUNCH(k_spme_forces_tiled<0>, nt, 256, smem, s, n, m1, m2, m3, nbsp, group, nt2, nt3,
                 b, f2, q, spl, cel, tst, tso, ft, frr, part);
    MDB_LAUNCH(k_spme_sum, 3, 1024, 0, s, part, nt, sums + 6);
  } else {
    const int gF = grid_for((long long)n * group, 128);
    MDB_LAUNCH(k_spme_forces, gF, 128, 0, s, n, m1, m2, m3, nbsp, group, b,
               -2.0 * rvol * chargeConst, q, c.spl.as<double>(), c.cell.as<int>(), ft,
               c.fr.as<double>(), part);
    MDB_LAUNCH(k_spme_sum, 3, 1024, 0, s, part, gF, sums + 6);
  }
  MDB_LAUNCH(k_spme_energy, gE, 256, 0, s, mm, ft, c.qsp.as<double>(), part);
  MDB_LAUNCH(k_spme_sum, 1, 1024, 0, s, part, gE, sums + 9);
  MDB_LAUNCH(k_spme_add, grid_for(n, 256), 256, 0, s, n, c.fr.as<double>(), sums + 6, fx, fy,
             fz);
  c.f1 = rvol * chargeConst;
  return MDBAS_NB_OK;
}

int spme_run(int n, const PBC *box, double alpha, double chargeConst, int m1, int m2, int m3,
             int nbsp, const double *x, const double *y, const double *z, const double *q,
             double systq, double sumq2, double *fx, double *fy, double *fz, double out[8],
             cudaStream_t s) {
  SpmeWork &c = spme_ctx();
  MDB_TRY(spme_launch_impl(c, n, box, alpha, chargeConst, m1, m2, m3, nbsp, x, y, z, q, fx, fy,
                           fz, s));
  const SpmeBox b = make_spme_box(box);
  const double rvol = 6.283185307179586 / b.vol;
  double *sums = c.sums.as<double>();
  double h[16];
  MDB_CUDA(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  const double eself = -chargeConst * alpha * sumq2 / kSqrtPi;
  const double enn = -(0.5 * 3.141592653589793 * chargeConst) *
                     ((systq / alpha) * (systq / alpha) / b.vol);
  const double fact1 = rvol * chargeConst;
  const double erec = h[9];
  double st[6];
  st[0] = fact1 * (h[0] + erec) + enn;
  st[1] = fact1 * h[1];
  st[2] = fact1 * h[2];
  st[3] = fact1 * (h[3] + erec) + enn;
  st[4] = fact1 * h[4];
  st[5] = fact1 * (h[5] + erec) + enn;
  out[0] = fact1 * erec + eself + enn;
  out[1] = -(st[0] + st[3] + st[5]);
  for (int k = 0; k < 6; ++k) out[2 + k] = st[k];
  return MDBAS_NB_OK;
}

int check_grid(int m1, int m2, int m3, int nbsp) {
  if (m1 <= 0 || m2 <= 0 || m3 <= 0 || nbsp < 2 || nbsp > kMaxOrder) return MDBAS_NB_ERR_ARG;
  if (nbsp > m1 || nbsp > m2 || nbsp > m3) return MDBAS_NB_ERR_ARG;
  return MDBAS_NB_OK;
}

int nint_h(double x) { return (x >= 0.) ? (int)(x + 0.5) : (int)(x - 0.5); }

}  // namespace

int mdbas::spme_launch(SpmeWork &c, int n, const PBC *box, double alpha, double chargeConst,
                       int m1, int m2, int m3, int nbsp, const double *x, const double *y,
                       const double *z, const double *q, double *fx, double *fy, double *fz,
                       cudaStream_t s) {
  return spme_launch_impl(c, n, box, alpha, chargeConst, m1, m2, m3, nbsp, x, y, z, q, fx, fy, fz,
                          s);
}

extern "C" {

int mdbas_nb_spme(int nAtom, const PBC *box, double alpha, double chargeConst, int m1, int m2,
                  int m3, int nbsp, const double *x, const double *y, const double *z,
                  const double *q, double *fx, double *fy, double *fz, double out[8],
                  int device_ptrs, void *stream) {
  if (nAtom <= 0 || !box || !x || !y || !z || !q || !fx || !fy || !fz || !out || !(alpha > 0.))
    return MDBAS_NB_ERR_ARG;
  MDB_TRY(check_grid(m1, m2, m3, nbsp));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  SpmeWork &c = spme_ctx();
  double systq = 0., sumq2 = 0.;
  std::vector<double> hq;
  const double *qh = q;
  if (device_ptrs) {
    hq.resize(nAtom);
    MDB_CUDA(cudaMemcpy(hq.data(), q, sizeof(double) * nAtom, cudaMemcpyDeviceToHost));
    qh = hq.data();
  }
  for (int i = 0; i < nAtom; ++i) {
    systq += qh[i];
    sumq2 += qh[i] * qh[i];
  }
  if (device_ptrs)
    return spme_run(nAtom, box, alpha, chargeConst, m1, m2, m3, nbsp, x, y, z, q, systq, sumq2,
                    fx, fy, fz, out, s);
  // host arrays: stage through device buffers; forces are added to the
  // caller's arrays
  MDB_TRY(c.xyzq.ensure(sizeof(double) * 4 * (size_t)nAtom));
  MDB_TRY(c.fout.ensure(sizeof(double) * 3 * (size_t)nAtom));
  double *d = c.xyzq.as<double>(), *f = c.fout.as<double>();
  const size_t bytes = sizeof(double) * nAtom;
  MDB_CUDA(cudaMemcpyAsync(d, x, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d + nAtom, y, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d + 2 * (size_t)nAtom, z, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d + 3 * (size_t)nAtom, q, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemsetAsync(f, 0, 3 * bytes, s));
  MDB_TRY(spme_run(nAtom, box, alpha, chargeConst, m1, m2, m3, nbsp, d, d + nAtom,
                   d + 2 * (size_t)nAtom, d + 3 * (size_t)nAtom, systq, sumq2, f, f + nAtom,
                   f + 2 * (size_t)nAtom, out, s));
  std::vector<double> hf(3 * (size_t)nAtom);
  MDB_CUDA(cudaMemcpy(hf.data(), f, 3 * bytes, cudaMemcpyDeviceToHost));
  for (int i = 0; i < nAtom; ++i) {
    fx[i] += hf[i];
    fy[i] += hf[nAtom + i];
    fz[i] += hf[2 * (size_t)nAtom + i];
  }
  return MDBAS_NB_OK;
}

// MDBas's init_spme (src/spme.c:32-68): the grid of the reciprocal sum.
void init_spme(CTRL *ctrl, PARAM *param, EWALD *ewald, PBC *box) {
  ewald->prec = fmin(fabs(ewald->prec), 0.5);
  ewald->tol = sqrt(fabs(log(ewald->prec * param->cutOff)));
  if (!ctrl->keyAlpha)
    ewald->alpha = sqrt(fabs(log(ewald->prec * param->cutOff * ewald->tol))) / param->cutOff;
  const double ta = 2.0 * ewald->tol * ewald->alpha;
  ewald->tol1 = sqrt(-log(ewald->prec * param->cutOff * (ta * ta)));
  if (!ctrl->keyMmax) {
    ewald->m1max = nint_h(0.25 + box->pa * ewald->alpha * ewald->tol1 / 3.141592653589793);
    ewald->m2max = nint_h(0.25 + box->pb * ewald->alpha * ewald->tol1 / 3.141592653589793);
    ewald->m3max = nint_h(0.25 + box->pc * ewald->alpha * ewald->tol1 / 3.141592653589793);
  }
  int *m[3] = {&ewald->m1max, &ewald->m2max, &ewald->m3max};
  for (int d = 0; d < 3; ++d) {
    int p2 = 1;
    while (*m[d] > p2 && p2 < 256) p2 *= 2;
    *m[d] = 2 * p2;
  }
  ewald->mmax = ewald->m1max * ewald->m2max * ewald->m3max;
}

void spme_free(PARAM *param) { (void)param; }

// MDBas's spme_energy (src/spme.c:357-700) on the GPU.  As in MDBas the
// mean over the whole force arrays is removed after the reciprocal forces
// are added (energy() calls it first, on zeroed arrays).
double spme_energy(PARAM *param, EWALD *ewald, PBC *box, const double x[], const double y[],
                   const double z[], double fx[], double fy[], double fz[], const double q[],
                   double stress[6], double *virEwaldRec) {
  const int n = param->nAtom;
  std::vector<double> rx(n, 0.), ry(n, 0.), rz(n, 0.);
  double out[8];
  const int st = mdbas_nb_spme(n, box, ewald->alpha, param->chargeConst, ewald->m1max,
                               ewald->m2max, ewald->m3max, ewald->nbsp, x, y, z, q, rx.data(),
                               ry.data(), rz.data(), out, 0, nullptr);
  if (st != MDBAS_NB_OK) {
    fprintf(stderr, "spme_energy (GPU): %s: %s\n", mdbas_nb_status_string(st),
            mdbas_nb_last_message());
    exit(1);
  }
  double mx = 0., my = 0., mz = 0.;
  for (int i = 0; i < n; ++i) {
    fx[i] += rx[i];
    fy[i] += ry[i];
    fz[i] += rz[i];
    mx += fx[i];
    my += fy[i];
    mz += fz[i];
  }
  // rx had its own mean removed; MDBas removes the mean of the whole array
  mx /= (double)n;
  my /= (double)n;
  mz /= (double)n;
  for (int i = 0; i < n; ++i) {
    fx[i] -= mx;
    fy[i] -= my;
    fz[i] -= mz;
  }
  for (int k = 0; k < 6; ++k) stress[k] = out[2 + k];
  *virEwaldRec = out[1];
  return out[0];
}

}  // extern "C"
