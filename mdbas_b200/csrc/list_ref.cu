// list_ref.cu -- MDBas-format half Verlet lists built on the GPU.
//
// Two builders with MDBas's exact output (same entries in the same order):
//
//  * link cells (link_cell_verlet_list[_update], src/list.c:1793-2619): atoms
//    are binned with MDBas's FP64 fractional coordinates; each cell lists its
//    atoms in descending index (MDBas's LIFO head/link chains); neighOrder is
//    that cell-major order; atom i scans the stencil cells in table order
//    (link_stencil.h) and, in its own cell, only the atoms after it.
//  * all pairs (verlet_list[_update], src/list.c:896-1123): j = i+1..N-1 with
//    MDBas's dist() minimum image; neighOrder is the identity.
//
// Layout: after binning, positions/fractional coordinates are gathered into
// cell order so that a warp scanning a cell reads consecutive addresses.  One
// warp owns one atom i: lanes test 32 consecutive candidates, a ballot gives
// the survivors and their order, so the fill pass writes j in exactly the
// order MDBas's serial loop does.  Each builder runs a count pass, a scan
// of the counts in neighOrder order (entry offsets) and a fill pass.
//
// All distance arithmetic uses __dadd_rn/__dmul_rn (no FMA contraction) in
// MDBas's association order, so every r^2 <= (rc+delr)^2 decision is the
// one MDBas's x86 build makes.
#include "common.cuh"
#include "link_stencil.h"
#include "list_ref.cuh"

namespace mdbas {

namespace {

__constant__ int c_stencil[LINK_STENCIL_MAX * 3];

__device__ __forceinline__ bool excluded_pair(int i, int j, const int *__restrict__ exclStart,
                                              const int *__restrict__ exclFlat) {
  const int e = exclStart[i + 1];
  for (int k = exclStart[i]; k < e; ++k)
    if (__ldg(exclFlat + k) == j) return true;
  return false;
}

// image_update (src/utils.c:162-218), in place.
__global__ void k_image_update(int n, DevBox b, double *x, double *y, double *z) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xi = x[i], yi = y[i], zi = z[i];
  image_d(b, xi, yi, zi);
  x[i] = xi;
  y[i] = yi;
  z[i] = zi;
}

// Fractional coordinates + 0.5 (src/list.c:1932-1937) and the link cell
// (src/list.c:1943-1955): truncation toward zero, clamped above only.
__global__ void k_lc_bin(int n, DevBox b, int nlcx, int nlcy, int nlcz,
                         const double *__restrict__ x, const double *__restrict__ y,
                         const double *__restrict__ z, double *__restrict__ xu,
                         double *__restrict__ yu, double *__restrict__ zu,
                         int *__restrict__ cellOf, int *__restrict__ cellCount,
                         int *__restrict__ flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = x[i], yi = y[i], zi = z[i];
  const double a = dadd(dadd(dadd(dmul(xi, b.u1), dmul(yi, b.u2)), dmul(zi, b.u3)), 0.5);
  const double c = dadd(dadd(dadd(dmul(xi, b.v1), dmul(yi, b.v2)), dmul(zi, b.v3)), 0.5);
  const double d = dadd(dadd(dadd(dmul(xi, b.w1), dmul(yi, b.w2)), dmul(zi, b.w3)), 0.5);
  xu[i] = a;
  yu[i] = c;
  zu[i] = d;
  if (!(isfinite(a) && isfinite(c) && isfinite(d))) {
    atomicOr(flags, FLAG_NONFINITE);
    cellOf[i] = -1;
    return;
  }
  int ix = __double2int_rz(dmul((double)nlcx, a));
  int iy = __double2int_rz(dmul((double)nlcy, c));
  int iz = __double2int_rz(dmul((double)nlcz, d));
  ix = min(ix, nlcx - 1);
  iy = min(iy, nlcy - 1);
  iz = min(iz, nlcz - 1);
  if (ix < 0 || iy < 0 || iz < 0) {
    // MDBas would index head[] out of bounds here; report instead.
    atomicOr(flags, FLAG_OUTSIDE);
    cellOf[i] = -1;
    return;
  }
  const int cell = ix + nlcx * (iy + nlcy * iz);
  cellOf[i] = cell;
  atomicAdd(cellCount + cell, 1);
}

__global__ void k_lc_scatter(int n, const int *__restrict__ cellOf,
                             const int *__restrict__ cellStart, int *__restrict__ cellFill,
                             int *__restrict__ tmpIdx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cellOf[i];
  if (c < 0) return;
  const int slot = atomicAdd(cellFill + c, 1);
  tmpIdx[cellStart[c] + slot] = i;
}

// Order each cell's atoms by descending index (MDBas's LIFO chain order):
// the rank of a member is the number of members with a larger index.
__global__ void k_lc_order(int ncell, const int *__restrict__ cellStart,
                           const int *__restrict__ tmpIdx, int *__restrict__ sortedIdx) {
  __shared__ int chunk[1024];
  const int c = blockIdx.x;
  if (c >= ncell) return;
  const int s = cellStart[c], e = cellStart[c + 1];
  for (int base = s; base < e; base += blockDim.x) {
    const int m = base + threadIdx.x;
    const int mine = (m < e) ? tmpIdx[m] : -1;
    int rank = 0;
    for (int cb = s; cb < e; cb += 1024) {
      const int cnt = min(1024, e - cb);
      __syncthreads();
      for (int t = threadIdx.x; t < cnt; t += blockDim.x) chunk[t] = tmpIdx[cb + t];
      __syncthreads();
      if (m < e)
        for (int t = 0; t < cnt; ++t) rank += (chunk[t] > mine);
    }
    if (m < e) sortedIdx[s + rank] = mine;
  }
}

__global__ void k_lc_gather(int n, const int *__restrict__ sortedIdx,
                            const double *__restrict__ xu, const double *__restrict__ yu,
                            const double *__restrict__ zu, const int *__restrict__ frozen,
                            double *__restrict__ xs, double *__restrict__ ys,
                            double *__restrict__ zs, int *__restrict__ fs,
                            int *__restrict__ posOf) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = sortedIdx[p];
  xs[p] = xu[i];
  ys[p] = yu[i];
  zs[p] = zu[i];
  fs[p] = frozen ? frozen[i] : 0;
  posOf[i] = p;
}

// One warp per atom (in neighOrder position p).  FILL=false: count entries
// into cnt[p] and neighPair[i].  FILL=true: write them at off[p].
template <bool FILL>
__global__ void __launch_bounds__(256)
k_lc_pairs(int n, DevBox b, int nlcx, int nlcy, int nlcz, int cellCheck, double cutnb2,
           const int *__restrict__ sortedIdx, const int *__restrict__ cellOf,
           const int *__restrict__ cellStart, const double *__restrict__ xs,
           const double *__restrict__ ys, const double *__restrict__ zs,
           const int *__restrict__ fs, const int *__restrict__ exclStart,
           const int *__restrict__ exclFlat, int *__restrict__ cnt, int *__restrict__ neighPair,
           const long long *__restrict__ off, int *__restrict__ list) {
  const int lane = threadIdx.x & 31;
  const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (p >= n) return;
  const int i = sortedIdx[p];
  const int k = cellOf[i];
  const int ix = k % nlcx, iy = (k / nlcx) % nlcy, iz = k / (nlcx * nlcy);
  const double xi = xs[p], yi = ys[p], zi = zs[p];
  const int fi = fs[p];
  long long out = FILL ? off[p] : 0;
  int count = 0;
  for (int l = 0; l < cellCheck; ++l) {
    int jx = ix + c_stencil[3 * l], jy = iy + c_stencil[3 * l + 1], jz = iz + c_stencil[3 * l + 2];
    double cx = 0., cy = 0., cz = 0.;
    if (jx > nlcx - 1) { jx -= nlcx; cx = 1.; } else if (jx < 0) { jx += nlcx; cx = -1.; }
    if (jy > nlcy - 1) { jy -= nlcy; cy = 1.; } else if (jy < 0) { jy += nlcy; cy = -1.; }
    if (jz > nlcz - 1) { jz -= nlcz; cz = 1.; } else if (jz < 0) { jz += nlcz; cz = -1.; }
    const int ll = jx + nlcx * (jy + nlcy * jz);
    const int lo = (ll == k) ? p + 1 : cellStart[ll];
    const int hi = cellStart[ll + 1];
    for (int base = lo; base < hi; base += 32) {
      const int q = base + lane;
      bool pass = false;
      int j = -1;
      if (q < hi) {
        j = sortedIdx[q];
        const double xt = dadd(dsub(xs[q], xi), cx);
        const double yt = dadd(dsub(ys[q], yi), cy);
        const double zt = dadd(dsub(zs[q], zi), cz);
        const double xd = dadd(dadd(dmul(xt, b.a1), dmul(yt, b.b1)), dmul(zt, b.c1));
        const double yd = dadd(dadd(dmul(xt, b.a2), dmul(yt, b.b2)), dmul(zt, b.c2));
        const double zd = dadd(dadd(dmul(xt, b.a3), dmul(yt, b.b3)), dmul(zt, b.c3));
        const double r2 = dadd(dadd(dmul(xd, xd), dmul(yd, yd)), dmul(zd, zd));
        pass = (r2 <= cutnb2) && (fi * fs[q] == 0) && !excluded_pair(i, j, exclStart, exclFlat);
      }
      const unsigned m = __ballot_sync(0xffffffffu, pass);
      if (FILL && pass) list[out + __popc(m & ((1u << lane) - 1u))] = j;
      out += __popc(m);
      count += __popc(m);
    }
  }
  if (!FILL && lane == 0) {
    cnt[p] = count;
    neighPair[i] = count;
  }
}

// All-pairs builder: one warp per atom i < n-1, candidates j = i+1..n-1.
template <bool FILL>
__global__ void __launch_bounds__(256)
k_vl_pairs(int n, DevBox b, double cutnb2, const double *__restrict__ x,
           const double *__restrict__ y, const double *__restrict__ z,
           const int *__restrict__ frozen, const int *__restrict__ exclStart,
           const int *__restrict__ exclFlat, int *__restrict__ cnt, int *__restrict__ neighPair,
           const long long *__restrict__ off, int *__restrict__ list) {
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  const double xi = x[i], yi = y[i], zi = z[i];
  const int fi = frozen ? frozen[i] : 0;
  long long out = FILL ? off[i] : 0;
  int count = 0;
  for (int base = i + 1; base < n; base += 32) {
    const int j = base + lane;
    bool pass = false;
    if (j < n) {
      double dx = dsub(x[j], xi), dy = dsub(y[j], yi), dz = dsub(z[j], zi);
      const double r2 = dist_d(b, dx, dy, dz);
      const int fj = frozen ? frozen[j] : 0;
      pass = (r2 <= cutnb2) && (fi * fj == 0) && !excluded_pair(i, j, exclStart, exclFlat);
    }
    const unsigned m = __ballot_sync(0xffffffffu, pass);
    if (FILL && pass) list[out + __popc(m & ((1u << lane) - 1u))] = j;
    out += __popc(m);
    count += __popc(m);
  }
  if (!FILL && lane == 0) {
    cnt[i] = count;
    neighPair[i] = count;
  }
}

__global__ void k_iota(int n, int *v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

__global__ void k_gather_counts(int n, const int *__restrict__ order,
                                const int *__restrict__ neighPair, int *__restrict__ cnt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) cnt[p] = neighPair[order[p]];
}

bool g_stencil_loaded[64];

int load_stencil() {
  int dev = 0;
  MDB_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && g_stencil_loaded[dev]) return MDBAS_NB_OK;
  int flat[LINK_STENCIL_MAX * 3];
  for (int l = 0; l < LINK_STENCIL_MAX; ++l)
    for (int d = 0; d < 3; ++d) flat[3 * l + d] = LINK_STENCIL[l][d];
  MDB_CUDA(cudaMemcpyToSymbol(c_stencil, flat, sizeof(flat)));
  if (dev >= 0 && dev < 64) g_stencil_loaded[dev] = true;
  return MDBAS_NB_OK;
}

int read_flags(const int *dflags, cudaStream_t s, int *h) {
  MDB_CUDA(cudaMemcpyAsync(h, dflags, sizeof(int), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  return MDBAS_NB_OK;
}

}  // namespace

int image_update_device(int n, const DevBox &b, double *x, double *y, double *z, cudaStream_t s) {
  if (n <= 0) return MDBAS_NB_OK;
  MDB_LAUNCH(k_image_update, grid_for(n, 256), 256, 0, s, n, b, x, y, z);
  return MDBAS_NB_OK;
}

int link_cell_dims(const DevBox &b, double cutOff, double delr, int linkRatio, int nlc[3]) {
  const double cutnb = cutOff + delr;
  nlc[0] = (int)(b.pa * (double)linkRatio / cutnb);
  nlc[1] = (int)(b.pb * (double)linkRatio / cutnb);
  nlc[2] = (int)(b.pc * (double)linkRatio / cutnb);
  return MDBAS_NB_OK;
}

int makelist_uses_link_cells(const DevBox &b, double cutOff, double delr, int linkRatio,
                             int noLink) {
  // makelist (src/list.c:40-57)
  int nlc[3];
  int r = linkRatio < 1 ? 1 : (linkRatio > 5 ? 5 : linkRatio);
  link_cell_dims(b, cutOff, delr, r, nlc);
  if (nlc[0] < 3 || nlc[1] < 3 || nlc[2] < 3) return 0;
  if (nlc[0] * nlc[1] * nlc[2] <= 27) return 0;
  if (noLink) return 0;
  return 1;
}

int build_ref_list(RefListWork &w, int n, const DevBox &b, double cutOff, double delr,
                   int linkRatio, int linkCells, const double *x, const double *y,
                   const double *z, const int *frozen, const int *exclStart,
                   const int *exclFlat, cudaStream_t s) {
  if (n <= 0) {
    w.entries = 0;
    return MDBAS_NB_OK;
  }
  const double cutnb = cutOff + delr;
  const double cutnb2 = cutnb * cutnb;
  w.linkCells = linkCells;
  MDB_TRY(w.neighPair.ensure(sizeof(int) * n));
  MDB_TRY(w.order.ensure(sizeof(int) * n));
  MDB_TRY(w.cnt.ensure(sizeof(int) * n));
  MDB_TRY(w.off.ensure(sizeof(long long) * (n + 1)));
  MDB_TRY(w.scanTmp.ensure(scan_tmp_bytes(n + 1)));
  MDB_TRY(w.flags.ensure(sizeof(int) * 4));
  MDB_CUDA(cudaMemsetAsync(w.flags.p, 0, sizeof(int) * 4, s));

  if (linkCells) {
    MDB_TRY(load_stencil());
    int r = linkRatio < 1 ? 1 : (linkRatio > 5 ? 5 : linkRatio);
    link_cell_dims(b, cutOff, delr, r, w.nlc);
    if (w.nlc[0] < 2 * r + 1 || w.nlc[1] < 2 * r + 1 || w.nlc[2] < 2 * r + 1)
      return MDBAS_NB_ERR_LINKCELL;  // LNKCELL_NCELLS_ERROR, src/list.c:1900-1908
    const int ncell = w.nlc[0] * w.nlc[1] * w.nlc[2];
    w.ncell = ncell;
    const int cellCheck = LINK_STENCIL_COUNT[r - 1];
    MDB_TRY(w.xu.ensure(sizeof(double) * n));
    MDB_TRY(w.yu.ensure(sizeof(double) * n));
    MDB_TRY(w.zu.ensure(sizeof(double) * n));
    MDB_TRY(w.xs.ensure(sizeof(double) * n));
    MDB_TRY(w.ys.ensure(sizeof(double) * n));
    MDB_TRY(w.zs.ensure(sizeof(double) * n));
    MDB_TRY(w.fs.ensure(sizeof(int) * n));
    MDB_TRY(w.cellOf.ensure(sizeof(int) * n));
    MDB_TRY(w.posOf.ensure(sizeof(int) * n));
    MDB_TRY(w.tmpIdx.ensure(sizeof(int) * n));
    MDB_TRY(w.cellCount.ensure(sizeof(int) * (ncell + 1)));
    MDB_TRY(w.cellFill.ensure(sizeof(int) * (ncell + 1)));
    MDB_TRY(w.cellStart.ensure(sizeof(int) * (ncell + 2)));
    MDB_TRY(w.scanTmp.ensure(scan_tmp_bytes(ncell + 1) > scan_tmp_bytes(n + 1)
                                 ? scan_tmp_bytes(ncell + 1)
                                 : scan_tmp_bytes(n + 1)));
    MDB_CUDA(cudaMemsetAsync(w.cellCount.p, 0, sizeof(int) * (ncell + 1), s));
    MDB_CUDA(cudaMemsetAsync(w.cellFill.p, 0, sizeof(int) * (ncell + 1), s));
    MDB_LAUNCH(k_lc_bin, grid_for(n, 256), 256, 0, s, n, b, w.nlc[0], w.nlc[1], w.nlc[2], x, y,
               z, w.xu.as<double>(), w.yu.as<double>(), w.zu.as<double>(), w.cellOf.as<int>(),
               w.cellCount.as<int>(), w.flags.as<int>());
    int hflags = 0;
    MDB_TRY(read_flags(w.flags.as<int>(), s, &hflags));
    if (hflags & FLAG_NONFINITE) return MDBAS_NB_ERR_NONFINITE;
    if (hflags & FLAG_OUTSIDE) return MDBAS_NB_ERR_BOX;
    MDB_TRY(exclusive_scan32(w.cellCount.as<int>(), w.cellStart.as<int>(), ncell,
                             w.scanTmp.p, s));
    MDB_LAUNCH(k_lc_scatter, grid_for(n, 256), 256, 0, s, n, w.cellOf.as<int>(),
               w.cellStart.as<int>(), w.cellFill.as<int>(), w.tmpIdx.as<int>());
    MDB_LAUNCH(k_lc_order, ncell, 256, 0, s, ncell, w.cellStart.as<int>(), w.tmpIdx.as<int>(),
               w.order.as<int>());
    MDB_LAUNCH(k_lc_gather, grid_for(n, 256), 256, 0, s, n, w.order.as<int>(), w.xu.as<double>(),
               w.yu.as<double>(), w.zu.as<double>(), frozen, w.xs.as<double>(),
               w.ys.as<double>(), w.zs.as<double>(), w.fs.as<int>(), w.posOf.as<int>());
    const int blocks = grid_for((long long)n * 32, 256);
    MDB_LAUNCH(k_lc_pairs<false>, blocks, 256, 0, s, n, b, w.nlc[0], w.nlc[1], w.nlc[2],
               cellCheck, cutnb2, w.order.as<int>(), w.cellOf.as<int>(), w.cellStart.as<int>(),
               w.xs.as<double>(), w.ys.as<double>(), w.zs.as<double>(), w.fs.as<int>(),
               exclStart, exclFlat, w.cnt.as<int>(), w.neighPair.as<int>(),
               (const long long *)nullptr, (int *)nullptr);
    MDB_TRY(exclusive_scan(w.cnt.as<int>(), w.off.as<long long>(), n, w.scanTmp.p, s));
    long long total = 0;
    MDB_CUDA(cudaMemcpyAsync(&total, w.off.as<long long>() + n, sizeof(long long),
                             cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaStreamSynchronize(s));
    w.entries = total;
    if (total > 0x7fffffffLL) return MDBAS_NB_ERR_CAPACITY;  // MDBas's int list index
    MDB_TRY(w.list.ensure(sizeof(int) * (size_t)(total > 0 ? total : 1)));
    MDB_LAUNCH(k_lc_pairs<true>, blocks, 256, 0, s, n, b, w.nlc[0], w.nlc[1], w.nlc[2],
               cellCheck, cutnb2, w.order.as<int>(), w.cellOf.as<int>(), w.cellStart.as<int>(),
               w.xs.as<double>(), w.ys.as<double>(), w.zs.as<double>(), w.fs.as<int>(),
               exclStart, exclFlat, w.cnt.as<int>(), w.neighPair.as<int>(),
               w.off.as<long long>(), w.list.as<int>());
  } else {
    w.ncell = 0;
    MDB_LAUNCH(k_iota, grid_for(n, 256), 256, 0, s, n, w.order.as<int>());
    const int blocks = grid_for((long long)n * 32, 256);
    MDB_LAUNCH(k_vl_pairs<false>, blocks, 256, 0, s, n, b, cutnb2, x, y, z, frozen, exclStart,
               exclFlat, w.cnt.as<int>(), w.neighPair.as<int>(), (const long long *)nullptr,
               (int *)nullptr);
    MDB_TRY(exclusive_scan(w.cnt.as<int>(), w.off.as<long long>(), n, w.scanTmp.p, s));
    long long total = 0;
    MDB_CUDA(cudaMemcpyAsync(&total, w.off.as<long long>() + n, sizeof(long long),
                             cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaStreamSynchronize(s));
    w.entries = total;
    if (total > 0x7fffffffLL) return MDBAS_NB_ERR_CAPACITY;
    MDB_TRY(w.list.ensure(sizeof(int) * (size_t)(total > 0 ? total : 1)));
    MDB_LAUNCH(k_vl_pairs<true>, blocks, 256, 0, s, n, b, cutnb2, x, y, z, frozen, exclStart,
               exclFlat, w.cnt.as<int>(), w.neighPair.as<int>(), w.off.as<long long>(),
               w.list.as<int>());
  }
  return MDBAS_NB_OK;
}

int ref_list_offsets(RefListWork &w, int n, cudaStream_t s) {
  // Entry offsets of a list supplied by the caller (neighPair/order on the
  // device): exclusive scan of neighPair in neighOrder order.
  MDB_TRY(w.cnt.ensure(sizeof(int) * n));
  MDB_TRY(w.off.ensure(sizeof(long long) * (n + 1)));
  MDB_TRY(w.scanTmp.ensure(scan_tmp_bytes(n + 1)));
  MDB_LAUNCH(k_gather_counts, grid_for(n, 256), 256, 0, s, n, w.order.as<int>(),
             w.neighPair.as<int>(), w.cnt.as<int>());
  MDB_TRY(exclusive_scan(w.cnt.as<int>(), w.off.as<long long>(), n, w.scanTmp.p, s));
  return MDBAS_NB_OK;
}

}  // namespace mdbas
