// dropin.cu -- MDBas's energy.c / list.c entry points, backed by the GPU.
//
// A MDBas build links libmdbas_nb.so in place of obj/energy.o and
// obj/list.o.  The prototypes are MDBas's (include/energy.h, include/list.h);
// the caller owns every array, list builders allocate the list arrays with
// malloc and grow them with realloc exactly as MDBas does, energy routines
// accumulate into the caller's force arrays.  The bonded terms of
// internal.o (bond_energy ... improper_energy, bonded.cu) and the k-space
// sums of ewald.o and spme.o (ewald_rec.cu, spme.cu) are the library's own,
// on the GPU.  Routines MDBas keeps in other objects (freeze_atoms in
// utils.o, my_error in errors.o, the outFile global of mdbas.o) are reached
// through weak references; when a routine the call needs is absent (e.g. the
// library is loaded into another program), the call fails with
// MDBAS_NB_ERR_MISSING.
//
// Errors: the void drop-ins report like MDBas's my_error (src/errors.c:15)
// -- through my_error itself when it is linked, with MDBas's error number
// where one exists -- and terminate; the mdbas_nb_*_status forms return the
// status instead.
//
// Single-threaded, like MDBas: one process-wide context holds the device
// copies of the last system seen.
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "cluster.cuh"
#include "engine.cuh"
#include "list_ref.cuh"
#include "pair_fp32.cuh"
#include "pair_fp64.cuh"

using namespace mdbas;

// ---------------------------------------------------------------------------
// MDBas routines reached through weak references.
// ---------------------------------------------------------------------------
extern "C" {
extern FILE *outFile __attribute__((weak));
void my_error(int errorNumber, char file[], int line, int num_optional_args, ...)
    __attribute__((weak));
void freeze_atoms(const PARAM *param, double *vx, double *vy, double *vz, double *fx, double *fy,
                  double *fz, const int *frozen) __attribute__((weak));
}

namespace {

// MDBas error numbers (include/errors.h) for statuses that have one.
int mdbas_error_number(int st) {
  switch (st) {
    case MDBAS_NB_ERR_ALLOC: return 1;      // MEM_ALLOC_ERROR
    case MDBAS_NB_ERR_LINKCELL: return 412; // LNKCELL_NCELLS_ERROR
    case MDBAS_NB_ERR_EXCL: return 111;     // EXCLLIST_LASTATOM_ERROR
    default: return 0;
  }
}

FILE *report_stream() { return (&outFile && outFile) ? outFile : stderr; }

[[noreturn]] void fail(int st, const char *where, int mdbas_code = 0) {
  set_last_status(st, nullptr);
  const int code = mdbas_code ? mdbas_code : mdbas_error_number(st);
  if (code && my_error) {
    char file[] = "libmdbas_nb";
    my_error(code, file, 0, 0);  // prints MDBas's message and exits
  }
  FILE *f = report_stream();
  fprintf(f, "MDBas failed due to error number: %d\n", code ? code : 500 + st);
  fprintf(f, "libmdbas_nb: %s in %s", mdbas_nb_status_string(st), where);
  const char *m = mdbas_nb_last_message();
  if (m && m[0]) fprintf(f, " (%s)", m);
  fprintf(f, "\n");
  fflush(f);
  exit(code ? code : 500 + st);
}

#define DROP_TRY(expr, where)                                                  \
  do {                                                                         \
    int s__ = (expr);                                                          \
    if (s__ != MDBAS_NB_OK) fail(s__, where);                                  \
  } while (0)

#define ST_TRY(expr)                                                           \
  do {                                                                         \
    int s__ = (expr);                                                          \
    if (s__ != MDBAS_NB_OK) {                                                  \
      set_last_status(s__, nullptr);                                           \
      return s__;                                                              \
    }                                                                          \
  } while (0)

// ---------------------------------------------------------------------------
// Process-wide context.
// ---------------------------------------------------------------------------
struct Ctx {
  bool ready = false;
  int device = 0;
  cudaStream_t s = nullptr;
  int n = 0;
  DBuf x, y, z, q, eps, sig, frozen, exclStart, exclFlat, f3, acc64, list14;
  // the exclusion rows made symmetric for the cluster search
  DBuf exclStartSym, exclFlatSym;
  std::vector<double> hq, heps, hsig;
  std::vector<int> hExclStart, hExclFlat, hFrozen, hExclStartSym, hExclFlatSym;
  bool hasFrozen = false;
  RefListWork ref;
  ClusterWork cl;
  // The device list equals the caller's host list while these match.
  // The device copy of a MDBas-format list stays resident between calls only
  // when this library's own builder wrote it (resOwned) into the caller's
  // arrays and those arrays still hold what it wrote: same pointers, same
  // counts and the same checksum of neighPair and of a sample of the list.  A
  // list built elsewhere (MDBas's own list.c behind the plugin entry) is
  // uploaded on every call, since its builder may refill the same arrays in
  // place (src/list.c:2276-2279, 2565-2574).
  const int *resList = nullptr, *resPair = nullptr, *resOrder = nullptr;
  long long resEntries = -1;
  int resN = -1;
  bool resOwned = false;
  unsigned long long resSum = 0;
  // mixed mode: positions at the last cluster build (displacement check)
  std::vector<double> bx, by, bz;
  bool clValid = false;
  bool clMoved = false;  // positions changed since the last cluster build
  DevBox clBox{};
  int elecType = FULL, vdwType = VSWITCH;
  bool ptrsSet = false;
  // page-locked staging for the positions going up and the forces coming
  // down (the caller's arrays are pageable), grown on demand
  double *pinIn = nullptr, *pinOut = nullptr;
  size_t pinInCap = 0, pinOutCap = 0;
};

Ctx g;

int ctx_init() {
  if (g.ready) return MDBAS_NB_OK;
  const char *d = getenv("MDBAS_NB_DEVICE");
  g.device = d ? atoi(d) : 0;
  ST_TRY(engine_check_device(g.device));
  MDB_CUDA(cudaSetDevice(g.device));
  MDB_CUDA(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking));
  g.ready = true;
  return MDBAS_NB_OK;
}

bool resident_enabled() {
  const char *v = getenv("MDBAS_NB_LIST_RESIDENT");
  return !(v && v[0] == '0');
}

// Page-locked host buffer of at least `count` doubles.  Every call that uses
// one ends with a stream synchronisation, so a buffer is never refilled while
// a copy from or into it is in flight.
int pinned(double *&buf, size_t &cap, size_t count) {
  if (cap >= count && buf) return MDBAS_NB_OK;
  if (buf) cudaFreeHost(buf);
  buf = nullptr;
  cap = 0;
  MDB_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&buf), sizeof(double) * count,
                         cudaHostAllocDefault));
  cap = count;
  return MDBAS_NB_OK;
}

int upload_positions(int n, const double *x, const double *y, const double *z) {
  ST_TRY(g.x.ensure(sizeof(double) * n));
  ST_TRY(g.y.ensure(sizeof(double) * n));
  ST_TRY(g.z.ensure(sizeof(double) * n));
  ST_TRY(pinned(g.pinIn, g.pinInCap, 3 * (size_t)n));
  double *h = g.pinIn;
  memcpy(h, x, sizeof(double) * n);
  memcpy(h + n, y, sizeof(double) * n);
  memcpy(h + 2 * (size_t)n, z, sizeof(double) * n);
  MDB_CUDA(cudaMemcpyAsync(g.x.p, h, sizeof(double) * n, cudaMemcpyHostToDevice, g.s));
  MDB_CUDA(cudaMemcpyAsync(g.y.p, h + n, sizeof(double) * n, cudaMemcpyHostToDevice, g.s));
  MDB_CUDA(cudaMemcpyAsync(g.z.p, h + 2 * (size_t)n, sizeof(double) * n,
                           cudaMemcpyHostToDevice, g.s));
  return MDBAS_NB_OK;
}

int upload_vec(DBuf &d, std::vector<double> &cache, const double *h, int n) {
  if ((int)cache.size() == n && memcmp(cache.data(), h, sizeof(double) * n) == 0 && d.p)
    return MDBAS_NB_OK;
  cache.assign(h, h + n);
  ST_TRY(d.ensure(sizeof(double) * n));
  MDB_CUDA(cudaMemcpyAsync(d.p, cache.data(), sizeof(double) * n, cudaMemcpyHostToDevice, g.s));
  g.clValid = false;  // the cluster layout holds charges and LJ parameters
  return MDBAS_NB_OK;
}

int upload_params(int n, const double *q, const double *eps, const double *sig) {
  if (q) ST_TRY(upload_vec(g.q, g.hq, q, n));
  if (eps) ST_TRY(upload_vec(g.eps, g.heps, eps, n));
  if (sig) ST_TRY(upload_vec(g.sig, g.hsig, sig, n));
  return MDBAS_NB_OK;
}

// MDBas exclusion rows (exclList[i][0..exclPair[i]-1]) -> device CSR.
int upload_exclusions(int n, int **exclList, const int *exclPair) {
  // rows as last uploaded (MDBas builds them once per run): compared in place
  if (g.exclStart.p && (int)g.hExclStart.size() == n + 1) {
    bool same = true;
    if (exclPair) {
      for (int i = 0; i < n && same; ++i) {
        const int s0 = g.hExclStart[i], c = exclPair[i];
        if (g.hExclStart[i + 1] - s0 != c) {
          same = false;
          break;
        }
        const int *row = exclList[i];
        for (int k = 0; k < c; ++k)
          if (row[k] != g.hExclFlat[s0 + k]) {
            same = false;
            break;
          }
      }
    } else {
      same = g.hExclStart[n] == 0;
    }
    if (same) return MDBAS_NB_OK;
  }
  std::vector<int> start(n + 1, 0), flat;
  if (exclPair) {
    for (int i = 0; i < n; ++i) start[i + 1] = start[i] + exclPair[i];
    flat.resize(start[n]);
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < exclPair[i]; ++k) flat[start[i] + k] = exclList[i][k];
  }
  if (start == g.hExclStart && flat == g.hExclFlat && g.exclStart.p) return MDBAS_NB_OK;
  g.hExclStart.swap(start);
  g.hExclFlat.swap(flat);
  ST_TRY(g.exclStart.ensure(sizeof(int) * (n + 1)));
  ST_TRY(g.exclFlat.ensure(sizeof(int) * std::max<size_t>(1, g.hExclFlat.size())));
  MDB_CUDA(cudaMemcpyAsync(g.exclStart.p, g.hExclStart.data(), sizeof(int) * (n + 1),
                           cudaMemcpyHostToDevice, g.s));
  if (!g.hExclFlat.empty())
    MDB_CUDA(cudaMemcpyAsync(g.exclFlat.p, g.hExclFlat.data(), sizeof(int) * g.hExclFlat.size(),
                             cudaMemcpyHostToDevice, g.s));
  // MDBas's all-pairs builder keeps half rows; the cluster search checks the
  // rows of the i cluster's atoms only, so it reads both directions
  cluster_symmetric_excl(n, g.hExclStart.data(), g.hExclFlat.data(), g.hExclStartSym,
                         g.hExclFlatSym);
  ST_TRY(g.exclStartSym.ensure(sizeof(int) * (n + 1)));
  ST_TRY(g.exclFlatSym.ensure(sizeof(int) * std::max<size_t>(1, g.hExclFlatSym.size())));
  MDB_CUDA(cudaMemcpyAsync(g.exclStartSym.p, g.hExclStartSym.data(), sizeof(int) * (n + 1),
                           cudaMemcpyHostToDevice, g.s));
  if (!g.hExclFlatSym.empty())
    MDB_CUDA(cudaMemcpyAsync(g.exclFlatSym.p, g.hExclFlatSym.data(),
                             sizeof(int) * g.hExclFlatSym.size(), cudaMemcpyHostToDevice, g.s));
  g.clValid = false;
  return MDBAS_NB_OK;
}

int upload_frozen(int n, const int *frozen) {
  bool any = false;
  if (frozen)
    for (int i = 0; i < n && !any; ++i) any = frozen[i] != 0;
  if (!any) {
    if (g.hasFrozen) g.clValid = false;
    g.hasFrozen = false;
    return MDBAS_NB_OK;
  }
  if (g.hasFrozen && (int)g.hFrozen.size() == n &&
      memcmp(g.hFrozen.data(), frozen, sizeof(int) * n) == 0)
    return MDBAS_NB_OK;
  g.hFrozen.assign(frozen, frozen + n);
  ST_TRY(g.frozen.ensure(sizeof(int) * n));
  MDB_CUDA(cudaMemcpyAsync(g.frozen.p, g.hFrozen.data(), sizeof(int) * n, cudaMemcpyHostToDevice,
                           g.s));
  g.hasFrozen = true;
  g.clValid = false;
  return MDBAS_NB_OK;
}

void print_grow(int from, int to) {
  FILE *f = report_stream();
  fprintf(f, "WARNING: List larger than estimated. Size increased from %d to %d.\n", from, to);
}

// FNV-1a style hash of neighPair and of every 61st list entry plus the last
// ones: a guard against arrays refilled since the library's build.
unsigned long long list_checksum(int n, const int *neighList, const int *neighPair,
                                 long long total) {
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&h](unsigned v) { h = (h ^ v) * 1099511628211ull; };
  for (int i = 0; i < n; ++i) mix((unsigned)neighPair[i]);
  for (long long k = 0; k < total; k += 61) mix((unsigned)neighList[k]);
  for (long long k = total > 64 ? total - 64 : 0; k < total; ++k) mix((unsigned)neighList[k]);
  return h;
}

// Build MDBas's list on the device and hand it to the caller's arrays.
//   first != 0: allocate *neighList / *neighPair / *neighOrder (first build);
//   first == 0: reuse them, growing *neighList by MDBas's 1% steps.
int list_common(int linkCells, int first, PARAM *param, PBC *box, NEIGH *neigh, double x[],
                double y[], double z[], int frozen[], int **neighList, int **neighPair,
                int **neighOrder, int *neighPairArr, int *neighOrderArr, int **exclList,
                int exclPair[]) {
  ST_TRY(ctx_init());
  const int n = param->nAtom;
  if (n <= 0) return MDBAS_NB_ERR_ARG;
  const DevBox b = make_devbox(box);
  if (linkCells) {
    neigh->linkRatio = std::min(std::max(neigh->linkRatio, 1), 5);
    int nlc[3];
    link_cell_dims(b, param->cutOff, param->delr, neigh->linkRatio, nlc);
    const int r = neigh->linkRatio;
    if (nlc[0] < 2 * r + 1 || nlc[1] < 2 * r + 1 || nlc[2] < 2 * r + 1)
      return MDBAS_NB_ERR_LINKCELL;
    neigh->nCells = nlc[0] * nlc[1] * nlc[2];
  }
  ST_TRY(upload_positions(n, x, y, z));
  if (linkCells && first) {
    // image_update (src/list.c:1927): wrap in place, caller's arrays too
    ST_TRY(image_update_device(n, b, g.x.as<double>(), g.y.as<double>(), g.z.as<double>(), g.s));
    MDB_CUDA(cudaMemcpyAsync(x, g.x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, g.s));
    MDB_CUDA(cudaMemcpyAsync(y, g.y.p, sizeof(double) * n, cudaMemcpyDeviceToHost, g.s));
    MDB_CUDA(cudaMemcpyAsync(z, g.z.p, sizeof(double) * n, cudaMemcpyDeviceToHost, g.s));
  }
  ST_TRY(upload_frozen(n, frozen));
  ST_TRY(upload_exclusions(n, exclList, exclPair));
  ST_TRY(build_ref_list(g.ref, n, b, param->cutOff, param->delr, neigh->linkRatio, linkCells,
                        g.x.as<double>(), g.y.as<double>(), g.z.as<double>(),
                        g.hasFrozen ? g.frozen.as<int>() : nullptr, g.exclStart.as<int>(),
                        g.exclFlat.as<int>(), g.s));
  const long long total = g.ref.entries;
  int *pairArr, *orderArr;
  if (first) {
    // sizeList = (int)(count * (1 + 2 TOLLIST)) + 1 (src/list.c:985, :2110)
    neigh->sizeList = (int)((double)total * (1. + 2. * kTolList)) + 1;
    *neighPair = (int *)malloc(sizeof(int) * n);
    *neighOrder = (int *)malloc(sizeof(int) * n);
    *neighList = (int *)malloc(sizeof(int) * (size_t)neigh->sizeList);
    if (!*neighPair || !*neighOrder || !*neighList) return MDBAS_NB_ERR_ALLOC;
    pairArr = *neighPair;
    orderArr = *neighOrder;
  } else {
    // grow by 1% (+1) while the entries do not fit (src/list.c:2567-2574)
    if (total > neigh->sizeList) {
      int size = neigh->sizeList;
      while ((long long)size < total) {
        const int next = (int)((double)size * (1. + kTolList)) + 1;
        print_grow(size, next);
        size = next;
      }
      int *p = (int *)realloc(*neighList, sizeof(int) * (size_t)size);
      if (!p) return MDBAS_NB_ERR_ALLOC;
      *neighList = p;
      neigh->sizeList = size;
    }
    pairArr = neighPairArr;
    orderArr = neighOrderArr;
  }
  if (total > 0)
    MDB_CUDA(cudaMemcpyAsync(*neighList, g.ref.list.p, sizeof(int) * total,
                             cudaMemcpyDeviceToHost, g.s));
  MDB_CUDA(cudaMemcpyAsync(pairArr, g.ref.neighPair.p, sizeof(int) * n, cudaMemcpyDeviceToHost,
                           g.s));
  if (orderArr)
    MDB_CUDA(cudaMemcpyAsync(orderArr, g.ref.order.p, sizeof(int) * n, cudaMemcpyDeviceToHost,
                             g.s));
  MDB_CUDA(cudaStreamSynchronize(g.s));
  g.resList = *neighList;
  g.resPair = pairArr;
  g.resOrder = orderArr;
  g.resEntries = total;
  g.resN = n;
  g.resOwned = orderArr != nullptr;
  g.resSum = list_checksum(n, *neighList, pairArr, total);
  return MDBAS_NB_OK;
}

// Bring the caller's list to the device unless it is the one this library
// built and still holds what the build wrote.
int ensure_list_on_device(int n, const int *neighList, const int *neighPair,
                          const int *neighOrder) {
  long long total = 0;
  for (int i = 0; i < n; ++i) total += neighPair[i];
  if (resident_enabled() && g.resOwned && neighList == g.resList && neighPair == g.resPair &&
      neighOrder == g.resOrder && total == g.resEntries && n == g.resN && g.ref.off.p &&
      list_checksum(n, neighList, neighPair, total) == g.resSum)
    return MDBAS_NB_OK;
  ST_TRY(g.ref.list.ensure(sizeof(int) * (size_t)std::max<long long>(1, total)));
  ST_TRY(g.ref.neighPair.ensure(sizeof(int) * n));
  ST_TRY(g.ref.order.ensure(sizeof(int) * n));
  if (total > 0)
    MDB_CUDA(cudaMemcpyAsync(g.ref.list.p, neighList, sizeof(int) * total, cudaMemcpyHostToDevice,
                             g.s));
  MDB_CUDA(cudaMemcpyAsync(g.ref.neighPair.p, neighPair, sizeof(int) * n, cudaMemcpyHostToDevice,
                           g.s));
  MDB_CUDA(cudaMemcpyAsync(g.ref.order.p, neighOrder, sizeof(int) * n, cudaMemcpyHostToDevice,
                           g.s));
  ST_TRY(ref_list_offsets(g.ref, n, g.s));
  g.resList = neighList;
  g.resPair = neighPair;
  g.resOrder = neighOrder;
  g.resEntries = total;
  g.resN = n;
  g.resOwned = false;  // a caller-built list: uploaded again on the next call
  return MDBAS_NB_OK;
}

// Download device forces and add them into the caller's arrays.
int add_forces(int n, const double *dsrc, double *fx, double *fy, double *fz) {
  ST_TRY(pinned(g.pinOut, g.pinOutCap, 3 * (size_t)n));
  MDB_CUDA(cudaMemcpyAsync(g.pinOut, dsrc, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost,
                           g.s));
  MDB_CUDA(cudaStreamSynchronize(g.s));
  const double *h = g.pinOut;
  for (int i = 0; i < n; ++i) {
    fx[i] += h[i];
    fy[i] += h[n + i];
    fz[i] += h[2 * n + i];
  }
  return MDBAS_NB_OK;
}

// What the cluster list needs for these positions: a rebuild (max
// displacement since the last build beyond half the skin, or no list), a
// refresh of the FP32 layout (moved, within half the skin), or nothing (the
// build's own positions: the inner list written by the build still holds).
enum ClusterNeed { CL_NEED_NONE = 0, CL_NEED_REFRESH = 1, CL_NEED_REBUILD = 2 };
int cluster_need(int n, const double *x, const double *y, const double *z, const DevBox &b,
                 double delr) {
  if (!g.clValid || (int)g.bx.size() != n) return CL_NEED_REBUILD;
  if (memcmp(&b, &g.clBox, sizeof(DevBox)) != 0) return CL_NEED_REBUILD;
  // one pass: the largest displacement since the build (minimum image, only
  // components beyond half a box are wrapped) and whether any atom moved
  const double lim2 = 0.25 * delr * delr;
  const double L[3] = {b.a1, b.type == CUBIC ? b.a1 : b.b2, b.type == CUBIC ? b.a1 : b.c3};
  const double h[3] = {0.5 * L[0], 0.5 * L[1], 0.5 * L[2]};
  const double *cur[3] = {x, y, z};
  const double *ref[3] = {g.bx.data(), g.by.data(), g.bz.data()};
  bool moved = false;
  for (int i = 0; i < n; ++i) {
    double r2 = 0.;
    for (int k = 0; k < 3; ++k) {
      double d = cur[k][i] - ref[k][i];
      moved |= d != 0.0;
      if (fabs(d) > h[k]) d -= L[k] * rint(d / L[k]);
      r2 += d * d;
    }
    if (r2 > lim2) return CL_NEED_REBUILD;
  }
  if (!moved) return g.clMoved ? CL_NEED_REFRESH : CL_NEED_NONE;
  return CL_NEED_REFRESH;
}

// The real-space work of ewald_energy (or the plugin): forces added into
// fx/fy/fz; e[0..5] = eDir, eCorr, evdw, virDir, virCorr, virvdw.
int real_space(int mode, int listRule, int n, const PARAM *param, double alpha, int vdwSwitch,
               const PBC *box,
               const double *x, const double *y, const double *z, double *fx, double *fy,
               double *fz, const double *q, const double *eps, const double *sig,
               const int *neighList, const int *neighPair, const int *neighOrder,
               int **exclList, const int *exclPair, const int *frozen, double e[6]) {
  ST_TRY(ctx_init());
  const DevBox b = make_devbox(box);
  const PairParams p = make_params(param->cutOff, param->cutOn, alpha, param->chargeConst,
                                   vdwSwitch, FULL);
  ST_TRY(upload_positions(n, x, y, z));
  ST_TRY(upload_params(n, q, eps, sig));
  ST_TRY(upload_exclusions(n, exclList, exclPair));
  ST_TRY(g.f3.ensure(sizeof(double) * 3 * (size_t)n));
  ST_TRY(g.acc64.ensure(sizeof(double) * kFp64AccCount));
  if (mode == 0 || b.type == TCLIN) {
    ST_TRY(ensure_list_on_device(n, neighList, neighPair, neighOrder));
    MDB_CUDA(cudaMemsetAsync(g.f3.p, 0, sizeof(double) * 3 * (size_t)n, g.s));
    MDB_CUDA(cudaMemsetAsync(g.acc64.p, 0, sizeof(double) * kFp64AccCount, g.s));
    double *fxd = g.f3.as<double>(), *fyd = fxd + n, *fzd = fyd + n;
    ST_TRY(pairs_fp64(1, n, b, p, g.ref.order.as<int>(), g.ref.neighPair.as<int>(),
                      g.ref.off.as<long long>(), g.ref.list.as<int>(), g.x.as<double>(),
                      g.y.as<double>(), g.z.as<double>(), g.q.as<double>(), g.eps.as<double>(),
                      g.sig.as<double>(), fxd, fyd, fzd, g.acc64.as<double>(), g.s));
    ST_TRY(excl_fp64(n, b, p, g.exclStart.as<int>(), g.exclFlat.as<int>(), g.x.as<double>(),
                     g.y.as<double>(), g.z.as<double>(), g.q.as<double>(), fxd, fyd, fzd,
                     g.acc64.as<double>(), g.s));
    double a[kFp64AccCount];
    MDB_CUDA(cudaMemcpyAsync(a, g.acc64.p, sizeof(a), cudaMemcpyDeviceToHost, g.s));
    ST_TRY(add_forces(n, g.f3.as<double>(), fx, fy, fz));
    e[0] = a[0];
    e[1] = a[5];
    e[2] = a[1];
    e[3] = a[2];
    e[4] = a[6];
    e[5] = a[3];
    return MDBAS_NB_OK;
  }
  // mixed precision over the library's own cluster-pair list
  ST_TRY(upload_frozen(n, frozen));
  const int need = cluster_need(n, x, y, z, b, param->delr);
  if (need == CL_NEED_REBUILD) {
    ST_TRY(cluster_build(g.cl, n, b, param->cutOff, param->delr, listRule,
                         sqrt(param->chargeConst), g.x.as<double>(), g.y.as<double>(),
                         g.z.as<double>(), g.q.as<double>(), g.eps.as<double>(),
                         g.sig.as<double>(), g.hasFrozen ? g.frozen.as<int>() : nullptr,
                         g.exclStartSym.as<int>(), g.exclFlatSym.as<int>(), g.s));
    g.bx.assign(x, x + n);
    g.by.assign(y, y + n);
    g.bz.assign(z, z + n);
    g.clBox = b;
    g.clValid = true;
    g.clMoved = false;
  } else if (need == CL_NEED_REFRESH) {
    ST_TRY(cluster_refresh(g.cl, g.x.as<double>(), g.y.as<double>(), g.z.as<double>(),
                           g.q.as<double>(), sqrt(param->chargeConst), g.s));
    g.clMoved = true;
  }
  ClusterWork &w = g.cl;
  MDB_CUDA(cudaMemsetAsync(w.facc.p, 0, sizeof(long long) * 3 * (size_t)w.slotCap, g.s));
  MDB_CUDA(cudaMemsetAsync(w.acc.p, 0, sizeof(long long) * ACC_COUNT, g.s));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g.device);
  ST_TRY(pair_fp32_launch(w, p, sms * 8, 256, g.s));
  ST_TRY(excl_fix_launch(w, n, p, g.exclStartSym.as<int>(), g.exclFlatSym.as<int>(),
                         g.x.as<double>(), g.y.as<double>(), g.z.as<double>(), g.q.as<double>(),
                         g.s));
  double *fxd = g.f3.as<double>();
  ST_TRY(forces_out_launch(w, n, 0, fxd, fxd + n, fxd + 2 * (size_t)n, g.s));
  long long a[ACC_COUNT];
  MDB_CUDA(cudaMemcpyAsync(a, w.acc.p, sizeof(a), cudaMemcpyDeviceToHost, g.s));
  ST_TRY(add_forces(n, fxd, fx, fy, fz));
  if (a[ACC_FLAGS] & FLAG_OVERFLOW) return MDBAS_NB_ERR_OVERFLOW;
  const double inv = 1.0 / kEnergyScale;
  e[0] = (double)a[ACC_E_DIR] * inv;
  e[1] = (double)a[ACC_E_CORR] * inv;
  e[2] = (double)a[ACC_E_VDW] * inv;
  e[3] = (double)a[ACC_V_DIR] * inv;
  e[4] = (double)a[ACC_V_CORR] * inv;
  e[5] = (double)a[ACC_V_VDW] * inv;
  return MDBAS_NB_OK;
}

// ---------------------------------------------------------------------------
// Host exclusion builders: exclude_list (src/list.c:108-894) and
// link_cell_exclude_list (src/list.c:1125-1791).  Rows are filled in MDBas's
// order: bonds, constraints (keyConstH), angles, dihedrals (recording the a-d
// pair as a 1-4 pair when it is new), impropers, then the bond-graph walk
// (1-3 pairs, and 1-4 pairs recorded in neighList14).  The half form stores
// (min, max) once and checks duplicates in the lower atom's row; the
// symmetric form stores both directions and checks the first atom's row.
// Bonds and constraints are stored without the duplicate check, as in MDBas.
// ---------------------------------------------------------------------------
struct ExclBuilder {
  bool symmetric;
  std::vector<std::vector<int>> rows;
  std::vector<std::vector<int>> connect;
  std::vector<int> pair14;
  int nDihedral = 0;
  int status = MDBAS_NB_OK;

  ExclBuilder(int n, bool sym) : symmetric(sym), rows(n), connect(n) {}

  bool has(int ii, int jj) const {
    for (int v : rows[ii])
      if (v == jj) return true;
    return false;
  }
  void put(int ii, int jj) {
    rows[ii].push_back(jj);
    if (symmetric) rows[jj].push_back(ii);
  }
  // ordered pair as MDBas forms it for each form
  void order(int a, int b, int &ii, int &jj) const {
    if (symmetric) {
      ii = a;
      jj = b;
    } else if (b < a) {
      ii = b;
      jj = a;
    } else {
      ii = a;
      jj = b;
    }
  }
  void add_unchecked(int a, int b) {
    int ii, jj;
    order(a, b, ii, jj);
    connect[ii].push_back(jj);
    connect[jj].push_back(ii);
    put(ii, jj);
  }
  bool add_checked(int a, int b) {
    int ii, jj;
    order(a, b, ii, jj);
    if (has(ii, jj)) return false;
    put(ii, jj);
    return true;
  }
  void walk() {
    const int n = (int)rows.size();
    for (int ia = 0; ia < n; ++ia) {
      for (size_t j = 0; j < connect[ia].size(); ++j) {
        const int ib = connect[ia][j];
        for (size_t k = 0; k < connect[ib].size(); ++k) {
          const int ic = connect[ib][k];
          if (ic == ia) continue;
          add_checked(ia, ic);
          for (size_t l = 0; l < connect[ic].size(); ++l) {
            const int id = connect[ic][l];
            if (id == ia || id == ib) continue;
            if ((int)(pair14.size() / 2) >= 5 * nDihedral) {
              status = MDBAS_NB_ERR_EXCL;  // DIHE_NONPARAM_ERROR
              return;
            }
            if (add_checked(ia, id)) {
              pair14.push_back(ia);
              pair14.push_back(id);
            }
          }
        }
      }
    }
  }
};

int build_exclusions(bool symmetric, CTRL *ctrl, PARAM *param, NEIGH *neigh,
                     CONSTRAINT constList[], BOND bond[], ANGLE angle[], DIHE dihe[],
                     DIHE impr[], int **neighList14, int ***exclList, int **exclPair,
                     int *dihe_error) {
  const int n = param->nAtom;
  if (n <= 0) return MDBAS_NB_ERR_ARG;
  ExclBuilder B(n, symmetric);
  B.nDihedral = param->nDihedral;
  for (int i = 0; i < param->nBond; ++i) B.add_unchecked(bond[i].a, bond[i].b);
  if (ctrl->keyConstH)
    for (int i = 0; i < param->nConst; ++i) B.add_unchecked(constList[i].a, constList[i].b);
  for (int i = 0; i < param->nAngle; ++i) {
    B.add_checked(angle[i].a, angle[i].b);
    B.add_checked(angle[i].a, angle[i].c);
    B.add_checked(angle[i].b, angle[i].c);
  }
  for (int i = 0; i < param->nDihedral; ++i) {
    const DIHE &d = dihe[i];
    B.add_checked(d.a, d.b);
    B.add_checked(d.a, d.c);
    if (B.add_checked(d.a, d.d)) {
      B.pair14.push_back(d.a);
      B.pair14.push_back(d.d);
    }
    B.add_checked(d.b, d.c);
    B.add_checked(d.b, d.d);
    B.add_checked(d.c, d.d);
  }
  for (int i = 0; i < param->nImproper; ++i) {
    const DIHE &d = impr[i];
    B.add_checked(d.a, d.b);
    B.add_checked(d.a, d.c);
    B.add_checked(d.a, d.d);
    B.add_checked(d.b, d.c);
    B.add_checked(d.b, d.d);
    B.add_checked(d.c, d.d);
  }
  B.walk();
  if (B.status != MDBAS_NB_OK) {
    *dihe_error = 1;
    return B.status;
  }
  if (!symmetric && !B.rows[n - 1].empty()) return MDBAS_NB_ERR_EXCL;  // src/list.c:880-881
  neigh->nPair14 = (int)(B.pair14.size() / 2);
  *neighList14 = (int *)malloc(sizeof(int) * std::max<size_t>(1, B.pair14.size()));
  *exclPair = (int *)malloc(sizeof(int) * n);
  const int nrows = symmetric ? n : n - 1;
  *exclList = (int **)malloc(sizeof(int *) * std::max(1, nrows));
  if (!*neighList14 || !*exclPair || !*exclList) return MDBAS_NB_ERR_ALLOC;
  if (!B.pair14.empty()) memcpy(*neighList14, B.pair14.data(), sizeof(int) * B.pair14.size());
  for (int i = 0; i < n; ++i) (*exclPair)[i] = (int)B.rows[i].size();
  for (int i = 0; i < nrows; ++i) {
    (*exclList)[i] = (int *)malloc(sizeof(int) * std::max<size_t>(1, B.rows[i].size()));
    if (!(*exclList)[i]) return MDBAS_NB_ERR_ALLOC;
    if (!B.rows[i].empty())
      memcpy((*exclList)[i], B.rows[i].data(), sizeof(int) * B.rows[i].size());
  }
  return MDBAS_NB_OK;
}

void exclusions_or_fail(bool symmetric, CTRL *ctrl, PARAM *param, NEIGH *neigh,
                        CONSTRAINT constList[], BOND bond[], ANGLE angle[], DIHE dihe[],
                        DIHE impr[], int **neighList14, int ***exclList, int **exclPair) {
  int dihe_error = 0;
  const int st = build_exclusions(symmetric, ctrl, param, neigh, constList, bond, angle, dihe,
                                  impr, neighList14, exclList, exclPair, &dihe_error);
  if (st != MDBAS_NB_OK)
    fail(st, symmetric ? "link_cell_exclude_list" : "exclude_list", dihe_error ? 110 : 0);
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void init_energy_ptrs(CTRL *ctrl) {
  switch (ctrl->elecType) {
    case NOELEC: case FULL: case SHIFT1: case SHIFT2: case SWITCH: break;
    default: fail(MDBAS_NB_ERR_ARG, "init_energy_ptrs", 201);  // UNKNOWN_ELEC_ERROR
  }
  switch (ctrl->vdwType) {
    case NOVDW: case VFULL: case VSWITCH: break;
    default: fail(MDBAS_NB_ERR_ARG, "init_energy_ptrs", 202);  // UNKNOWN_VDW_ERROR
  }
  g.elecType = ctrl->elecType;
  g.vdwType = ctrl->vdwType;
  g.ptrsSet = true;
}

void exclude_list(CTRL *ctrl, PARAM *param, NEIGH *neigh, CONSTRAINT constList[], BOND bond[],
                  ANGLE angle[], DIHE dihe[], DIHE impr[], int **neighList14, int ***exclList,
                  int **exclPair) {
  exclusions_or_fail(false, ctrl, param, neigh, constList, bond, angle, dihe, impr, neighList14,
                     exclList, exclPair);
}

void link_cell_exclude_list(CTRL *ctrl, PARAM *param, NEIGH *neigh, CONSTRAINT constList[],
                            BOND bond[], ANGLE angle[], DIHE dihe[], DIHE impr[],
                            int **neighList14, int ***exclList, int **exclPair) {
  exclusions_or_fail(true, ctrl, param, neigh, constList, bond, angle, dihe, impr, neighList14,
                     exclList, exclPair);
}

int mdbas_nb_verlet_list_status(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[],
                                double z[], int frozen[], int **neighList, int **neighPair,
                                int **neighOrder, int **exclList, int exclPair[], int update) {
  if (!param || !box || !neigh || !x || !y || !z || !neighList || !neighPair) return MDBAS_NB_ERR_ARG;
  if (update)
    return list_common(0, 0, param, box, neigh, x, y, z, frozen, neighList, nullptr, nullptr,
                       *neighPair, nullptr, exclList, exclPair);
  return list_common(0, 1, param, box, neigh, x, y, z, frozen, neighList, neighPair, neighOrder,
                     nullptr, nullptr, exclList, exclPair);
}

int mdbas_nb_link_cell_list_status(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[],
                                   double z[], int frozen[], int **neighList, int **neighPair,
                                   int **neighOrder, int **exclList, int exclPair[],
                                   int update) {
  if (!param || !box || !neigh || !x || !y || !z || !neighList || !neighPair || !neighOrder)
    return MDBAS_NB_ERR_ARG;
  if (update)
    return list_common(1, 0, param, box, neigh, x, y, z, frozen, neighList, nullptr, nullptr,
                       *neighPair, *neighOrder, exclList, exclPair);
  return list_common(1, 1, param, box, neigh, x, y, z, frozen, neighList, neighPair, neighOrder,
                     nullptr, nullptr, exclList, exclPair);
}

void verlet_list(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[], double z[],
                 int frozen[], int **neighList, int **neighPair, int **neighOrder,
                 int **exclList, int exclPair[]) {
  DROP_TRY(mdbas_nb_verlet_list_status(param, box, neigh, x, y, z, frozen, neighList, neighPair,
                                       neighOrder, exclList, exclPair, 0),
           "verlet_list");
}

void verlet_list_update(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[], double z[],
                        int frozen[], int **neighList, int neighPair[], int **exclList,
                        int exclPair[]) {
  DROP_TRY(mdbas_nb_verlet_list_status(param, box, neigh, x, y, z, frozen, neighList, &neighPair,
                                       nullptr, exclList, exclPair, 1),
           "verlet_list_update");
}

void link_cell_verlet_list(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[],
                           double z[], int frozen[], int **neighList, int **neighPair,
                           int **neighOrder, int **exclList, int exclPair[]) {
  DROP_TRY(mdbas_nb_link_cell_list_status(param, box, neigh, x, y, z, frozen, neighList,
                                          neighPair, neighOrder, exclList, exclPair, 0),
           "link_cell_verlet_list");
}

void link_cell_verlet_list_update(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[],
                                  double z[], int frozen[], int **neighList, int neighPair[],
                                  int neighOrder[], int **exclList, int exclPair[]) {
  DROP_TRY(mdbas_nb_link_cell_list_status(param, box, neigh, x, y, z, frozen, neighList,
                                          &neighPair, &neighOrder, exclList, exclPair, 1),
           "link_cell_verlet_list_update");
}

// makelist (src/list.c:29-106).
void makelist(CTRL *ctrl, PARAM *param, PBC *box, NEIGH *neigh, CONSTRAINT constList[],
              BOND bond[], ANGLE angle[], DIHE dihe[], DIHE impr[], double x[], double y[],
              double z[], int frozen[], int **neighList, int **neighPair, int **neighOrder,
              int **neighList14, int ***exclList, int **exclPair) {
  if (ctrl->newjob == 1) {
    neigh->linkRatio = std::min(std::max(neigh->linkRatio, 1), 5);
    const DevBox b = make_devbox(box);
    ctrl->keyLink = makelist_uses_link_cells(b, param->cutOff, param->delr, neigh->linkRatio,
                                             ctrl->noLink);
    if (ctrl->keyLink) {
      link_cell_exclude_list(ctrl, param, neigh, constList, bond, angle, dihe, impr, neighList14,
                             exclList, exclPair);
      link_cell_verlet_list(param, box, neigh, x, y, z, frozen, neighList, neighPair, neighOrder,
                            *exclList, *exclPair);
    } else {
      exclude_list(ctrl, param, neigh, constList, bond, angle, dihe, impr, neighList14, exclList,
                   exclPair);
      verlet_list(param, box, neigh, x, y, z, frozen, neighList, neighPair, neighOrder,
                  *exclList, *exclPair);
    }
    ctrl->newjob = 0;
  } else if (param->step % neigh->update == 0) {
    if (ctrl->keyLink)
      link_cell_verlet_list_update(param, box, neigh, x, y, z, frozen, neighList, *neighPair,
                                   *neighOrder, *exclList, *exclPair);
    else
      verlet_list_update(param, box, neigh, x, y, z, frozen, neighList, *neighPair, *exclList,
                         *exclPair);
  }
}

int mdbas_nb_ewald_energy_status(CTRL *ctrl, PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box,
                                 const double x[], const double y[], const double z[], double fx[],
                                 double fy[], double fz[], const double q[], const double eps[],
                                 const double sig[], const int neighList[], const int neighPair[],
                                 const int neighOrder[], int **exclList, const int exclPair[]) {
  if (!ctrl || !param || !ener || !ewald || !box || !x || !fx || !q) return MDBAS_NB_ERR_ARG;
  double eRec = 0., virRec = 0., stress1[6] = {0., 0., 0., 0., 0., 0.};
  // k-space first, as in MDBas: ewald_rec rescales the force arrays.
  if (ctrl->keyEwald == 1)
    eRec = ewald_rec(param, ewald, box, x, y, z, fx, fy, fz, q, stress1, &virRec);
  else if (ctrl->keyEwald == 2)
    eRec = spme_energy(param, ewald, box, x, y, z, fx, fy, fz, q, stress1, &virRec);
  const int vdwSwitch = (g.ptrsSet ? g.vdwType : ctrl->vdwType) == VSWITCH;
  double e[6];
  ST_TRY(real_space(mdbas_nb_get_mode(), list_rule(1, ctrl ? ctrl->noLink : 0), param->nAtom,
                    param, ewald->alpha, vdwSwitch, box, x, y,
                    z, fx, fy, fz, q, eps, sig, neighList, neighPair, neighOrder, exclList,
                    exclPair, nullptr, e));
  ener->elec += e[0] + eRec + e[1];
  ener->vdw += e[2];
  ener->virelec += e[3] + virRec + e[4];
  ener->virvdw += e[5];
  return MDBAS_NB_OK;
}

void ewald_energy(CTRL *ctrl, PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box, const double x[],
                  const double y[], const double z[], double fx[], double fy[], double fz[],
                  const double q[], const double eps[], const double sig[], const int neighList[],
                  const int neighPair[], const int neighOrder[], int **exclList,
                  const int exclPair[]) {
  DROP_TRY(mdbas_nb_ewald_energy_status(ctrl, param, ener, ewald, box, x, y, z, fx, fy, fz, q, eps,
                                        sig, neighList, neighPair, neighOrder, exclList, exclPair),
           "ewald_energy");
}

void nonbond_energy(PARAM *param, ENERGY *ener, PBC *box, const double x[], const double y[],
                    const double z[], double fx[], double fy[], double fz[], const double q[],
                    const double eps[], const double sig[], const int neighList[],
                    const int neighPair[], const int neighOrder[]) {
  const int n = param->nAtom;
  auto run = [&]() -> int {
    ST_TRY(ctx_init());
    const DevBox b = make_devbox(box);
    const PairParams p = make_params(param->cutOff, param->cutOn, 0.0, param->chargeConst,
                                     g.vdwType == VSWITCH, g.elecType);
    ST_TRY(upload_positions(n, x, y, z));
    ST_TRY(upload_params(n, q, eps, sig));
    ST_TRY(ensure_list_on_device(n, neighList, neighPair, neighOrder));
    ST_TRY(g.f3.ensure(sizeof(double) * 3 * (size_t)n));
    ST_TRY(g.acc64.ensure(sizeof(double) * kFp64AccCount));
    MDB_CUDA(cudaMemsetAsync(g.f3.p, 0, sizeof(double) * 3 * (size_t)n, g.s));
    MDB_CUDA(cudaMemsetAsync(g.acc64.p, 0, sizeof(double) * kFp64AccCount, g.s));
    double *fxd = g.f3.as<double>();
    ST_TRY(pairs_fp64(0, n, b, p, g.ref.order.as<int>(), g.ref.neighPair.as<int>(),
                      g.ref.off.as<long long>(), g.ref.list.as<int>(), g.x.as<double>(),
                      g.y.as<double>(), g.z.as<double>(), g.q.as<double>(), g.eps.as<double>(),
                      g.sig.as<double>(), fxd, fxd + n, fxd + 2 * (size_t)n, g.acc64.as<double>(),
                      g.s));
    double a[kFp64AccCount];
    MDB_CUDA(cudaMemcpyAsync(a, g.acc64.p, sizeof(a), cudaMemcpyDeviceToHost, g.s));
    ST_TRY(add_forces(n, fxd, fx, fy, fz));
    ener->elec += a[0];
    ener->vdw += a[1];
    ener->virelec += a[2];
    ener->virvdw += a[3];
    return MDBAS_NB_OK;
  };
  DROP_TRY(run(), "nonbond_energy");
}

static int pairs14_common(int ewaldForm, PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box,
                          NEIGH *neigh, const double x[], const double y[], const double z[],
                          double fx[], double fy[], double fz[], const double q[],
                          const double eps[], const double sig[], const int neighList14[]) {
  const int n = param->nAtom;
  const int np = neigh->nPair14;
  if (np <= 0) return MDBAS_NB_OK;
  ST_TRY(ctx_init());
  const DevBox b = make_devbox(box);
  PairParams p = make_params(param->cutOff, param->cutOn, ewald ? ewald->alpha : 0.0,
                             param->chargeConst, g.vdwType == VSWITCH, g.elecType);
  p.scal14 = param->scal14;
  ST_TRY(upload_positions(n, x, y, z));
  // 1-4 parameters (eps14/sig14) differ from the pair parameters: upload
  // them into scratch rather than the cached topology.
  ST_TRY(g.f3.ensure(sizeof(double) * 3 * (size_t)n));
  ST_TRY(g.acc64.ensure(sizeof(double) * kFp64AccCount));
  ST_TRY(g.list14.ensure(sizeof(int) * 2 * (size_t)np + sizeof(double) * 3 * (size_t)n));
  int *l14 = g.list14.as<int>();
  double *q14 = reinterpret_cast<double *>(l14 + 2 * (size_t)np + ((2 * np) & 1));
  double *e14 = q14 + n, *s14 = e14 + n;
  MDB_CUDA(cudaMemcpyAsync(l14, neighList14, sizeof(int) * 2 * np, cudaMemcpyHostToDevice, g.s));
  MDB_CUDA(cudaMemcpyAsync(q14, q, sizeof(double) * n, cudaMemcpyHostToDevice, g.s));
  MDB_CUDA(cudaMemcpyAsync(e14, eps, sizeof(double) * n, cudaMemcpyHostToDevice, g.s));
  MDB_CUDA(cudaMemcpyAsync(s14, sig, sizeof(double) * n, cudaMemcpyHostToDevice, g.s));
  MDB_CUDA(cudaMemsetAsync(g.f3.p, 0, sizeof(double) * 3 * (size_t)n, g.s));
  MDB_CUDA(cudaMemsetAsync(g.acc64.p, 0, sizeof(double) * kFp64AccCount, g.s));
  double *fxd = g.f3.as<double>();
  ST_TRY(pairs14_fp64(ewaldForm, np, b, p, l14, g.x.as<double>(), g.y.as<double>(),
                      g.z.as<double>(), q14, e14, s14, fxd, fxd + n, fxd + 2 * (size_t)n,
                      g.acc64.as<double>(), g.s));
  double a[kFp64AccCount];
  MDB_CUDA(cudaMemcpyAsync(a, g.acc64.p, sizeof(a), cudaMemcpyDeviceToHost, g.s));
  ST_TRY(add_forces(n, fxd, fx, fy, fz));
  ener->elec += a[0];
  ener->vdw += a[1];
  ener->virelec += a[2];
  ener->virvdw += a[3];
  return MDBAS_NB_OK;
}

void ewald14_energy(PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box, NEIGH *neigh,
                    const double x[], const double y[], const double z[], double fx[], double fy[],
                    double fz[], const double q[], const double eps[], const double sig[],
                    const int neighList14[]) {
  DROP_TRY(pairs14_common(1, param, ener, ewald, box, neigh, x, y, z, fx, fy, fz, q, eps, sig,
                          neighList14),
           "ewald14_energy");
}

void nonbond14_energy(PARAM *param, ENERGY *ener, PBC *box, NEIGH *neigh, const double x[],
                      const double y[], const double z[], double fx[], double fy[], double fz[],
                      const double q[], const double eps[], const double sig[],
                      const int neighList14[]) {
  DROP_TRY(pairs14_common(0, param, ener, nullptr, box, neigh, x, y, z, fx, fy, fz, q, eps, sig,
                          neighList14),
           "nonbond14_energy");
}

// energy (src/energy.c:103-205).
void energy(CTRL *ctrl, PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box, NEIGH *neigh,
            BOND bond[], BOND ub[], ANGLE angle[], DIHE dihe[], DIHE impr[], const double x[],
            const double y[], const double z[], double vx[], double vy[], double vz[],
            double fx[], double fy[], double fz[], const double q[], const double eps[],
            const double sig[], const double eps14[], const double sig14[], const int frozen[],
            const int neighList[], const int neighPair[], const int neighOrder[],
            const int neighList14[], int **exclList, const int exclPair[]) {
  ener->elec = 0.;
  ener->vdw = 0.;
  ener->bond = 0.;
  ener->ub = 0.;
  ener->ang = 0.;
  ener->dihe = 0.;
  ener->impr = 0.;
  ener->virelec = 0.;
  ener->virvdw = 0.;
  ener->virbond = 0.;
  ener->virub = 0.;
  ener->virpot = 0.;
  box->stress1 = box->stress2 = box->stress3 = 0.;
  box->stress4 = box->stress5 = box->stress6 = 0.;
  box->stress7 = box->stress8 = box->stress9 = 0.;
  for (int i = 0; i < param->nAtom; ++i) {
    fx[i] = 0.;
    fy[i] = 0.;
    fz[i] = 0.;
  }
  if (ctrl->keyEwald != 0) {
    ewald_energy(ctrl, param, ener, ewald, box, x, y, z, fx, fy, fz, q, eps, sig, neighList,
                 neighPair, neighOrder, exclList, exclPair);
    if (ctrl->keyNb14)
      ewald14_energy(param, ener, ewald, box, neigh, x, y, z, fx, fy, fz, q, eps14, sig14,
                     neighList14);
  } else {
    nonbond_energy(param, ener, box, x, y, z, fx, fy, fz, q, eps, sig, neighList, neighPair,
                   neighOrder);
    if (ctrl->keyNb14)
      nonbond14_energy(param, ener, box, neigh, x, y, z, fx, fy, fz, q, eps14, sig14,
                       neighList14);
  }
  if (param->nBond > 0) {
    bond_energy(param, ener, box, bond, x, y, z, fx, fy, fz);
  }
  if (param->nAngle > 0) {
    angle_energy(param, ener, box, angle, x, y, z, fx, fy, fz);
  }
  if (param->nUb > 0) {
    ub_energy(param, ener, box, ub, x, y, z, fx, fy, fz);
  }
  if (param->nDihedral > 0) {
    dihedral_energy(param, ener, box, dihe, x, y, z, fx, fy, fz);
  }
  if (param->nImproper > 0) {
    improper_energy(param, ener, box, impr, x, y, z, fx, fy, fz);
  }
  ener->pot = ener->elec + ener->vdw + ener->bond + ener->ang + ener->ub + ener->dihe +
              ener->impr;
  ener->virpot = ener->virbond + ener->virub + ener->virelec + ener->virvdw;
  if (param->nFrozen > 0) {
    if (!freeze_atoms) fail(MDBAS_NB_ERR_MISSING, "energy (freeze_atoms)");
    freeze_atoms(param, vx, vy, vz, fx, fy, fz, frozen);
  }
}

// ---------------------------------------------------------------------------
// Bonded terms (src/internal.c:21-620), MDBas's prototypes (include/internal.h)
// ---------------------------------------------------------------------------
namespace {
// kind as mdbas_nb_bonded numbers them; energies into *e, virial into *vir
void bonded_dropin(int kind, const PARAM *param, const PBC *box, int nTerms, const void *terms,
                   const double *x, const double *y, const double *z, double *fx, double *fy,
                   double *fz, double *e, double *vir, const char *where) {
  double out[2];
  DROP_TRY(mdbas_nb_bonded(kind, param->nAtom, box, nTerms, terms, x, y, z, fx, fy, fz, out),
           where);
  *e += out[0];
  if (vir) *vir += out[1];
}
}  // namespace

void bond_energy(const PARAM *param, ENERGY *ener, const PBC *box, const BOND bond[],
                 const double *x, const double *y, const double *z, double *fx, double *fy,
                 double *fz) {
  bonded_dropin(0, param, box, param->nBond, bond, x, y, z, fx, fy, fz, &ener->bond,
                &ener->virbond, "bond_energy");
}

void angle_energy(const PARAM *param, ENERGY *ener, const PBC *box, const ANGLE angle[],
                  const double *x, const double *y, const double *z, double *fx, double *fy,
                  double *fz) {
  bonded_dropin(1, param, box, param->nAngle, angle, x, y, z, fx, fy, fz, &ener->ang, nullptr,
                "angle_energy");
}

void ub_energy(const PARAM *param, ENERGY *ener, const PBC *box, const BOND ub[], const double *x,
               const double *y, const double *z, double *fx, double *fy, double *fz) {
  bonded_dropin(2, param, box, param->nUb, ub, x, y, z, fx, fy, fz, &ener->ub, &ener->virub,
                "ub_energy");
}

void dihedral_energy(const PARAM *param, ENERGY *ener, const PBC *box, const DIHE dihe[],
                     const double *x, const double *y, const double *z, double *fx, double *fy,
                     double *fz) {
  bonded_dropin(3, param, box, param->nDihedral, dihe, x, y, z, fx, fy, fz, &ener->dihe, nullptr,
                "dihedral_energy");
}

void improper_energy(const PARAM *param, ENERGY *ener, const PBC *box, const DIHE impr[],
                     const double *x, const double *y, const double *z, double *fx, double *fy,
                     double *fz) {
  bonded_dropin(4, param, box, param->nImproper, impr, x, y, z, fx, fy, fz, &ener->impr, nullptr,
                "improper_energy");
}

// ---------------------------------------------------------------------------
// UserEnergyPtr plugin
// ---------------------------------------------------------------------------
static struct {
  bool ready = false;
  int n = 0;
  std::vector<double> q, eps, sig;
  std::vector<int> exclPair;
  std::vector<std::vector<int>> rows;
  std::vector<int *> rowPtr;
  double alpha = 0.;
  int vdwSwitch = 1;
  double last[4] = {0., 0., 0., 0.};
} g_plugin;

int mdbas_nb_plugin_init(int nAtom, const double q[], const double eps[], const double sig[],
                         const int exclPair[], int **exclList, double alpha, int vdwSwitch) {
  if (nAtom <= 0 || !q || !eps || !sig) return MDBAS_NB_ERR_ARG;
  g_plugin.n = nAtom;
  g_plugin.q.assign(q, q + nAtom);
  g_plugin.eps.assign(eps, eps + nAtom);
  g_plugin.sig.assign(sig, sig + nAtom);
  g_plugin.exclPair.assign(nAtom, 0);
  g_plugin.rows.assign(nAtom, {});
  g_plugin.rowPtr.assign(nAtom, nullptr);
  if (exclPair && exclList) {
    for (int i = 0; i < nAtom; ++i) {
      g_plugin.exclPair[i] = exclPair[i];
      g_plugin.rows[i].assign(exclList[i], exclList[i] + exclPair[i]);
    }
  }
  for (int i = 0; i < nAtom; ++i) g_plugin.rowPtr[i] = g_plugin.rows[i].data();
  g_plugin.alpha = alpha;
  g_plugin.vdwSwitch = vdwSwitch ? 1 : 0;
  g_plugin.ready = true;
  return MDBAS_NB_OK;
}

double mdbas_nb_user_energy(const PARAM *param, const PBC *box, const double x[], const double y[],
                            const double z[], double fx[], double fy[], double fz[],
                            const int neighList[], const int neighPair[], const int neighOrder[],
                            const int neighList14[]) {
  (void)neighList14;
  if (!g_plugin.ready || !param || param->nAtom != g_plugin.n) {
    set_last_status(MDBAS_NB_ERR_STATE, "mdbas_nb_plugin_init was not called for this system");
    fail(MDBAS_NB_ERR_STATE, "mdbas_nb_user_energy");
  }
  double e[6];
  DROP_TRY(real_space(mdbas_nb_get_mode(), list_rule(1, 0), param->nAtom, param, g_plugin.alpha,
                      g_plugin.vdwSwitch, box, x, y, z, fx, fy, fz, g_plugin.q.data(),
                      g_plugin.eps.data(), g_plugin.sig.data(), neighList, neighPair, neighOrder,
                      g_plugin.rowPtr.data(), g_plugin.exclPair.data(), nullptr, e),
           "mdbas_nb_user_energy");
  g_plugin.last[0] = e[0] + e[1];
  g_plugin.last[1] = e[2];
  g_plugin.last[2] = e[3] + e[4];
  g_plugin.last[3] = e[5];
  return g_plugin.last[0] + g_plugin.last[1];
}

int mdbas_nb_plugin_last_energy(double out[4]) {
  if (!out) return MDBAS_NB_ERR_ARG;
  if (!g_plugin.ready) return MDBAS_NB_ERR_STATE;
  memcpy(out, g_plugin.last, sizeof(g_plugin.last));
  return MDBAS_NB_OK;
}

void mdbas_nb_plugin_release(void) {
  g_plugin.ready = false;
  g_plugin.q.clear();
  g_plugin.eps.clear();
  g_plugin.sig.clear();
  g_plugin.rows.clear();
  g_plugin.rowPtr.clear();
  g_plugin.exclPair.clear();
}

}  // extern "C"
