// noalloc.cu -- the plain FP64 real-space Ewald evaluation without any
// device allocation.
//
// Some callers cannot let a library call cudaMalloc: a host program that
// owns all device memory through its own pool allocator and forbids others,
// a solver step that must not trigger the implicit device synchronisation
// cudaMalloc/cudaFree cause, or a real-time loop with a fixed memory budget.
// For them this file provides one entry point that works only on memory the
// caller passes in plus a fixed scratch area compiled into the library.
//
// The scratch area is a file-scope __device__ array of MDBAS_NB_NOALLOC_SCRATCH_BYTES
// (about 1.6 MB, for up to MDBAS_NB_NOALLOC_MAX_ATOMS atoms).  Every GPU
// that loads the library holds it until the process exits.  All calls share
// it and it keeps the previous call's contents, so the parts that must start
// at zero are cleared by each call, and two calls that overlap on the GPU
// (different streams, no ordering between them) race on it.
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side shadow).  The first call on each device, with that device
// current, asks the runtime for the array's device address with
// cudaGetSymbolAddress and remembers it (one atomic slot per device, so
// threads making their first calls at once store the same value without a
// data race); make that first call before any stream capture.  A
// cudaDeviceReset unloads the library's device code and the remembered
// address with it: after a reset, do not call this entry point again on that
// device in the same process.
#include <atomic>

#include "common.cuh"
#include "pair_fp64.cuh"

namespace mdbas {
namespace {

constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

constexpr int kMaxAtoms = MDBAS_NB_NOALLOC_MAX_ATOMS;
// scratch layout: per-position entry counts, entry offsets, scan tile sums,
// FP64 energy accumulators
constexpr size_t kCountsOff = 0;
constexpr size_t kCountsBytes = align256(sizeof(int) * (kMaxAtoms + 1));
constexpr size_t kOffsOff = kCountsOff + kCountsBytes;
constexpr size_t kOffsBytes = align256(sizeof(long long) * (kMaxAtoms + 2));
constexpr size_t kScanOff = kOffsOff + kOffsBytes;
constexpr size_t kScanBytes = align256(sizeof(long long) * 128);
constexpr size_t kAccOff = kScanOff + kScanBytes;
constexpr size_t kAccBytes = align256(sizeof(double) * kFp64AccCount);
constexpr size_t kScratchBytes = kAccOff + kAccBytes;
static_assert(kScratchBytes == MDBAS_NB_NOALLOC_SCRATCH_BYTES, "scratch size changed: update the header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::atomic<void *> g_scratch_addr[kMaxDevices];

__global__ void k_noalloc_counts(int n, const int *__restrict__ order,
                                 const int *__restrict__ neighPair, int *__restrict__ cnt) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) cnt[p] = neighPair[order[p]];
}

int scratch_for_current_device(unsigned char **out) {
  int dev = 0;
  MDB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return MDBAS_NB_ERR_ARG;
  void *p = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!p) {
    MDB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[dev].store(p, std::memory_order_release);
  }
  *out = static_cast<unsigned char *>(p);
  return MDBAS_NB_OK;
}

}  // namespace
}  // namespace mdbas

extern "C" int mdbas_nb_ewald_fp64_noalloc(
    int nAtom, const PBC *box, double cutOff, double cutOn, double alpha, double chargeConst,
    int vdwSwitch, const double *x, const double *y, const double *z, const double *q,
    const double *eps, const double *sig, const int *neighList, const int *neighPair,
    const int *neighOrder, const int *exclStart, const int *exclFlat, double *fx, double *fy,
    double *fz, double energies[6], void *stream) {
  using namespace mdbas;
  if (nAtom <= 0 || !box || !x || !y || !z || !q || !eps || !sig || !neighList || !neighPair ||
      !neighOrder || !exclStart || !exclFlat || !fx || !fy || !fz || !energies) {
    set_last_status(MDBAS_NB_ERR_ARG, "mdbas_nb_ewald_fp64_noalloc: null argument");
    return MDBAS_NB_ERR_ARG;
  }
  if (nAtom > kMaxAtoms) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "mdbas_nb_ewald_fp64_noalloc: %d atoms exceed the fixed scratch limit of %d",
             nAtom, kMaxAtoms);
    set_last_status(MDBAS_NB_ERR_CAPACITY, msg);
    return MDBAS_NB_ERR_CAPACITY;
  }
  unsigned char *base = nullptr;
  int st = scratch_for_current_device(&base);
  if (st != MDBAS_NB_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int *cnt = reinterpret_cast<int *>(base + kCountsOff);
  long long *off = reinterpret_cast<long long *>(base + kOffsOff);
  void *scanTmp = base + kScanOff;
  double *acc = reinterpret_cast<double *>(base + kAccOff);

  const DevBox b = make_devbox(box);
  PairParams p;
  p.chargeConst = chargeConst;
  p.alpha = alpha;
  p.cutOff2 = cutOff * cutOff;
  p.cutOn2 = cutOn * cutOn;
  p.switch2 = 1. / ((p.cutOff2 - p.cutOn2) * (p.cutOff2 - p.cutOn2) * (p.cutOff2 - p.cutOn2));
  p.rcutOff = 1. / cutOff;
  p.rcutOff2 = 1. / p.cutOff2;
  p.scal14 = 1.0;
  p.vdwSwitch = vdwSwitch ? 1 : 0;
  p.elecType = FULL;

  // the accumulators keep the previous call's sums: clear them first
  MDB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * kFp64AccCount, s));
  MDB_LAUNCH(k_noalloc_counts, grid_for(nAtom, 256), 256, 0, s, nAtom, neighOrder, neighPair,
             cnt);
  st = exclusive_scan(cnt, off, nAtom, scanTmp, s);
  if (st != MDBAS_NB_OK) return st;
  st = pairs_fp64(1, nAtom, b, p, neighOrder, neighPair, off, neighList, x, y, z, q, eps, sig,
                  fx, fy, fz, acc, s);
  if (st != MDBAS_NB_OK) return st;
  st = excl_fp64(nAtom, b, p, exclStart, exclFlat, x, y, z, q, fx, fy, fz, acc, s);
  if (st != MDBAS_NB_OK) return st;
  double a[kFp64AccCount];
  MDB_CUDA(cudaMemcpyAsync(a, acc, sizeof(a), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  energies[0] = a[0];  // direct Ewald
  energies[1] = a[5];  // exclusion correction
  energies[2] = a[1];  // switched LJ
  energies[3] = a[2];  // virial, direct
  energies[4] = a[6];  // virial, correction
  energies[5] = a[3];  // virial, LJ
  return MDBAS_NB_OK;
}
