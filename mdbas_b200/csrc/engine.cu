// engine.cu -- device-resident nonbonded engine (mdbas_nb_engine_* C ABI).
//
// The engine owns every device array of one system: FP64 positions and
// topology in the caller's atom order, the MDBas-format list (precision 0)
// or the cluster layout and cluster-pair list (precision 1), and the force,
// energy and virial accumulators.  Calls run on the engine's stream and are
// asynchronous unless they return data to the host.
#include <math.h>
#include <string.h>

#include <vector>

#include "cluster.cuh"
#include "engine.cuh"
#include "list_ref.cuh"
#include "pair_fp32.cuh"
#include "pair_fp64.cuh"

using namespace mdbas;

namespace mdbas {

namespace {

__global__ void k_export_cluster_pairs(long long nEntries, const int4 *__restrict__ items,
                                       long long nItems, const CPairEntry *__restrict__ entries,
                                       const uint2 *__restrict__ masks,
                                       const float4 *__restrict__ xq,
                                       const int *__restrict__ slotAtom, float r2max,
                                       int *__restrict__ pairs, long long cap,
                                       unsigned long long *__restrict__ count) {
  // one warp per item; lane = (i slot, j half) as in the pair kernel
  const int lane = threadIdx.x & 31;
  const long long it = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (it >= nItems) return;
  const int4 item = items[it];
  const int il = lane & 7, jh = lane >> 3;
  const float4 xi = xq[item.x * kClusterSize + il];
  const int ai = slotAtom[item.x * kClusterSize + il];
  for (int e = item.y; e < item.y + item.z; ++e) {
    const CPairEntry en = entries[e];
    const uint2 mk = masks[e];
    for (int h = 0; h < 2; ++h) {
      const int jl = jh + 4 * h;
      const bool bit = ((h ? mk.y : mk.x) >> lane) & 1u;
      const float4 xj = xq[en.j * kClusterSize + jl];
      const float dx = xj.x + (en.sx - xi.x), dy = xj.y + (en.sy - xi.y),
                  dz = xj.z + (en.sz - xi.z);
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (bit && r2 <= r2max) {
        const int aj = slotAtom[en.j * kClusterSize + jl];
        const unsigned long long k = atomicAdd(count, 1ull);
        if ((long long)k < cap) {
          pairs[2 * k] = min(ai, aj);
          pairs[2 * k + 1] = max(ai, aj);
        }
      }
    }
  }
  (void)nEntries;
}

__global__ void k_export_ref_pairs(int n, DevBox b, const int *__restrict__ order,
                                   const int *__restrict__ neighPair,
                                   const long long *__restrict__ off,
                                   const int *__restrict__ list, const double *__restrict__ x,
                                   const double *__restrict__ y, const double *__restrict__ z,
                                   double r2max, int *__restrict__ pairs, long long cap,
                                   unsigned long long *__restrict__ count) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = order[p];
  const long long s = off[p];
  for (int k = 0; k < neighPair[i]; ++k) {
    const int j = list[s + k];
    double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
    const double r2 = dist_d(b, dx, dy, dz);
    if (r2 <= r2max) {
      const unsigned long long c = atomicAdd(count, 1ull);
      if ((long long)c < cap) {
        pairs[2 * c] = min(i, j);
        pairs[2 * c + 1] = max(i, j);
      }
    }
  }
}

}  // namespace

int engine_check_device(int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= 0) {
    set_last_status(MDBAS_NB_ERR_NO_DEVICE, "no CUDA device");
    return MDBAS_NB_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return MDBAS_NB_ERR_ARG;
  cudaDeviceProp prop;
  MDB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_last_status(MDBAS_NB_ERR_NO_DEVICE, "libmdbas_nb is built for sm_100a only");
    return MDBAS_NB_ERR_NO_DEVICE;
  }
  return MDBAS_NB_OK;
}

PairParams make_params(double cutOff, double cutOn, double alpha, double chargeConst,
                       int vdwSwitch, int elecType) {
  PairParams p;
  p.chargeConst = chargeConst;
  p.alpha = alpha;
  p.cutOff2 = cutOff * cutOff;
  p.cutOn2 = cutOn * cutOn;
  p.switch2 = 1. / ((p.cutOff2 - p.cutOn2) * (p.cutOff2 - p.cutOn2) * (p.cutOff2 - p.cutOn2));
  p.rcutOff = 1. / cutOff;
  p.rcutOff2 = 1. / p.cutOff2;
  p.scal14 = 1.0;
  p.vdwSwitch = vdwSwitch;
  p.elecType = elecType;
  return p;
}

}  // namespace mdbas

#define ENG_TRY(e, expr)                                                       \
  do {                                                                         \
    int s__ = (expr);                                                          \
    if (s__ != MDBAS_NB_OK) {                                                  \
      set_last_status(s__, nullptr);                                           \
      return s__;                                                              \
    }                                                                          \
  } while (0)

static int ev_record(cudaEvent_t ev, cudaStream_t s) {
  MDB_CUDA(cudaEventRecord(ev, s));
  return MDBAS_NB_OK;
}

static int set_dev(mdbas_nb_engine *e) {
  MDB_CUDA(cudaSetDevice(e->device));
  return MDBAS_NB_OK;
}

// The replicas' boxes on the device, as the dynamics kernels read them.
static int upload_boxes(mdbas_nb_engine *e) {
  MDB_TRY(e->boxesDev.ensure(sizeof(DevBox) * e->repBoxes.size()));
  MDB_CUDA(cudaMemcpy(e->boxesDev.p, e->repBoxes.data(), sizeof(DevBox) * e->repBoxes.size(),
                      cudaMemcpyHostToDevice));
  return MDBAS_NB_OK;
}

// The cluster-pair list built and its counts read back (grows the list until
// it fits).
static int sync_build(mdbas_nb_engine *e) {
  const int *frozen = e->hasFrozen ? e->frozen.as<int>() : nullptr;
  return cluster_build(e->cl, e->n, e->nRep, e->repBoxes.data(), e->repOff.data(),
                       e->cfg.cutOff, e->cfg.delr, engine_list_rule(e), sqrt(e->cfg.chargeConst),
                       e->x.as<double>(), e->y.as<double>(), e->z.as<double>(),
                       e->q.as<double>(), e->eps.as<double>(), e->sig.as<double>(), frozen,
                       e->exclStartSym.as<int>(), e->exclFlatSym.as<int>(), e->stream);
}

// Error bits of the cached accumulators (mixed precision only).
static int acc_status(const mdbas_nb_engine *e) {
  if (e->cfg.precision == 0) return MDBAS_NB_OK;
  const long long f = e->accCache[ACC_FLAGS];
  if (f & FLAG_OVERFLOW) {
    set_last_status(MDBAS_NB_ERR_OVERFLOW, "fixed-point force overflow");
    return MDBAS_NB_ERR_OVERFLOW;
  }
  if (f & FLAG_STAGE) {
    set_last_status(MDBAS_NB_ERR_CUDA, "a bulk copy into shared memory timed out");
    return MDBAS_NB_ERR_CUDA;
  }
  return MDBAS_NB_OK;
}

int mdbas::engine_side_stream(mdbas_nb_engine *e) {
  if (e->side) return MDBAS_NB_OK;
  MDB_CUDA(cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking));
  MDB_CUDA(cudaEventCreateWithFlags(&e->evFork, cudaEventDisableTiming));
  MDB_CUDA(cudaEventCreateWithFlags(&e->evJoin, cudaEventDisableTiming));
  return MDBAS_NB_OK;
}

int mdbas::engine_resolve_build(mdbas_nb_engine *e) {
  if (!e->buildPending) return MDBAS_NB_OK;
  e->buildPending = false;
  long long sticky = 0;
  MDB_CUDA(cudaMemcpyAsync(&sticky, e->cl.sticky.p, sizeof(sticky), cudaMemcpyDeviceToHost,
                           e->stream));
  MDB_CUDA(cudaStreamSynchronize(e->stream));
  if (!(sticky & (CL_OVERFLOW | CL_NONFINITE))) return MDBAS_NB_OK;
  return engine_settle_build(e, sticky);
}

// A pending build's error word read back with a failure in it: a list that
// outgrew its room is rebuilt with room (and evaluated again if it had been);
// a non-finite position is reported.
int mdbas::engine_settle_build(mdbas_nb_engine *e, long long sticky) {
  MDB_CUDA(cudaMemsetAsync(e->cl.sticky.p, 0, sizeof(long long), e->stream));
  if (sticky & CL_NONFINITE) {
    e->built = false;
    set_last_status(MDBAS_NB_ERR_NONFINITE, "non-finite position in the list build");
    return MDBAS_NB_ERR_NONFINITE;
  }
  const bool redo = e->computed;
  ENG_TRY(e, sync_build(e));
  if (redo) return mdbas_nb_engine_compute(e);
  return MDBAS_NB_OK;
}

extern "C" {

int mdbas_nb_engine_create(mdbas_nb_engine **out, const mdbas_nb_engine_config *cfg,
                           const PBC *box) {
  if (!out || !cfg || !box || cfg->nAtom <= 0) return MDBAS_NB_ERR_ARG;
  if (cfg->precision != 0 && cfg->precision != 1) return MDBAS_NB_ERR_ARG;
  if (!(cfg->cutOff > 0.) || cfg->delr < 0. || cfg->cutOn > cfg->cutOff) return MDBAS_NB_ERR_ARG;
  int st = engine_check_device(cfg->device);
  if (st != MDBAS_NB_OK) return st;
  mdbas_nb_engine *e = new mdbas_nb_engine();
  e->cfg = *cfg;
  if (e->cfg.linkRatio < 1) e->cfg.linkRatio = 1;
  if (e->cfg.linkRatio > 5) e->cfg.linkRatio = 5;
  e->n = cfg->nAtom;
  e->device = cfg->device;
  e->hostBox = *box;
  e->box = make_devbox(box);
  e->repBoxes.assign(1, e->box);
  e->repOff = {0, e->n};
  e->pp = make_params(cfg->cutOff, cfg->cutOn, cfg->alpha, cfg->chargeConst, cfg->vdwSwitch,
                      FULL);
  if (set_dev(e) != MDBAS_NB_OK || cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) !=
                                         cudaSuccess) {
    delete e;
    return MDBAS_NB_ERR_CUDA;
  }
  e->ownStream = true;
  cudaEventCreate(&e->ev0);
  cudaEventCreate(&e->ev1);
  if (upload_boxes(e) != MDBAS_NB_OK) {
    mdbas_nb_engine_destroy(e);
    return MDBAS_NB_ERR_CUDA;
  }
  *out = e;
  return MDBAS_NB_OK;
}

int mdbas_nb_batch_create(mdbas_nb_engine **out, const mdbas_nb_engine_config *cfg, int nRep,
                          const PBC *boxes, const int *repAtoms) {
  if (!out || !cfg || !boxes || !repAtoms || nRep <= 0) return MDBAS_NB_ERR_ARG;
  if (cfg->precision != 1) return MDBAS_NB_ERR_UNSUPPORTED;
  long long total = 0;
  for (int r = 0; r < nRep; ++r) {
    if (repAtoms[r] <= 0) return MDBAS_NB_ERR_ARG;
    total += repAtoms[r];
  }
  if (total != cfg->nAtom || total > 0x7fffffffLL) return MDBAS_NB_ERR_ARG;
  mdbas_nb_engine *e = nullptr;
  int st = mdbas_nb_engine_create(&e, cfg, &boxes[0]);
  if (st != MDBAS_NB_OK) return st;
  e->nRep = nRep;
  e->repBoxes.resize(nRep);
  e->repOff.assign(nRep + 1, 0);
  std::vector<int> rep(cfg->nAtom);
  for (int r = 0; r < nRep; ++r) {
    e->repBoxes[r] = make_devbox(&boxes[r]);
    e->repOff[r + 1] = e->repOff[r] + repAtoms[r];
    for (int i = e->repOff[r]; i < e->repOff[r + 1]; ++i) rep[i] = r;
  }
  st = upload_boxes(e);
  if (st == MDBAS_NB_OK) st = e->atomRepDev.ensure(sizeof(int) * (size_t)cfg->nAtom);
  if (st == MDBAS_NB_OK &&
      cudaMemcpy(e->atomRepDev.p, rep.data(), sizeof(int) * (size_t)cfg->nAtom,
                 cudaMemcpyHostToDevice) != cudaSuccess)
    st = MDBAS_NB_ERR_CUDA;
  if (st != MDBAS_NB_OK) {
    mdbas_nb_engine_destroy(e);
    return st;
  }
  *out = e;
  return MDBAS_NB_OK;
}

int mdbas_nb_batch_count(mdbas_nb_engine *e) { return e ? e->nRep : -1; }

int mdbas_nb_engine_destroy(mdbas_nb_engine *e) {
  if (!e) return MDBAS_NB_OK;
  cudaSetDevice(e->device);
  cudaStreamSynchronize(e->stream);
  md_release(e);
  kspace_release(e);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->side) {
    cudaStreamSynchronize(e->side);
    cudaStreamDestroy(e->side);
    cudaEventDestroy(e->evFork);
    cudaEventDestroy(e->evJoin);
  }
  if (e->ownStream) cudaStreamDestroy(e->stream);
  delete e;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_set_stream(mdbas_nb_engine *e, void *stream) {
  if (!e) return MDBAS_NB_ERR_ARG;
  ENG_TRY(e, set_dev(e));
  if (e->ownStream) {
    cudaStreamSynchronize(e->stream);
    cudaStreamDestroy(e->stream);
    e->ownStream = false;
  }
  e->stream = static_cast<cudaStream_t>(stream);
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_set_box(mdbas_nb_engine *e, const PBC *box) {
  if (!e || !box) return MDBAS_NB_ERR_ARG;
  if (e->nRep > 1) return MDBAS_NB_ERR_UNSUPPORTED;
  ENG_TRY(e, set_dev(e));
  e->hostBox = *box;
  e->box = make_devbox(box);
  e->repBoxes.assign(1, e->box);
  ENG_TRY(e, upload_boxes(e));
  e->built = false;
  e->mdGraphStale = true;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_set_topology(mdbas_nb_engine *e, const double *q, const double *eps,
                                 const double *sig, const int *frozen, const int *exclPair,
                                 const int *exclFlat) {
  if (!e || !q || !eps || !sig || !exclPair) return MDBAS_NB_ERR_ARG;
  ENG_TRY(e, set_dev(e));
  LaunchScope ls(e);
  const int n = e->n;
  std::vector<int> start(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    if (exclPair[i] < 0) return MDBAS_NB_ERR_EXCL;
    start[i + 1] = start[i] + exclPair[i];
  }
  const int nex = start[n];
  if (nex > 0 && !exclFlat) return MDBAS_NB_ERR_ARG;
  for (int k = 0; k < nex; ++k)
    if (exclFlat[k] < 0 || exclFlat[k] >= n) return MDBAS_NB_ERR_EXCL;
  ENG_TRY(e, e->q.ensure(sizeof(double) * n));
  ENG_TRY(e, e->eps.ensure(sizeof(double) * n));
  ENG_TRY(e, e->sig.ensure(sizeof(double) * n));
  ENG_TRY(e, e->exclStart.ensure(sizeof(int) * (n + 1)));
  ENG_TRY(e, e->exclFlat.ensure(sizeof(int) * (nex > 0 ? nex : 1)));
  cudaStream_t s = e->stream;
  MDB_CUDA(cudaMemcpyAsync(e->q.p, q, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(e->eps.p, eps, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(e->sig.p, sig, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(e->exclStart.p, start.data(), sizeof(int) * (n + 1),
                           cudaMemcpyHostToDevice, s));
  if (nex > 0)
    MDB_CUDA(cudaMemcpyAsync(e->exclFlat.p, exclFlat, sizeof(int) * nex, cudaMemcpyHostToDevice,
                             s));
  // the cluster search reads each excluded pair from both atoms' rows
  cluster_symmetric_excl(n, start.data(), exclFlat, e->hExclStartSym, e->hExclFlatSym);
  ENG_TRY(e, e->exclStartSym.ensure(sizeof(int) * (n + 1)));
  ENG_TRY(e, e->exclFlatSym.ensure(sizeof(int) * std::max<size_t>(1, e->hExclFlatSym.size())));
  MDB_CUDA(cudaMemcpyAsync(e->exclStartSym.p, e->hExclStartSym.data(), sizeof(int) * (n + 1),
                           cudaMemcpyHostToDevice, s));
  if (!e->hExclFlatSym.empty())
    MDB_CUDA(cudaMemcpyAsync(e->exclFlatSym.p, e->hExclFlatSym.data(),
                             sizeof(int) * e->hExclFlatSym.size(), cudaMemcpyHostToDevice, s));
  e->hasFrozen = false;
  if (frozen) {
    bool any = false;
    for (int i = 0; i < n; ++i) any |= frozen[i] != 0;
    if (any) {
      ENG_TRY(e, e->frozen.ensure(sizeof(int) * n));
      MDB_CUDA(cudaMemcpyAsync(e->frozen.p, frozen, sizeof(int) * n, cudaMemcpyHostToDevice, s));
      e->hasFrozen = true;
    }
  }
  // Ewald self term on the device: -C alpha/sqrt(pi) sum q^2 (src/ewald.c:
  // 165-171), the sum taken in fixed point so it is order independent.
  double qmax2 = 0.;
  for (int i = 0; i < n; ++i) qmax2 = fmax(qmax2, q[i] * q[i]);
  if (qmax2 * (double)n >= 8.0e6) return MDBAS_NB_ERR_OVERFLOW;  // 2^63 / 2^40
  ENG_TRY(e, e->acc64.ensure(sizeof(double) * kFp64AccCount));
  e->accCached = false;  // the accumulators serve as scratch here
  MDB_CUDA(cudaMemsetAsync(e->acc64.p, 0, sizeof(double) * kFp64AccCount, s));
  ENG_TRY(e, sum_q2(n, e->q.as<double>(), reinterpret_cast<long long *>(e->acc64.p), s));
  long long q2 = 0;
  MDB_CUDA(cudaMemcpyAsync(&q2, e->acc64.p, sizeof(q2), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  e->selfE = -e->cfg.chargeConst * e->cfg.alpha * ((double)q2 / kQ2Scale) / kSqrtPi;
  e->topoSet = true;
  e->built = false;
  e->mdGraphStale = true;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_set_positions(mdbas_nb_engine *e, const double *x, const double *y,
                                  const double *z, int device_ptrs) {
  if (!e || !x || !y || !z) return MDBAS_NB_ERR_ARG;
  ENG_TRY(e, set_dev(e));
  // a pending build belongs to the positions about to be replaced
  ENG_TRY(e, engine_resolve_build(e));
  const int n = e->n;
  ENG_TRY(e, e->x.ensure(sizeof(double) * n));
  ENG_TRY(e, e->y.ensure(sizeof(double) * n));
  ENG_TRY(e, e->z.ensure(sizeof(double) * n));
  const cudaMemcpyKind k = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  MDB_CUDA(cudaMemcpyAsync(e->x.p, x, sizeof(double) * n, k, e->stream));
  MDB_CUDA(cudaMemcpyAsync(e->y.p, y, sizeof(double) * n, k, e->stream));
  MDB_CUDA(cudaMemcpyAsync(e->z.p, z, sizeof(double) * n, k, e->stream));
  e->posSet = true;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_build(mdbas_nb_engine *e) {
  if (!e) return MDBAS_NB_ERR_ARG;
  if (!e->topoSet || !e->posSet) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  LaunchScope ls(e);
  const int n = e->n;
  const int *frozen = e->hasFrozen ? e->frozen.as<int>() : nullptr;
  if (e->cfg.precision == 0) {
    const int lc = makelist_uses_link_cells(e->box, e->cfg.cutOff, e->cfg.delr,
                                            e->cfg.linkRatio, e->cfg.noLink);
    ENG_TRY(e, build_ref_list(e->ref, n, e->box, e->cfg.cutOff, e->cfg.delr, e->cfg.linkRatio,
                              lc, e->x.as<double>(), e->y.as<double>(), e->z.as<double>(),
                              frozen, e->exclStart.as<int>(), e->exclFlat.as<int>(), e->stream));
  } else {
    e->buildPending = false;
    if (e->built && e->cl.entryCap > 0 && e->cl.sticky.p) {
      // Grid, tables and capacities of the previous build still fit: build
      // without waiting for the counts.  An overflow zeroes the list on the
      // device and is settled by the next call that returns results.
      MDB_CUDA(cudaMemsetAsync(e->cl.sticky.p, 0, sizeof(long long), e->stream));
      const int st = cluster_build(e->cl, n, e->nRep, e->repBoxes.data(), e->repOff.data(),
                                   e->cfg.cutOff, e->cfg.delr, engine_list_rule(e),
                                   sqrt(e->cfg.chargeConst), e->x.as<double>(),
                                   e->y.as<double>(), e->z.as<double>(), e->q.as<double>(),
                                   e->eps.as<double>(), e->sig.as<double>(), frozen,
                                   e->exclStartSym.as<int>(), e->exclFlatSym.as<int>(),
                                   e->stream, false);
      if (st == MDBAS_NB_OK) {
        e->buildPending = true;
        return MDBAS_NB_OK;
      }
      if (st != MDBAS_NB_ERR_STATE) ENG_TRY(e, st);
    }
    ENG_TRY(e, sync_build(e));
  }
  e->built = true;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_refresh(mdbas_nb_engine *e) {
  if (!e) return MDBAS_NB_ERR_ARG;
  if (!e->built) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  LaunchScope ls(e);
  if (e->cfg.precision == 1)
    ENG_TRY(e, cluster_refresh(e->cl, e->x.as<double>(), e->y.as<double>(),
                               e->z.as<double>(), e->q.as<double>(), sqrt(e->cfg.chargeConst),
                               e->stream));
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_compute(mdbas_nb_engine *e) {
  if (!e) return MDBAS_NB_ERR_ARG;
  if (!e->built) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  LaunchScope ls(e);
  const int n = e->n;
  cudaStream_t s = e->stream;
  if (e->cfg.precision == 0) {
    ENG_TRY(e, e->f64.ensure(sizeof(double) * 3 * (size_t)n));
    MDB_CUDA(cudaMemsetAsync(e->f64.p, 0, sizeof(double) * 3 * (size_t)n, s));
    MDB_CUDA(cudaMemsetAsync(e->acc64.p, 0, sizeof(double) * kFp64AccCount, s));
    double *fx = e->f64.as<double>(), *fy = fx + n, *fz = fy + n;
    if (e->timing) MDB_CUDA(cudaEventRecord(e->ev0, s));
    ENG_TRY(e, pairs_fp64(1, n, e->box, e->pp, e->ref.order.as<int>(), e->ref.neighPair.as<int>(),
                          e->ref.off.as<long long>(), e->ref.list.as<int>(), e->x.as<double>(),
                          e->y.as<double>(), e->z.as<double>(), e->q.as<double>(),
                          e->eps.as<double>(), e->sig.as<double>(), fx, fy, fz,
                          e->acc64.as<double>(), s));
    if (e->timing) MDB_CUDA(cudaEventRecord(e->ev1, s));
    ENG_TRY(e, excl_fp64(n, e->box, e->pp, e->exclStart.as<int>(), e->exclFlat.as<int>(),
                         e->x.as<double>(), e->y.as<double>(), e->z.as<double>(),
                         e->q.as<double>(), fx, fy, fz, e->acc64.as<double>(), s));
  } else {
    ClusterWork &w = e->cl;
    MDB_CUDA(cudaMemsetAsync(w.facc.p, 0, sizeof(long long) * 3 * (size_t)w.slotCap, s));
    MDB_CUDA(cudaMemsetAsync(w.acc.p, 0, sizeof(long long) * ACC_COUNT, s));
    if (e->grid <= 0) {
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
      e->grid = sms * 8;
      e->block = 256;
    }
    ENG_TRY(e, engine_side_stream(e));
    // the exclusion correction on the side stream, overlapping the pair
    // kernel's tail; the main stream waits for it before anything reads.
    // Once forked, the join is made whatever fails in between, so no later
    // work on the main stream can run beside the side stream's kernel.
    MDB_CUDA(cudaEventRecord(e->evFork, s));
    MDB_CUDA(cudaStreamWaitEvent(e->side, e->evFork, 0));
    int st = excl_fix_launch(w, n, e->pp, e->exclStartSym.as<int>(), e->exclFlatSym.as<int>(),
                             e->x.as<double>(), e->y.as<double>(), e->z.as<double>(),
                             e->q.as<double>(), e->side);
    const cudaError_t rj = cudaEventRecord(e->evJoin, e->side);
    if (st == MDBAS_NB_OK && e->timing) st = ev_record(e->ev0, s);
    if (st == MDBAS_NB_OK) st = pair_fp32_launch(w, e->pp, e->grid, e->block, s, e->variant);
    if (st == MDBAS_NB_OK && e->timing) st = ev_record(e->ev1, s);
    if (rj == cudaSuccess) {
      MDB_CUDA(cudaStreamWaitEvent(s, e->evJoin, 0));
    } else {
      MDB_CUDA(cudaStreamSynchronize(e->side));  // no join event: wait for the side work
      MDB_CUDA(rj);
    }
    ENG_TRY(e, st);
  }
  if (e->timing) {
    MDB_CUDA(cudaEventSynchronize(e->ev1));
    float ms = 0.f;
    MDB_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    e->pairMs += ms;
    e->pairCount += 1;
  }
  e->computed = true;
  e->accCached = false;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_get_forces(mdbas_nb_engine *e, double *fx, double *fy, double *fz,
                               int device_ptrs) {
  if (!e || !fx || !fy || !fz) return MDBAS_NB_ERR_ARG;
  if (!e->computed) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  // Host arrays after a build that did not wait for its counts: the build's
  // error word is read with the forces and the energy words, one wait for all
  // three; a build that failed is settled (rebuilt and evaluated again) and
  // the copies are made once more.
  const bool settleAfter = !device_ptrs && e->buildPending;
  if (!settleAfter) ENG_TRY(e, engine_resolve_build(e));
  LaunchScope ls(e);
  const int n = e->n;
  cudaStream_t s = e->stream;
  for (int pass = 0;; ++pass) {
    double *src;
    if (e->cfg.precision == 0) {
      src = e->f64.as<double>();
    } else {
      ENG_TRY(e, e->fout.ensure(sizeof(double) * 3 * (size_t)n));
      src = e->fout.as<double>();
      ENG_TRY(e, forces_out_launch(e->cl, n, 0, src, src + n, src + 2 * (size_t)n, s));
    }
    const cudaMemcpyKind k = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    MDB_CUDA(cudaMemcpyAsync(fx, src, sizeof(double) * n, k, s));
    MDB_CUDA(cudaMemcpyAsync(fy, src + n, sizeof(double) * n, k, s));
    MDB_CUDA(cudaMemcpyAsync(fz, src + 2 * (size_t)n, sizeof(double) * n, k, s));
    if (device_ptrs) return MDBAS_NB_OK;
    // the energy words ride along with the forces: one wait for both, and the
    // fixed-point error bits checked here too
    if (e->cfg.precision == 0)
      MDB_CUDA(cudaMemcpyAsync(e->acc64Cache, e->acc64.p, sizeof(e->acc64Cache),
                               cudaMemcpyDeviceToHost, s));
    else
      MDB_CUDA(cudaMemcpyAsync(e->accCache, e->cl.acc.p, sizeof(e->accCache),
                               cudaMemcpyDeviceToHost, s));
    long long sticky = 0;
    const bool settle = settleAfter && pass == 0 && e->buildPending;
    if (settle)
      MDB_CUDA(cudaMemcpyAsync(&sticky, e->cl.sticky.p, sizeof(sticky), cudaMemcpyDeviceToHost,
                               s));
    MDB_CUDA(cudaStreamSynchronize(s));
    if (!settle) break;
    e->buildPending = false;
    if (!(sticky & (CL_OVERFLOW | CL_NONFINITE))) break;
    ENG_TRY(e, engine_settle_build(e, sticky));
  }
  e->accCached = true;
  return acc_status(e);
}

int mdbas_nb_engine_energies(mdbas_nb_engine *e, mdbas_nb_energies *out) {
  if (!e || !out) return MDBAS_NB_ERR_ARG;
  if (!e->computed) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  ENG_TRY(e, engine_resolve_build(e));
  cudaStream_t s = e->stream;
  memset(out, 0, sizeof(*out));
  out->elec_self = e->selfE;
  if (!e->accCached) {
    if (e->cfg.precision == 0)
      MDB_CUDA(cudaMemcpyAsync(e->acc64Cache, e->acc64.p, sizeof(e->acc64Cache),
                               cudaMemcpyDeviceToHost, s));
    else
      MDB_CUDA(cudaMemcpyAsync(e->accCache, e->cl.acc.p, sizeof(e->accCache),
                               cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaStreamSynchronize(s));
    e->accCached = true;
  }
  if (e->cfg.precision == 0) {
    const double *a = e->acc64Cache;
    out->elec_direct = a[0];
    out->vdw = a[1];
    out->vir_direct = a[2];
    out->vir_vdw = a[3];
    out->n_pairs = a[4];
    out->elec_corr = a[5];
    out->vir_corr = a[6];
    return MDBAS_NB_OK;
  }
  const long long *a = e->accCache;
  const double inv = 1.0 / kEnergyScale;
  out->elec_direct = (double)a[ACC_E_DIR] * inv;
  out->elec_corr = (double)a[ACC_E_CORR] * inv;
  out->vdw = (double)a[ACC_E_VDW] * inv;
  out->vir_direct = (double)a[ACC_V_DIR] * inv;
  out->vir_corr = (double)a[ACC_V_CORR] * inv;
  out->vir_vdw = (double)a[ACC_V_VDW] * inv;
  out->n_pairs = (double)a[ACC_NPAIR];
  return acc_status(e);
}

int mdbas_nb_engine_evaluate(mdbas_nb_engine *e, const double *x, const double *y,
                             const double *z, int rebuild, double *fx, double *fy, double *fz,
                             mdbas_nb_energies *out) {
  if (!e || !x || !y || !z || !fx || !fy || !fz) return MDBAS_NB_ERR_ARG;
  int st = mdbas_nb_engine_set_positions(e, x, y, z, 0);
  if (st != MDBAS_NB_OK) return st;
  st = (rebuild || !e->built) ? mdbas_nb_engine_build(e) : mdbas_nb_engine_refresh(e);
  if (st != MDBAS_NB_OK) return st;
  st = mdbas_nb_engine_compute(e);
  if (st != MDBAS_NB_OK) return st;
  st = mdbas_nb_engine_get_forces(e, fx, fy, fz, 0);
  if (st != MDBAS_NB_OK || !out) return st;
  return mdbas_nb_engine_energies(e, out);
}

int mdbas_nb_engine_list_stats(mdbas_nb_engine *e, long long out[4]) {
  if (!e || !out) return MDBAS_NB_ERR_ARG;
  if (!e->built) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  ENG_TRY(e, engine_resolve_build(e));
  if (e->cfg.precision == 0) {
    out[0] = e->n;
    out[1] = e->ref.entries;
    out[2] = e->ref.entries;
    out[3] = (long long)(e->ref.list.bytes / sizeof(int));
  } else {
    ENG_TRY(e, set_dev(e));
    ENG_TRY(e, cluster_read_counts(e->cl, e->stream));
    out[0] = e->cl.nClusters;
    out[1] = e->cl.nEntries;
    // pair slots the default kernel evaluates: 64 per warp step, one step
    // per two inner-list halves (rounded up per item), or per full-list entry
    out[2] = (e->cl.useInner ? e->cl.nInSteps : e->cl.nEntries) * 64;
    out[3] = e->cl.entryCap;
  }
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_export_pairs(mdbas_nb_engine *e, double r2max, int *pairs,
                                 long long capacity, long long *count) {
  if (!e || !count) return MDBAS_NB_ERR_ARG;
  if (!e->built) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  ENG_TRY(e, engine_resolve_build(e));
  LaunchScope ls(e);
  cudaStream_t s = e->stream;
  ENG_TRY(e, e->exportCount.ensure(sizeof(unsigned long long)));
  MDB_CUDA(cudaMemsetAsync(e->exportCount.p, 0, sizeof(unsigned long long), s));
  long long cap = pairs ? capacity : 0;
  ENG_TRY(e, e->exportBuf.ensure(sizeof(int) * 2 * (size_t)(cap > 0 ? cap : 1)));
  if (e->cfg.precision == 0) {
    MDB_LAUNCH(k_export_ref_pairs, grid_for(e->n, 128), 128, 0, s, e->n, e->box,
               e->ref.order.as<int>(), e->ref.neighPair.as<int>(), e->ref.off.as<long long>(),
               e->ref.list.as<int>(), e->x.as<double>(), e->y.as<double>(), e->z.as<double>(),
               r2max, e->exportBuf.as<int>(), cap, e->exportCount.as<unsigned long long>());
  } else {
    ENG_TRY(e, cluster_read_counts(e->cl, s));
    MDB_LAUNCH(k_export_cluster_pairs, grid_for(e->cl.nItems * 32, 128), 128, 0, s,
               e->cl.nEntries, e->cl.items.as<int4>(), e->cl.nItems,
               e->cl.entries.as<CPairEntry>(), e->cl.masks.as<uint2>(), e->cl.xq.as<float4>(),
               e->cl.slotAtom.as<int>(), (float)r2max, e->exportBuf.as<int>(), cap,
               e->exportCount.as<unsigned long long>());
  }
  unsigned long long c = 0;
  MDB_CUDA(cudaMemcpyAsync(&c, e->exportCount.p, sizeof(c), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  *count = (long long)c;
  if (pairs && cap > 0) {
    const long long m = (long long)c < cap ? (long long)c : cap;
    MDB_CUDA(cudaMemcpy(pairs, e->exportBuf.p, sizeof(int) * 2 * (size_t)m,
                        cudaMemcpyDeviceToHost));
  }
  return MDBAS_NB_OK;
}

long long mdbas_nb_engine_launch_count(mdbas_nb_engine *e) { return e ? e->launches : -1; }

int mdbas_nb_engine_build_stages(mdbas_nb_engine *e, double ms[6]) {
  if (!e || !ms) return MDBAS_NB_ERR_ARG;
  if (e->cfg.precision != 1) return MDBAS_NB_ERR_UNSUPPORTED;
  if (!e->topoSet || !e->posSet) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  ENG_TRY(e, engine_resolve_build(e));
  LaunchScope ls(e);
  const int *frozen = e->hasFrozen ? e->frozen.as<int>() : nullptr;
  ENG_TRY(e, cluster_build_stages(e->cl, e->n, e->nRep, e->repBoxes.data(), e->repOff.data(),
                                  e->cfg.cutOff, e->cfg.delr, engine_list_rule(e),
                                  sqrt(e->cfg.chargeConst), e->x.as<double>(),
                                  e->y.as<double>(), e->z.as<double>(), e->q.as<double>(),
                                  e->eps.as<double>(), e->sig.as<double>(), frozen,
                                  e->exclStartSym.as<int>(), e->exclFlatSym.as<int>(),
                                  e->stream, ms));
  e->built = true;
  e->buildPending = false;
  e->computed = false;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_autotune(mdbas_nb_engine *e, int out[4]) {
  if (!e || !out) return MDBAS_NB_ERR_ARG;
  if (e->cfg.precision != 1) return MDBAS_NB_ERR_UNSUPPORTED;
  if (!e->built) return MDBAS_NB_ERR_STATE;
  ENG_TRY(e, set_dev(e));
  ENG_TRY(e, engine_resolve_build(e));
  e->accCached = false;  // the trial launches overwrite the accumulators
  LaunchScope ls(e);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  struct Cand { int variant, block, bps; };
  std::vector<Cand> cands;
  // the dense kernel takes at most 256 threads per block (launch bounds)
  for (int variant : {kPairHalf, kPairHalfLean, kPairHalf3, kPairQuad, kPairPacked, kPairBulk,
                      kPairDense})
    for (int block : {64, 128, 256})
      for (int bps : {2, 4, 8, 16, 32})
        if (block * bps <= 2048 && bps <= 24) cands.push_back({variant, block, bps});
  for (int bps : {2, 4, 5}) cands.push_back({kPairCompact, 128, bps});
  ClusterWork &w = e->cl;
  cudaStream_t s = e->stream;
  float best = 1e30f;
  Cand pick = cands[0];
  for (const Cand &c : cands) {
    float tmin = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      MDB_CUDA(cudaMemsetAsync(w.facc.p, 0, sizeof(long long) * 3 * (size_t)w.slotCap, s));
      MDB_CUDA(cudaMemsetAsync(w.acc.p, 0, sizeof(long long) * ACC_COUNT, s));
      MDB_CUDA(cudaEventRecord(e->ev0, s));
      ENG_TRY(e, pair_fp32_launch(w, e->pp, sms * c.bps, c.block, s, c.variant));
      MDB_CUDA(cudaEventRecord(e->ev1, s));
      MDB_CUDA(cudaEventSynchronize(e->ev1));
      float ms = 0.f;
      MDB_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
      if (rep > 0) tmin = std::min(tmin, ms);  // the first run warms up
    }
    if (tmin < best) {
      best = tmin;
      pick = c;
    }
  }
  e->variant = pick.variant;
  e->grid = sms * pick.bps;
  e->block = pick.block;
  e->computed = false;
  e->mdGraphStale = true;
  out[0] = pick.variant;
  out[1] = pick.block;
  out[2] = pick.bps;
  out[3] = (int)cands.size();
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_set_variant(mdbas_nb_engine *e, int variant) {
  if (!e || (variant != kPairDense && variant != kPairCompact && variant != kPairPacked &&
             variant != kPairBulk && variant != kPairHalf && variant != kPairHalf3 &&
             variant != kPairQuad && variant != kPairHalfLean))
    return MDBAS_NB_ERR_ARG;
  e->variant = variant;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_set_timing(mdbas_nb_engine *e, int enable) {
  if (!e) return MDBAS_NB_ERR_ARG;
  e->timing = enable != 0;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_kernel_time(mdbas_nb_engine *e, int which, double *avg_ms, long long *count,
                                int reset) {
  if (!e || !avg_ms || !count) return MDBAS_NB_ERR_ARG;
  (void)which;
  *count = e->pairCount;
  *avg_ms = e->pairCount ? e->pairMs / (double)e->pairCount : 0.0;
  if (reset) {
    e->pairMs = 0.0;
    e->pairCount = 0;
  }
  return MDBAS_NB_OK;
}

}  // extern "C"
