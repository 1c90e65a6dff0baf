// bonded.cu -- MDBas's bonded terms on the GPU: harmonic and Morse bonds,
// Urey-Bradley, harmonic angles, cosine and harmonic dihedrals and impropers
// (src/internal.c:21-620), in FP64 with MDBas's operation order.
//
// One thread per term writes the term's energy and its force on each of its
// atoms into private slots; one thread per atom then adds its slots to the
// atom's force in MDBas's accumulation order (kind, term, atom within the
// term).  This file is compiled with --fmad=false, so the arithmetic that
// has no library call in it (harmonic bonds and Urey-Bradley terms) gives
// MDBas's bits exactly; exp, acos, atan2, cos and sin are CUDA's and may
// differ from the host C library's in the last place.
#include <float.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "bonded.cuh"
#include "engine.cuh"

namespace mdbas {
namespace {

constexpr int kBondedBlock = 128;

struct BondedArgs {
  const BOND *bond;
  const ANGLE *angle;
  const BOND *ub;
  const DIHE *dihe;
  const DIHE *impr;
  int termBase[KIND_COUNT + 1];
  int slotBase[KIND_COUNT + 1];
  int nSlots;
};

__device__ __forceinline__ void put(double *c, int nSlots, int slot, double vx, double vy,
                                    double vz) {
  c[slot] = vx;
  c[nSlots + slot] = vy;
  c[2 * (size_t)nSlots + slot] = vz;
}

// Harmonic (BHARM and any unknown type) or Morse bond; Urey-Bradley terms
// are always harmonic (src/internal.c:21-171).
__device__ void eval_bond(const BOND &bd, bool ub, const DevBox &b, const double *x,
                          const double *y, const double *z, double *c, int nSlots, int slot,
                          double &e, double &v) {
  const int i = bd.a, j = bd.b;
  double d0 = x[j] - x[i], d1 = y[j] - y[i], d2 = z[j] - z[i];
  const double r = sqrt(dist_d(b, d0, d1, d2));
  const double dr = r - bd.r0;
  double db;
  if (!ub && bd.type == BMORSE) {
    const double ma = exp(-bd.beta * dr);
    const double mb = ma * ma;
    e = bd.k * (mb - 2. * ma) + bd.k;
    db = 2. * bd.k * bd.beta * (ma - mb);
  } else {
    e = 0.5 * bd.k * (dr * dr);
    db = bd.k * dr;
  }
  v = db * r;
  const double tx = db * d0 / r, ty = db * d1 / r, tz = db * d2 / r;
  put(c, nSlots, slot, tx, ty, tz);
  put(c, nSlots, slot + 1, -tx, -ty, -tz);
}

// Harmonic angle (src/internal.c:173-256).
__device__ void eval_angle(const ANGLE &an, const DevBox &b, const double *x, const double *y,
                           const double *z, double *c, int nSlots, int slot, double &e) {
  const int i = an.a, j = an.b, k = an.c;
  double ab0 = x[i] - x[j], ab1 = y[i] - y[j], ab2 = z[i] - z[j];
  const double rab = sqrt(dist_d(b, ab0, ab1, ab2));
  const double rabt = 1. / rab;
  double bc0 = x[k] - x[j], bc1 = y[k] - y[j], bc2 = z[k] - z[j];
  const double rbc = sqrt(dist_d(b, bc0, bc1, bc2));
  const double rbct = 1. / rbc;
  const double cost = (ab0 * bc0 + ab1 * bc1 + ab2 * bc2) / (rab * rbc);
  const double s = sqrt(1. - (cost * cost));
  const double sint = 1.e-8 >= s ? 1.e-8 : s;
  const double theta = acos(cost);
  const double dt = theta - an.theta0;
  e = 0.5 * an.k * (dt * dt);
  const double da = an.k * dt / sint;
  const double fxa = da * (bc0 * rbct - ab0 * cost * rabt) * rabt;
  const double fya = da * (bc1 * rbct - ab1 * cost * rabt) * rabt;
  const double fza = da * (bc2 * rbct - ab2 * cost * rabt) * rabt;
  const double fxc = da * (ab0 * rabt - bc0 * cost * rbct) * rbct;
  const double fyc = da * (ab1 * rabt - bc1 * cost * rbct) * rbct;
  const double fzc = da * (ab2 * rabt - bc2 * cost * rbct) * rbct;
  put(c, nSlots, slot, fxa, fya, fza);
  put(c, nSlots, slot + 1, -fxa - fxc, -fya - fyc, -fza - fzc);
  put(c, nSlots, slot + 2, fxc, fyc, fzc);
}

// Dihedral or improper: cosine (DCOS and any unknown type) or harmonic
// (DHARM) in the angle between the planes (i,j,k) and (j,k,l)
// (src/internal.c:258-620; both routines are the same formula).
__device__ void eval_torsion(const DIHE &dh, const DevBox &b, const double *x, const double *y,
                             const double *z, double *c, int nSlots, int slot, double &e) {
  const int i = dh.a, j = dh.b, k = dh.c, l = dh.d;
  double ab0 = x[i] - x[j], ab1 = y[i] - y[j], ab2 = z[i] - z[j];
  dist_d(b, ab0, ab1, ab2);
  double bc0 = x[j] - x[k], bc1 = y[j] - y[k], bc2 = z[j] - z[k];
  const double rbc = sqrt(dist_d(b, bc0, bc1, bc2));
  double cd0 = x[k] - x[l], cd1 = y[k] - y[l], cd2 = z[k] - z[l];
  dist_d(b, cd0, cd1, cd2);
  // normals of the two planes
  const double pb0 = ab1 * bc2 - ab2 * bc1;
  const double pb1 = ab2 * bc0 - ab0 * bc2;
  const double pb2 = ab0 * bc1 - ab1 * bc0;
  const double r2pb = pb0 * pb0 + pb1 * pb1 + pb2 * pb2;
  const double rpb = sqrt(r2pb);
  const double pc0 = bc1 * cd2 - bc2 * cd1;
  const double pc1 = bc2 * cd0 - bc0 * cd2;
  const double pc2 = bc0 * cd1 - bc1 * cd0;
  const double r2pc = pc0 * pc0 + pc1 * pc1 + pc2 * pc2;
  const double rpc = sqrt(r2pc);
  const double pbpc = pb0 * pc0 + pb1 * pc1 + pb2 * pc2;
  const double cosp = pbpc / (rpb * rpc);
  double sinp = (bc0 * (pc1 * pb2 - pc2 * pb1) + bc1 * (pb0 * pc2 - pb2 * pc0) +
                 bc2 * (pc0 * pb1 - pc1 * pb0)) / (rpb * rpc * rbc);
  double phi = atan2(sinp, cosp);
  // keep sinp away from zero, with its sign
  const double as = fabs(sinp);
  const double asc = DBL_EPSILON >= as ? DBL_EPSILON : as;
  sinp = sinp >= 0. ? asc : -asc;
  double dd;
  if (dh.type == DHARM) {
    const double twopi = 2. * 3.141592653589793;
    phi = phi - dh.phi0;
    phi = phi - (double)nint_d(phi / twopi) * twopi;
    e = 0.5 * dh.k * (phi * phi);
    dd = dh.k * phi / (rpb * rpc * sinp);
  } else {
    const double arg = dh.mult * phi - dh.phi0;
    e = dh.k * (1. + cos(arg));
    dd = -dh.k * dh.mult * sin(arg) / (rpb * rpc * sinp);
  }
  const double fax = dd * ((-pc1 * bc2 + pc2 * bc1) - pbpc * (-pb1 * bc2 + pb2 * bc1) / r2pb);
  const double fay = dd * (( pc0 * bc2 - pc2 * bc0) - pbpc * ( pb0 * bc2 - pb2 * bc0) / r2pb);
  const double faz = dd * ((-pc0 * bc1 + pc1 * bc0) - pbpc * (-pb0 * bc1 + pb1 * bc0) / r2pb);
  const double fcx = dd * ((-pc1 * ab2 + pc2 * ab1) - pbpc * (-pb1 * ab2 + pb2 * ab1) / r2pb);
  const double fcy = dd * (( pc0 * ab2 - pc2 * ab0) - pbpc * ( pb0 * ab2 - pb2 * ab0) / r2pb);
  const double fcz = dd * ((-pc0 * ab1 + pc1 * ab0) - pbpc * (-pb0 * ab1 + pb1 * ab0) / r2pb);
  const double fbx = dd * ((-pb1 * cd2 + pb2 * cd1) - pbpc * (-pc1 * cd2 + pc2 * cd1) / r2pc);
  const double fby = dd * (( pb0 * cd2 - pb2 * cd0) - pbpc * ( pc0 * cd2 - pc2 * cd0) / r2pc);
  const double fbz = dd * ((-pb0 * cd1 + pb1 * cd0) - pbpc * (-pc0 * cd1 + pc1 * cd0) / r2pc);
  const double fdx = dd * ((-pb1 * bc2 + pb2 * bc1) - pbpc * (-pc1 * bc2 + pc2 * bc1) / r2pc);
  const double fdy = dd * (( pb0 * bc2 - pb2 * bc0) - pbpc * ( pc0 * bc2 - pc2 * bc0) / r2pc);
  const double fdz = dd * ((-pb0 * bc1 + pb1 * bc0) - pbpc * (-pc0 * bc1 + pc1 * bc0) / r2pc);
  put(c, nSlots, slot, fax, fay, faz);
  put(c, nSlots, slot + 1, -fax - fcx + fbx, -fay - fcy + fby, -faz - fcz + fbz);
  put(c, nSlots, slot + 2, fcx - fbx - fdx, fcy - fby - fdy, fcz - fbz - fdz);
  put(c, nSlots, slot + 3, fdx, fdy, fdz);
}

// One thread per term (all kinds in one launch); per-block partial sums of
// the five energies and two virials into part[q * gridDim.x + block].
__global__ void __launch_bounds__(kBondedBlock)
    k_bonded_terms(BondedArgs a, const DevBox *__restrict__ boxes, const int *__restrict__ atomRep,
                   const double *__restrict__ x, const double *__restrict__ y,
                   const double *__restrict__ z, double *__restrict__ contrib,
                   double *__restrict__ part) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int kind = -1;
  double e = 0., v = 0.;
  if (t < a.termBase[KIND_COUNT]) {
    kind = t < a.termBase[1] ? 0 : t < a.termBase[2] ? 1 : t < a.termBase[3] ? 2
           : t < a.termBase[4] ? 3 : 4;
    const int u = t - a.termBase[kind];
    switch (kind) {
      case KIND_BOND: {
        const BOND bd = a.bond[u];
        const DevBox &b = boxes[atomRep ? atomRep[bd.a] : 0];
        eval_bond(bd, false, b, x, y, z, contrib, a.nSlots, a.slotBase[KIND_BOND] + 2 * u, e, v);
        break;
      }
      case KIND_ANGLE: {
        const ANGLE an = a.angle[u];
        const DevBox &b = boxes[atomRep ? atomRep[an.a] : 0];
        eval_angle(an, b, x, y, z, contrib, a.nSlots, a.slotBase[KIND_ANGLE] + 3 * u, e);
        break;
      }
      case KIND_UB: {
        const BOND bd = a.ub[u];
        const DevBox &b = boxes[atomRep ? atomRep[bd.a] : 0];
        eval_bond(bd, true, b, x, y, z, contrib, a.nSlots, a.slotBase[KIND_UB] + 2 * u, e, v);
        break;
      }
      default: {
        const DIHE dh = kind == KIND_DIHEDRAL ? a.dihe[u] : a.impr[u];
        const DevBox &b = boxes[atomRep ? atomRep[dh.a] : 0];
        eval_torsion(dh, b, x, y, z, contrib, a.nSlots, a.slotBase[kind] + 4 * u, e);
        break;
      }
    }
  }
  __shared__ double red[BS_FIX][kBondedBlock / 32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < BS_FIX; ++q) {
    const double val = q < KIND_COUNT ? (kind == q ? e : 0.)
                       : q == BS_VIRBOND ? (kind == KIND_BOND ? v : 0.)
                                         : (kind == KIND_UB ? v : 0.);
    const double sw = warp_sum_d(val);
    if (lane == 0) red[q][w] = sw;
  }
  __syncthreads();
  if (threadIdx.x < BS_FIX) {
    double s = 0.;
    for (int k = 0; k < kBondedBlock / 32; ++k) s += red[threadIdx.x][k];
    part[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
}

// f[i] += the atom's slots, in slot order (MDBas's order of additions).
__global__ void k_bonded_gather(int n, const int *__restrict__ start,
                                const int *__restrict__ slots, const double *__restrict__ contrib,
                                int nSlots, double *__restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s0 = start[i], s1 = start[i + 1];
  if (s0 == s1) return;
  double fx = f[i], fy = f[n + i], fz = f[2 * (size_t)n + i];
  for (int s = s0; s < s1; ++s) {
    const int k = slots[s];
    fx += contrib[k];
    fy += contrib[nSlots + k];
    fz += contrib[2 * (size_t)nSlots + k];
  }
  f[i] = fx;
  f[n + i] = fy;
  f[2 * (size_t)n + i] = fz;
}

// Sums of the block partials in a fixed order; the total energy also in
// fixed point (int64 bits in sums[BS_FIX]) for the dynamics rows.
__global__ void k_bonded_finish(int nPart, const double *__restrict__ part,
                                double *__restrict__ sums) {
  __shared__ double red[256 / 32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = 0; q < BS_FIX; ++q) {
    double s = 0.;
    for (int b = threadIdx.x; b < nPart; b += blockDim.x) s += part[(size_t)q * nPart + b];
    s = warp_sum_d(s);
    if (lane == 0) red[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double tot = 0.;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) tot += red[k];
      sums[q] = tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double tot = (((sums[0] + sums[1]) + sums[2]) + sums[3]) + sums[4];
    reinterpret_cast<long long *>(sums)[BS_FIX] = fix_e(tot);
  }
}

const int kArity[KIND_COUNT] = {2, 3, 2, 4, 4};
const size_t kTermSize[KIND_COUNT] = {sizeof(BOND), sizeof(ANGLE), sizeof(BOND), sizeof(DIHE),
                                      sizeof(DIHE)};

void term_atoms(int kind, const void *terms, int u, int out[4]) {
  if (kind == KIND_BOND || kind == KIND_UB) {
    const BOND &b = static_cast<const BOND *>(terms)[u];
    out[0] = b.a;
    out[1] = b.b;
  } else if (kind == KIND_ANGLE) {
    const ANGLE &a = static_cast<const ANGLE *>(terms)[u];
    out[0] = a.a;
    out[1] = a.b;
    out[2] = a.c;
  } else {
    const DIHE &d = static_cast<const DIHE *>(terms)[u];
    out[0] = d.a;
    out[1] = d.b;
    out[2] = d.c;
    out[3] = d.d;
  }
}

}  // namespace

int bonded_set(BondedTerms &t, int nAtom, const int count[KIND_COUNT],
               const void *const terms[KIND_COUNT], cudaStream_t s) {
  if (nAtom <= 0) return MDBAS_NB_ERR_ARG;
  long long nt = 0, ns = 0;
  for (int k = 0; k < KIND_COUNT; ++k) {
    if (count[k] < 0 || (count[k] > 0 && !terms[k])) return MDBAS_NB_ERR_ARG;
    nt += count[k];
    ns += (long long)kArity[k] * count[k];
  }
  if (ns > 0x7fffffffLL) return MDBAS_NB_ERR_ARG;
  // slot lists: count per atom, then fill in slot order
  std::vector<int> start(nAtom + 1, 0), slots((size_t)ns);
  for (int k = 0; k < KIND_COUNT; ++k)
    for (int u = 0; u < count[k]; ++u) {
      int at[4];
      term_atoms(k, terms[k], u, at);
      for (int p = 0; p < kArity[k]; ++p) {
        if (at[p] < 0 || at[p] >= nAtom) {
          set_last_status(MDBAS_NB_ERR_ARG, "bonded term atom index out of range");
          return MDBAS_NB_ERR_ARG;
        }
        ++start[at[p] + 1];
      }
    }
  for (int i = 0; i < nAtom; ++i) start[i + 1] += start[i];
  std::vector<int> fill(start.begin(), start.end() - 1);
  int slot = 0;
  for (int k = 0; k < KIND_COUNT; ++k)
    for (int u = 0; u < count[k]; ++u) {
      int at[4];
      term_atoms(k, terms[k], u, at);
      for (int p = 0; p < kArity[k]; ++p) slots[fill[at[p]]++] = slot++;
    }
  t.nAtom = 0;  // invalid until every upload below is queued
  for (int k = 0; k < KIND_COUNT; ++k) {
    MDB_TRY(t.terms[k].ensure(kTermSize[k] * (size_t)(count[k] > 0 ? count[k] : 1)));
    if (count[k] > 0)
      MDB_CUDA(cudaMemcpyAsync(t.terms[k].p, terms[k], kTermSize[k] * (size_t)count[k],
                               cudaMemcpyHostToDevice, s));
  }
  const size_t nsl = (size_t)(ns > 0 ? ns : 1);
  MDB_TRY(t.contrib.ensure(sizeof(double) * 3 * nsl));
  MDB_TRY(t.atomStart.ensure(sizeof(int) * (size_t)(nAtom + 1)));
  MDB_TRY(t.atomSlot.ensure(sizeof(int) * nsl));
  const int nb = grid_for(nt, kBondedBlock);
  MDB_TRY(t.part.ensure(sizeof(double) * BS_FIX * (size_t)nb));
  MDB_TRY(t.sums.ensure(sizeof(double) * BS_COUNT));
  MDB_CUDA(cudaMemcpyAsync(t.atomStart.p, start.data(), sizeof(int) * (size_t)(nAtom + 1),
                           cudaMemcpyHostToDevice, s));
  if (ns > 0)
    MDB_CUDA(cudaMemcpyAsync(t.atomSlot.p, slots.data(), sizeof(int) * (size_t)ns,
                             cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemsetAsync(t.sums.p, 0, sizeof(double) * BS_COUNT, s));
  // the host vectors go out of scope: finish the copies first
  MDB_CUDA(cudaStreamSynchronize(s));
  t.nAtom = nAtom;
  t.termBase[0] = 0;
  t.slotBase[0] = 0;
  for (int k = 0; k < KIND_COUNT; ++k) {
    t.count[k] = count[k];
    t.termBase[k + 1] = t.termBase[k] + count[k];
    t.slotBase[k + 1] = t.slotBase[k] + kArity[k] * count[k];
  }
  return MDBAS_NB_OK;
}

int bonded_eval(BondedTerms &t, const DevBox *boxes, const int *atomRep, const double *x,
                const double *y, const double *z, double *f, cudaStream_t s) {
  const int nt = t.nTerms();
  if (nt == 0 || t.nAtom == 0) return MDBAS_NB_OK;
  BondedArgs a;
  a.bond = t.terms[KIND_BOND].as<BOND>();
  a.angle = t.terms[KIND_ANGLE].as<ANGLE>();
  a.ub = t.terms[KIND_UB].as<BOND>();
  a.dihe = t.terms[KIND_DIHEDRAL].as<DIHE>();
  a.impr = t.terms[KIND_IMPROPER].as<DIHE>();
  for (int k = 0; k <= KIND_COUNT; ++k) {
    a.termBase[k] = t.termBase[k];
    a.slotBase[k] = t.slotBase[k];
  }
  a.nSlots = t.nSlots();
  const int nb = grid_for(nt, kBondedBlock);
  double *c = t.contrib.as<double>(), *part = t.part.as<double>();
  MDB_LAUNCH(k_bonded_terms, nb, kBondedBlock, 0, s, a, boxes, atomRep, x, y, z, c, part);
  MDB_LAUNCH(k_bonded_gather, grid_for(t.nAtom, 256), 256, 0, s, t.nAtom,
             t.atomStart.as<int>(), t.atomSlot.as<int>(), c, a.nSlots, f);
  MDB_LAUNCH(k_bonded_finish, 1, 256, 0, s, nb, part, t.sums.as<double>());
  return MDBAS_NB_OK;
}

}  // namespace mdbas

using namespace mdbas;

namespace {

// Standalone calls (one kind per call, MDBas's per-routine interface).
struct BondedCall {
  BondedTerms terms;
  int kind = -1;
  DBuf xyz, f, box;
};

BondedCall &bonded_call() {
  static BondedCall c;
  return c;
}

const size_t kCallTermSize[KIND_COUNT] = {sizeof(BOND), sizeof(ANGLE), sizeof(BOND),
                                          sizeof(DIHE), sizeof(DIHE)};

}  // namespace

extern "C" int mdbas_nb_bonded(int kind, int nAtom, const PBC *box, int nTerms,
                               const void *terms, const double *x, const double *y,
                               const double *z, double *fx, double *fy, double *fz,
                               double out[2]) {
  if (kind < 0 || kind >= KIND_COUNT || nAtom <= 0 || !box || nTerms < 0 || !x || !y || !z ||
      !fx || !fy || !fz || !out)
    return MDBAS_NB_ERR_ARG;
  out[0] = out[1] = 0.;
  if (nTerms == 0) return MDBAS_NB_OK;
  if (!terms) return MDBAS_NB_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = 0;
  }
  MDB_TRY(engine_check_device(dev));
  BondedCall &c = bonded_call();
  cudaStream_t s = nullptr;
  // the term upload and slot lists are reused while the same terms come back
  const size_t tb = kCallTermSize[kind] * (size_t)nTerms;
  const bool same = c.kind == kind && c.terms.nAtom == nAtom && c.terms.count[kind] == nTerms &&
                    c.terms.hostCopy.size() == tb &&
                    memcmp(c.terms.hostCopy.data(), terms, tb) == 0;
  if (!same) {
    int count[KIND_COUNT] = {0, 0, 0, 0, 0};
    const void *ptrs[KIND_COUNT] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    count[kind] = nTerms;
    ptrs[kind] = terms;
    c.kind = -1;
    MDB_TRY(bonded_set(c.terms, nAtom, count, ptrs, s));
    c.terms.hostCopy.assign(static_cast<const char *>(terms),
                            static_cast<const char *>(terms) + tb);
    c.kind = kind;
  }
  const size_t bytes = sizeof(double) * (size_t)nAtom;
  MDB_TRY(c.xyz.ensure(3 * bytes));
  MDB_TRY(c.f.ensure(3 * bytes));
  MDB_TRY(c.box.ensure(sizeof(DevBox)));
  double *d = c.xyz.as<double>(), *f = c.f.as<double>();
  const DevBox hb = make_devbox(box);
  MDB_CUDA(cudaMemcpyAsync(c.box.p, &hb, sizeof(hb), cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d, x, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d + nAtom, y, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(d + 2 * (size_t)nAtom, z, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(f, fx, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(f + nAtom, fy, bytes, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(f + 2 * (size_t)nAtom, fz, bytes, cudaMemcpyHostToDevice, s));
  MDB_TRY(bonded_eval(c.terms, c.box.as<DevBox>(), nullptr, d, d + nAtom, d + 2 * (size_t)nAtom,
                      f, s));
  double sums[BS_COUNT];
  MDB_CUDA(cudaMemcpyAsync(sums, c.terms.sums.p, sizeof(sums), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaMemcpyAsync(fx, f, bytes, cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaMemcpyAsync(fy, f + nAtom, bytes, cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaMemcpyAsync(fz, f + 2 * (size_t)nAtom, bytes, cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  out[0] = sums[kind];
  out[1] = kind == KIND_BOND ? sums[BS_VIRBOND] : kind == KIND_UB ? sums[BS_VIRUB] : 0.;
  return MDBAS_NB_OK;
}

extern "C" int mdbas_nb_engine_set_bonded(mdbas_nb_engine *e, int nBond, const BOND *bond,
                                          int nAngle, const ANGLE *angle, int nUb, const BOND *ub,
                                          int nDihedral, const DIHE *dihe, int nImproper,
                                          const DIHE *impr) {
  if (!e) return MDBAS_NB_ERR_ARG;
  MDB_CUDA(cudaSetDevice(e->device));
  const int count[KIND_COUNT] = {nBond, nAngle, nUb, nDihedral, nImproper};
  const void *ptrs[KIND_COUNT] = {bond, angle, ub, dihe, impr};
  MDB_TRY(bonded_set(e->bonded, e->n, count, ptrs, e->stream));
  MDB_TRY(e->bondedF.ensure(sizeof(double) * 3 * (size_t)e->n));
  e->mdGraphStale = true;  // the dynamics graph holds the old launches
  return MDBAS_NB_OK;
}

extern "C" int mdbas_nb_engine_bonded(mdbas_nb_engine *e, double *fx, double *fy, double *fz,
                                      int device_ptrs, double out[7]) {
  if (!e || !out || (fx && (!fy || !fz))) return MDBAS_NB_ERR_ARG;
  if (!e->posSet) return MDBAS_NB_ERR_STATE;
  MDB_CUDA(cudaSetDevice(e->device));
  LaunchScope ls(e);
  cudaStream_t s = e->stream;
  for (int k = 0; k < 7; ++k) out[k] = 0.;
  if (e->bonded.nTerms() == 0) return MDBAS_NB_OK;
  const int n = e->n;
  const size_t bytes = sizeof(double) * (size_t)n;
  double *f = e->bondedF.as<double>();
  const cudaMemcpyKind in = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind back = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (fx) {
    // start from the caller's forces so the additions follow MDBas's order
    MDB_CUDA(cudaMemcpyAsync(f, fx, bytes, in, s));
    MDB_CUDA(cudaMemcpyAsync(f + n, fy, bytes, in, s));
    MDB_CUDA(cudaMemcpyAsync(f + 2 * (size_t)n, fz, bytes, in, s));
  } else {
    MDB_CUDA(cudaMemsetAsync(f, 0, 3 * bytes, s));
  }
  MDB_TRY(bonded_eval(e->bonded, e->boxesDev.as<DevBox>(), e->atomRepPtr(), e->x.as<double>(),
                      e->y.as<double>(), e->z.as<double>(), f, s));
  double sums[BS_COUNT];
  MDB_CUDA(cudaMemcpyAsync(sums, e->bonded.sums.p, sizeof(sums), cudaMemcpyDeviceToHost, s));
  if (fx) {
    MDB_CUDA(cudaMemcpyAsync(fx, f, bytes, back, s));
    MDB_CUDA(cudaMemcpyAsync(fy, f + n, bytes, back, s));
    MDB_CUDA(cudaMemcpyAsync(fz, f + 2 * (size_t)n, bytes, back, s));
  }
  MDB_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < 7; ++k) out[k] = sums[k];
  return MDBAS_NB_OK;
}
