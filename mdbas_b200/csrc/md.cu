// md.cu -- device-resident velocity-Verlet dynamics (mdbas_nb_engine_md_*).
//
// One step restates MDBas's VV-NVE step (vv_nve, src/integrate.c:1518-1634,
// driven as in src/mdbas.c:244-300):
//   stage 1: v += dt/2 f/m, x += dt v, then SHAKE on positions (vv_shake_r,
//            src/shake.c:209-326) with the constraint vectors taken before
//            the drift (image_array, src/integrate.c:1542-1553);
//   list:    rebuilt every `listUpdate` steps (MDBas's fixed `list N` cadence,
//            src/list.c:87-105) or, with listUpdate = 0, when some atom moved
//            more than half the skin since the last build (the displacement
//            criterion is new behaviour);
//   forces:  the engine's nonbonded evaluation (either precision form);
//   stage 2: v += dt/2 f/m, SHAKE on velocities (vv_shake_v,
//            src/shake.c:328-456), kinetic energy (kinetic, src/utils.c:502),
//            positions wrapped into the box (image_update).
// Everything stays on the GPU; the host only reads one word per step (the
// displacement test) and the energies when asked.
//
// Constraints are solved molecule by molecule (connected components of the
// constraint graph, one thread each) with MDBas's iteration: every constraint
// of the molecule contributes a correction, atoms take the average over the
// constraints they belong to (nAtConst), until the largest relative bond
// error is below tolShake.  MDBas iterates all molecules together until the
// worst one converges; here each molecule stops when it has converged, which
// changes the positions only within tolShake.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "engine.cuh"
#include "list_ref.cuh"
#include "pair_fp32.cuh"

using namespace mdbas;

namespace mdbas {
namespace {

// Molecule size classes of the SHAKE kernels: (atoms, constraints).
constexpr int kMolTinyAtoms = 3, kMolTinyCons = 3;      // rigid water, X-H bonds
constexpr int kMolSmallAtoms = 4, kMolSmallCons = 6;    // CH3, NH3+ ...
constexpr int kMolMaxAtoms = 16, kMolMaxCons = 32;      // the largest accepted

// stage 1 of vv_nve: half kick then drift (src/integrate.c:1555-1580)
// (atoms with skip[i] != 0 are integrated by the fused rigid-triangle kernels)
__global__ void k_vv_stage1(int n, double dt, const double *__restrict__ fx,
                            const double *__restrict__ fy, const double *__restrict__ fz,
                            const double *__restrict__ rmass, double *__restrict__ vx,
                            double *__restrict__ vy, double *__restrict__ vz,
                            double *__restrict__ x, double *__restrict__ y,
                            double *__restrict__ z, const int *__restrict__ skip) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || (skip && skip[i])) return;
  vx[i] += 0.5 * dt * fx[i] * rmass[i];
  vy[i] += 0.5 * dt * fy[i] * rmass[i];
  vz[i] += 0.5 * dt * fz[i] * rmass[i];
  x[i] += dt * vx[i];
  y[i] += dt * vy[i];
  z[i] += dt * vz[i];
}

__global__ void k_vv_kick(int n, double dt, const double *__restrict__ fx,
                          const double *__restrict__ fy, const double *__restrict__ fz,
                          const double *__restrict__ rmass, double *__restrict__ vx,
                          double *__restrict__ vy, double *__restrict__ vz,
                          const int *__restrict__ skip) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || (skip && skip[i])) return;
  vx[i] += 0.5 * dt * fx[i] * rmass[i];
  vy[i] += 0.5 * dt * fy[i] * rmass[i];
  vz[i] += 0.5 * dt * fz[i] * rmass[i];
}

// constraint vectors before the drift, minimum image (dist2, src/utils.c:82)
__global__ void k_cons_vectors(int nc, const DevBox *__restrict__ boxes,
                               const int *__restrict__ atomRep, const int *__restrict__ ca,
                               const int *__restrict__ cb, const double *__restrict__ x,
                               const double *__restrict__ y, const double *__restrict__ z,
                               double *__restrict__ ddx, double *__restrict__ ddy,
                               double *__restrict__ ddz) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const DevBox &b = boxes[atomRep ? atomRep[ca[c]] : 0];
  double dx = x[cb[c]] - x[ca[c]], dy = y[cb[c]] - y[ca[c]], dz = z[cb[c]] - z[ca[c]];
  dist_d(b, dx, dy, dz);
  ddx[c] = dx;
  ddy[c] = dy;
  ddz[c] = dz;
}

// --- per-molecule SHAKE / RATTLE ----------------------------------------------
// One thread per molecule holds the molecule's atoms (at most MA) and
// constraints (at most MC) in registers for the whole iteration: local atom
// numbers are resolved once, and every access by a run-time local number is
// a compile-time select over MA registers, so nothing goes to local memory.

// (The large class indexes its arrays directly, from local memory.)
template <int MA>
__device__ __forceinline__ double pick(const double (&v)[MA], int i) {
  if constexpr (MA > kMolSmallAtoms) {
    return v[i];
  } else {
    double r = 0.;
#pragma unroll
    for (int t = 0; t < MA; ++t)
      if (t == i) r = v[t];
    return r;
  }
}

template <int MA>
__device__ __forceinline__ void add_to(double (&v)[MA], int i, double d) {
  if constexpr (MA > kMolSmallAtoms) {
    v[i] += d;
  } else {
#pragma unroll
    for (int t = 0; t < MA; ++t)
      if (t == i) v[t] += d;
  }
}

// Local numbering of the molecule's atoms in order of first appearance;
// false when it has more than MA atoms.
template <int MA, int MC>
__device__ __forceinline__ bool mol_table(int c0, int ncons, const int *__restrict__ ca,
                                          const int *__restrict__ cb, int (&atoms)[MA], int &na,
                                          int (&la)[MC], int (&lb)[MC]) {
  na = 0;
#pragma unroll
  for (int t = 0; t < MA; ++t) atoms[t] = -1;
#pragma unroll
  for (int k = 0; k < MC; ++k) {
    la[k] = 0;
    lb[k] = 0;
    if (k < ncons) {
      const int a = ca[c0 + k], b = cb[c0 + k];
      int ia = -1, ib = -1;
#pragma unroll
      for (int t = 0; t < MA; ++t) {
        if (atoms[t] == a) ia = t;
        if (atoms[t] == b) ib = t;
      }
      if (ia < 0) {
        if (na >= MA) return false;
        ia = na;
#pragma unroll
        for (int t = 0; t < MA; ++t)
          if (t == na) atoms[t] = a;
        ++na;
      }
      if (ib < 0) {
        if (na >= MA) return false;
        ib = na;
#pragma unroll
        for (int t = 0; t < MA; ++t)
          if (t == na) atoms[t] = b;
        ++na;
      }
      la[k] = ia;
      lb[k] = ib;
    }
  }
  return true;
}

// Largest iteration count over the warp, one atomic per warp.
__device__ __forceinline__ void report_cycles(int *status, int icycle) {
  const int m = __reduce_max_sync(0xffffffffu, icycle);
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(status + 1, m);
}

// SHAKE on positions (vv_shake_r, src/shake.c:209-326): Jacobi corrections
// of all constraints, averaged over each atom's constraint count, until the
// largest relative bond error is below tol; positions and velocities move.
template <int MA, int MC>
__global__ void __launch_bounds__(128)
k_shake_positions(int nMol, const DevBox *__restrict__ boxes, const int *__restrict__ atomRep,
                  double dt, double tol, int maxCycle,
                  const int *__restrict__ molCons, const int *__restrict__ ca,
                  const int *__restrict__ cb, const double *__restrict__ rc2g,
                  const double *__restrict__ ddxg, const double *__restrict__ ddyg,
                  const double *__restrict__ ddzg, const double *__restrict__ rmass,
                  const int *__restrict__ nAtConst, double *__restrict__ x,
                  double *__restrict__ y, double *__restrict__ z, double *__restrict__ vx,
                  double *__restrict__ vy, double *__restrict__ vz, int *__restrict__ status) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  int c0 = 0, ncons = 0;
  if (m < nMol) {
    c0 = molCons[m];
    ncons = molCons[m + 1] - c0;
  }
  int icycle = 0;
  int atoms[MA], la[MC], lb[MC], na = 0;
  bool active = ncons > 0;
  if (active && (ncons > MC || !mol_table<MA, MC>(c0, ncons, ca, cb, atoms, na, la, lb))) {
    atomicOr(status, 2);
    active = false;
  }
  if (active) {
    const DevBox &b = boxes[atomRep ? atomRep[atoms[0]] : 0];
    double px[MA], py[MA], pz[MA], qx[MA], qy[MA], qz[MA], rm[MA], inv[MA];
#pragma unroll
    for (int t = 0; t < MA; ++t) {
      px[t] = py[t] = pz[t] = qx[t] = qy[t] = qz[t] = rm[t] = inv[t] = 0.;
      if (t < na) {
        const int a = atoms[t];
        px[t] = x[a];
        py[t] = y[a];
        pz[t] = z[a];
        qx[t] = vx[a];
        qy[t] = vy[a];
        qz[t] = vz[a];
        rm[t] = rmass[a];
        inv[t] = 1.0 / (double)nAtConst[a];
      }
    }
    double dcx[MC], dcy[MC], dcz[MC], r2c[MC], irc[MC];
#pragma unroll
    for (int k = 0; k < MC; ++k) {
      dcx[k] = dcy[k] = dcz[k] = 0.;
      r2c[k] = irc[k] = 1.;
      if (k < ncons) {
        dcx[k] = ddxg[c0 + k];
        dcy[k] = ddyg[c0 + k];
        dcz[k] = ddzg[c0 + k];
        r2c[k] = rc2g[c0 + k];
        irc[k] = 1.0 / sqrt(r2c[k]);
      }
    }
    bool converged = false;
    do {
      // current bond vectors (minimum image) and the largest relative error
      double tx[MC], ty[MC], tz[MC], rt2[MC];
      double maxdist = 0.;
#pragma unroll
      for (int k = 0; k < MC; ++k) {
        tx[k] = ty[k] = tz[k] = rt2[k] = 0.;
        if (k < ncons) {
          tx[k] = pick(px, lb[k]) - pick(px, la[k]);
          ty[k] = pick(py, lb[k]) - pick(py, la[k]);
          tz[k] = pick(pz, lb[k]) - pick(pz, la[k]);
          rt2[k] = dist_d(b, tx[k], ty[k], tz[k]);
          maxdist = fmax(maxdist, fabs(rt2[k] - r2c[k]) * irc[k]);
        }
      }
      maxdist = 0.5 * maxdist;
      if (maxdist < tol) converged = true;
      if (!converged) {
        double xt[MA], yt[MA], zt[MA];
#pragma unroll
        for (int t = 0; t < MA; ++t) xt[t] = yt[t] = zt[t] = 0.;
#pragma unroll
        for (int k = 0; k < MC; ++k) {
          if (k < ncons) {
            const double dx = tx[k], dy = ty[k], dz = tz[k];
            const double trmi = dt * pick(rm, la[k]);
            const double trmj = dt * pick(rm, lb[k]);
            const double lambda = -(r2c[k] - rt2[k]) /
                                  (dt * (trmi + trmj) *
                                   ((dcx[k] * dx) + (dcy[k] * dy) + (dcz[k] * dz)));
            const double lambdai = 0.5 * lambda * trmi;
            add_to(xt, la[k], dcx[k] * lambdai);
            add_to(yt, la[k], dcy[k] * lambdai);
            add_to(zt, la[k], dcz[k] * lambdai);
            const double lambdaj = -0.5 * lambda * trmj;
            add_to(xt, lb[k], dcx[k] * lambdaj);
            add_to(yt, lb[k], dcy[k] * lambdaj);
            add_to(zt, lb[k], dcz[k] * lambdaj);
          }
        }
        // applied per constraint, each atom's share scaled by 1/nAtConst
#pragma unroll
        for (int k = 0; k < MC; ++k) {
          if (k < ncons) {
            const double nia = pick(inv, la[k]), nib = pick(inv, lb[k]);
            const double xa = pick(xt, la[k]), ya = pick(yt, la[k]), za = pick(zt, la[k]);
            const double xb = pick(xt, lb[k]), yb = pick(yt, lb[k]), zb = pick(zt, lb[k]);
            add_to(px, la[k], dt * xa * nia);
            add_to(py, la[k], dt * ya * nia);
            add_to(pz, la[k], dt * za * nia);
            add_to(px, lb[k], dt * xb * nib);
            add_to(py, lb[k], dt * yb * nib);
            add_to(pz, lb[k], dt * zb * nib);
            add_to(qx, la[k], xa * nia);
            add_to(qy, la[k], ya * nia);
            add_to(qz, la[k], za * nia);
            add_to(qx, lb[k], xb * nib);
            add_to(qy, lb[k], yb * nib);
            add_to(qz, lb[k], zb * nib);
          }
        }
      }
      ++icycle;
    } while (!converged && icycle < maxCycle);
    if (!converged) atomicOr(status, 1);  // CONVERG_SHAKE_ERROR
#pragma unroll
    for (int t = 0; t < MA; ++t) {
      if (t < na) {
        const int a = atoms[t];
        x[a] = px[t];
        y[a] = py[t];
        z[a] = pz[t];
        vx[a] = qx[t];
        vy[a] = qy[t];
        vz[a] = qz[t];
      }
    }
  }
  report_cycles(status, icycle);
}

// SHAKE on velocities (vv_shake_v, src/shake.c:328-456).
template <int MA, int MC>
__global__ void __launch_bounds__(128)
k_shake_velocities(int nMol, double dt, double tolvel, int maxCycle,
                   const int *__restrict__ molCons, const int *__restrict__ ca,
                   const int *__restrict__ cb, const double *__restrict__ ddxg,
                   const double *__restrict__ ddyg, const double *__restrict__ ddzg,
                   const double *__restrict__ rmass, const int *__restrict__ nAtConst,
                   double *__restrict__ vx, double *__restrict__ vy, double *__restrict__ vz,
                   int *__restrict__ status) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  int c0 = 0, ncons = 0;
  if (m < nMol) {
    c0 = molCons[m];
    ncons = molCons[m + 1] - c0;
  }
  int atoms[MA], la[MC], lb[MC], na = 0;
  const bool active =
      ncons > 0 && ncons <= MC && mol_table<MA, MC>(c0, ncons, ca, cb, atoms, na, la, lb);
  if (!active) return;
  double qx[MA], qy[MA], qz[MA], rm[MA], inv[MA];
#pragma unroll
  for (int t = 0; t < MA; ++t) {
    qx[t] = qy[t] = qz[t] = rm[t] = inv[t] = 0.;
    if (t < na) {
      const int a = atoms[t];
      qx[t] = vx[a];
      qy[t] = vy[a];
      qz[t] = vz[a];
      rm[t] = rmass[a];
      inv[t] = 1.0 / (double)nAtConst[a];
    }
  }
  double dcx[MC], dcy[MC], dcz[MC];
#pragma unroll
  for (int k = 0; k < MC; ++k) {
    dcx[k] = dcy[k] = dcz[k] = 0.;
    if (k < ncons) {
      dcx[k] = ddxg[c0 + k];
      dcy[k] = ddyg[c0 + k];
      dcz[k] = ddzg[c0 + k];
    }
  }
  bool converged = false;
  int icycle = 0;
  do {
    double xt[MA], yt[MA], zt[MA];
#pragma unroll
    for (int t = 0; t < MA; ++t) xt[t] = yt[t] = zt[t] = 0.;
    double maxdist = 0.;
#pragma unroll
    for (int k = 0; k < MC; ++k) {
      if (k < ncons) {
        const double trmi = 0.5 * dt * pick(rm, la[k]);
        const double trmj = 0.5 * dt * pick(rm, lb[k]);
        const double lambda =
            (dcx[k] * (pick(qx, lb[k]) - pick(qx, la[k])) +
             dcy[k] * (pick(qy, lb[k]) - pick(qy, la[k])) +
             dcz[k] * (pick(qz, lb[k]) - pick(qz, la[k]))) /
            ((trmi + trmj) * (dcx[k] * dcx[k] + dcy[k] * dcy[k] + dcz[k] * dcz[k]));
        maxdist = fmax(maxdist, fabs(lambda));
        const double lambdai = lambda * trmi;
        add_to(xt, la[k], dcx[k] * lambdai);
        add_to(yt, la[k], dcy[k] * lambdai);
        add_to(zt, la[k], dcz[k] * lambdai);
        const double lambdaj = -lambda * trmj;
        add_to(xt, lb[k], dcx[k] * lambdaj);
        add_to(yt, lb[k], dcy[k] * lambdaj);
        add_to(zt, lb[k], dcz[k] * lambdaj);
      }
    }
    if (maxdist < tolvel) converged = true;
    if (!converged) {
#pragma unroll
      for (int k = 0; k < MC; ++k) {
        if (k < ncons) {
          const double nia = pick(inv, la[k]), nib = pick(inv, lb[k]);
          add_to(qx, la[k], pick(xt, la[k]) * nia);
          add_to(qy, la[k], pick(yt, la[k]) * nia);
          add_to(qz, la[k], pick(zt, la[k]) * nia);
          add_to(qx, lb[k], pick(xt, lb[k]) * nib);
          add_to(qy, lb[k], pick(yt, lb[k]) * nib);
          add_to(qz, lb[k], pick(zt, lb[k]) * nib);
        }
      }
    }
    ++icycle;
  } while (!converged && icycle < maxCycle);
  if (!converged) atomicOr(status, 1);
#pragma unroll
  for (int t = 0; t < MA; ++t) {
    if (t < na) {
      const int a = atoms[t];
      vx[a] = qx[t];
      vy[a] = qy[t];
      vz[a] = qz[t];
    }
  }
}

// --- rigid triangles (3 atoms, 3 constraints: rigid water) ---------------------
// All of a molecule's stage-1 (or stage-2) work in one thread with the local
// numbering fixed at compile time: constraint 0 = (a0, a1), 1 = (a0, a2),
// 2 = (a1, a2); every atom belongs to two constraints (nAtConst = 2).  The
// iteration is vv_shake_r / vv_shake_v's.
__device__ __forceinline__ void tri_vectors(const DevBox &b, const double (&px)[3],
                                            const double (&py)[3], const double (&pz)[3],
                                            double (&dx)[3], double (&dy)[3], double (&dz)[3],
                                            double (&r2)[3]) {
  constexpr int LA[3] = {0, 0, 1}, LB[3] = {1, 2, 2};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dx[k] = px[LB[k]] - px[LA[k]];
    dy[k] = py[LB[k]] - py[LA[k]];
    dz[k] = pz[LB[k]] - pz[LA[k]];
    r2[k] = dist_d(b, dx[k], dy[k], dz[k]);
  }
}

// Orthorhombic (and cubic) boxes: the minimum-image term dist() subtracts
// from each component of a constraint vector, a box edge times -1, 0 or 1
// (exact), fixed for the SHAKE iterations of one step (the corrections move
// atoms by far less than half an edge); the iterations then form the vectors
// without the conversions of the image test, with the same bits.
__device__ __forceinline__ void tri_image_terms(const DevBox &b, const double (&px)[3],
                                                const double (&py)[3], const double (&pz)[3],
                                                double (&cx)[3], double (&cy)[3],
                                                double (&cz)[3]) {
  constexpr int LA[3] = {0, 0, 1}, LB[3] = {1, 2, 2};
  const double ex = b.a1, ey = b.type == CUBIC ? b.a1 : b.b2, ez = b.type == CUBIC ? b.a1 : b.c3;
  const double ux = b.u1, uy = b.type == CUBIC ? b.u1 : b.v2, uz = b.type == CUBIC ? b.u1 : b.w3;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    cx[k] = dmul(ex, (double)nint_d(dmul(px[LB[k]] - px[LA[k]], ux)));
    cy[k] = dmul(ey, (double)nint_d(dmul(py[LB[k]] - py[LA[k]], uy)));
    cz[k] = dmul(ez, (double)nint_d(dmul(pz[LB[k]] - pz[LA[k]], uz)));
  }
}

__global__ void __launch_bounds__(128)
k_tri_stage1(int nTri, const DevBox *__restrict__ boxes, const int *__restrict__ atomRep,
             double dt, double tol, int maxCycle,
             const int4 *__restrict__ tri, const double4 *__restrict__ len2,
             const double *__restrict__ fx, const double *__restrict__ fy,
             const double *__restrict__ fz, const double *__restrict__ rmass,
             double *__restrict__ x, double *__restrict__ y, double *__restrict__ z,
             double *__restrict__ vx, double *__restrict__ vy, double *__restrict__ vz,
             int *__restrict__ status) {
  constexpr int LA[3] = {0, 0, 1}, LB[3] = {1, 2, 2};
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  int icycle = 0;
  if (m < nTri) {
    const int4 t = tri[m];
    const int A[3] = {t.x, t.y, t.z};
    const DevBox &b = boxes[atomRep ? atomRep[t.x] : 0];
    const double4 l2 = len2[m];
    const double r2c[3] = {l2.x, l2.y, l2.z};
    double irc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) irc[k] = 1.0 / sqrt(r2c[k]);
    double px[3], py[3], pz[3], qx[3], qy[3], qz[3], rm[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      px[i] = x[A[i]];
      py[i] = y[A[i]];
      pz[i] = z[A[i]];
      qx[i] = vx[A[i]];
      qy[i] = vy[A[i]];
      qz[i] = vz[A[i]];
      rm[i] = rmass[A[i]];
    }
    // constraint vectors before the drift
    double dcx[3], dcy[3], dcz[3], unused[3];
    tri_vectors(b, px, py, pz, dcx, dcy, dcz, unused);
    // half kick and drift
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      qx[i] += 0.5 * dt * fx[A[i]] * rm[i];
      qy[i] += 0.5 * dt * fy[A[i]] * rm[i];
      qz[i] += 0.5 * dt * fz[A[i]] * rm[i];
      px[i] += dt * qx[i];
      py[i] += dt * qy[i];
      pz[i] += dt * qz[i];
    }
    const bool ortho = b.type == CUBIC || b.type == ORBIC;
    double cx[3] = {0., 0., 0.}, cy[3] = {0., 0., 0.}, cz[3] = {0., 0., 0.};
    if (ortho) tri_image_terms(b, px, py, pz, cx, cy, cz);
    bool converged = false;
    do {
      double tx[3], ty[3], tz[3], rt2[3];
      if (ortho) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          tx[k] = dsub(px[LB[k]] - px[LA[k]], cx[k]);
          ty[k] = dsub(py[LB[k]] - py[LA[k]], cy[k]);
          tz[k] = dsub(pz[LB[k]] - pz[LA[k]], cz[k]);
          rt2[k] = dadd(dadd(dmul(tx[k], tx[k]), dmul(ty[k], ty[k])), dmul(tz[k], tz[k]));
        }
      } else {
        tri_vectors(b, px, py, pz, tx, ty, tz, rt2);
      }
      double maxdist = 0.;
#pragma unroll
      for (int k = 0; k < 3; ++k) maxdist = fmax(maxdist, fabs(rt2[k] - r2c[k]) * irc[k]);
      maxdist = 0.5 * maxdist;
      if (maxdist < tol) converged = true;
      if (!converged) {
        double xt[3] = {0., 0., 0.}, yt[3] = {0., 0., 0.}, zt[3] = {0., 0., 0.};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int ia = LA[k], ib = LB[k];
          const double trmi = dt * rm[ia], trmj = dt * rm[ib];
          const double lambda = -(r2c[k] - rt2[k]) /
                                (dt * (trmi + trmj) *
                                 ((dcx[k] * tx[k]) + (dcy[k] * ty[k]) + (dcz[k] * tz[k])));
          const double lambdai = 0.5 * lambda * trmi;
          xt[ia] += dcx[k] * lambdai;
          yt[ia] += dcy[k] * lambdai;
          zt[ia] += dcz[k] * lambdai;
          const double lambdaj = -0.5 * lambda * trmj;
          xt[ib] += dcx[k] * lambdaj;
          yt[ib] += dcy[k] * lambdaj;
          zt[ib] += dcz[k] * lambdaj;
        }
        // each atom takes half its correction from each of its two constraints
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int ia = LA[k], ib = LB[k];
          px[ia] += dt * xt[ia] * 0.5;
          py[ia] += dt * yt[ia] * 0.5;
          pz[ia] += dt * zt[ia] * 0.5;
          px[ib] += dt * xt[ib] * 0.5;
          py[ib] += dt * yt[ib] * 0.5;
          pz[ib] += dt * zt[ib] * 0.5;
          qx[ia] += xt[ia] * 0.5;
          qy[ia] += yt[ia] * 0.5;
          qz[ia] += zt[ia] * 0.5;
          qx[ib] += xt[ib] * 0.5;
          qy[ib] += yt[ib] * 0.5;
          qz[ib] += zt[ib] * 0.5;
        }
      }
      ++icycle;
    } while (!converged && icycle < maxCycle);
    if (!converged) atomicOr(status, 1);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      x[A[i]] = px[i];
      y[A[i]] = py[i];
      z[A[i]] = pz[i];
      vx[A[i]] = qx[i];
      vy[A[i]] = qy[i];
      vz[A[i]] = qz[i];
    }
  }
  report_cycles(status, icycle);
}

__global__ void __launch_bounds__(128)
k_tri_stage2(int nTri, const DevBox *__restrict__ boxes, const int *__restrict__ atomRep,
             double dt, double tolvel, int maxCycle,
             const int4 *__restrict__ tri, const double *__restrict__ fx,
             const double *__restrict__ fy, const double *__restrict__ fz,
             const double *__restrict__ rmass, const double *__restrict__ x,
             const double *__restrict__ y, const double *__restrict__ z,
             double *__restrict__ vx, double *__restrict__ vy, double *__restrict__ vz,
             int *__restrict__ status) {
  constexpr int LA[3] = {0, 0, 1}, LB[3] = {1, 2, 2};
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nTri) return;
  const int4 t = tri[m];
  const int A[3] = {t.x, t.y, t.z};
  const DevBox &b = boxes[atomRep ? atomRep[t.x] : 0];
  double px[3], py[3], pz[3], qx[3], qy[3], qz[3], rm[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    px[i] = x[A[i]];
    py[i] = y[A[i]];
    pz[i] = z[A[i]];
    rm[i] = rmass[A[i]];
    qx[i] = vx[A[i]] + 0.5 * dt * fx[A[i]] * rm[i];
    qy[i] = vy[A[i]] + 0.5 * dt * fy[A[i]] * rm[i];
    qz[i] = vz[A[i]] + 0.5 * dt * fz[A[i]] * rm[i];
  }
  // constraint vectors at the new positions; the denominators are fixed
  double dcx[3], dcy[3], dcz[3], dd2[3], trm[3][2], iden[3];
  tri_vectors(b, px, py, pz, dcx, dcy, dcz, dd2);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    trm[k][0] = 0.5 * dt * rm[LA[k]];
    trm[k][1] = 0.5 * dt * rm[LB[k]];
    iden[k] = 1.0 / ((trm[k][0] + trm[k][1]) * dd2[k]);
  }
  bool converged = false;
  int icycle = 0;
  do {
    double xt[3] = {0., 0., 0.}, yt[3] = {0., 0., 0.}, zt[3] = {0., 0., 0.};
    double maxdist = 0.;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int ia = LA[k], ib = LB[k];
      const double lambda = (dcx[k] * (qx[ib] - qx[ia]) + dcy[k] * (qy[ib] - qy[ia]) +
                             dcz[k] * (qz[ib] - qz[ia])) * iden[k];
      maxdist = fmax(maxdist, fabs(lambda));
      const double lambdai = lambda * trm[k][0];
      xt[ia] += dcx[k] * lambdai;
      yt[ia] += dcy[k] * lambdai;
      zt[ia] += dcz[k] * lambdai;
      const double lambdaj = -lambda * trm[k][1];
      xt[ib] += dcx[k] * lambdaj;
      yt[ib] += dcy[k] * lambdaj;
      zt[ib] += dcz[k] * lambdaj;
    }
    if (maxdist < tolvel) converged = true;
    if (!converged) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int ia = LA[k], ib = LB[k];
        qx[ia] += xt[ia] * 0.5;
        qy[ia] += yt[ia] * 0.5;
        qz[ia] += zt[ia] * 0.5;
        qx[ib] += xt[ib] * 0.5;
        qy[ib] += yt[ib] * 0.5;
        qz[ib] += zt[ib] * 0.5;
      }
    }
    ++icycle;
  } while (!converged && icycle < maxCycle);
  if (!converged) atomicOr(status, 1);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    vx[A[i]] = qx[i];
    vy[A[i]] = qy[i];
    vz[A[i]] = qz[i];
  }
}

// positions back into their box (image_update, src/utils.c:162-218)
__global__ void k_wrap(int n, const DevBox *__restrict__ boxes, const int *__restrict__ atomRep,
                       double *__restrict__ x, double *__restrict__ y, double *__restrict__ z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xi = x[i], yi = y[i], zi = z[i];
  image_d(boxes[atomRep ? atomRep[i] : 0], xi, yi, zi);
  x[i] = xi;
  y[i] = yi;
  z[i] = zi;
}

// kinetic energy (src/utils.c:502-515), sum in fixed point (2^-24 units).
// A term at or above termLimit (2^62 / n in fixed-point units, so that no
// sum of n terms can wrap) or not finite raises FLAG_OVERFLOW in *flags.
__global__ void k_kinetic(int n, const double *__restrict__ mass, const double *__restrict__ vx,
                          const double *__restrict__ vy, const double *__restrict__ vz,
                          double termLimit, long long *__restrict__ acc,
                          long long *__restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  long long v = 0;
  if (i < n) {
    const double t = 0.5 * mass[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
    if (!(t * kEnergyScale < termLimit)) {
      atomicOr(reinterpret_cast<unsigned long long *>(flags), (unsigned long long)FLAG_OVERFLOW);
    } else {
      v = fix_e(t);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red_add(acc, v);
}

// largest squared displacement since the last build (minimum image) and,
// when xp is given, since the last prune; each as the bit pattern of a
// non-negative double (which orders like the double)
__global__ void k_max_disp(int n, const DevBox *__restrict__ boxes,
                           const int *__restrict__ atomRep, const double *__restrict__ x,
                           const double *__restrict__ y, const double *__restrict__ z,
                           const double *__restrict__ xb, const double *__restrict__ yb,
                           const double *__restrict__ zb, const double *__restrict__ xp,
                           const double *__restrict__ yp, const double *__restrict__ zp,
                           unsigned long long *__restrict__ outB,
                           unsigned long long *__restrict__ outP) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r2 = 0., p2 = 0.;
  if (i < n) {
    const DevBox &b = boxes[atomRep ? atomRep[i] : 0];
    double dx = x[i] - xb[i], dy = y[i] - yb[i], dz = z[i] - zb[i];
    r2 = dist_d(b, dx, dy, dz);
    if (!(r2 == r2)) r2 = 1e300;  // NaN forces a rebuild (which reports it)
    if (xp) {
      double ex = x[i] - xp[i], ey = y[i] - yp[i], ez = z[i] - zp[i];
      p2 = dist_d(b, ex, ey, ez);
      if (!(p2 == p2)) p2 = 1e300;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
    p2 = fmax(p2, __shfl_xor_sync(0xffffffffu, p2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(outB, (unsigned long long)__double_as_longlong(r2));
    if (xp) atomicMax(outP, (unsigned long long)__double_as_longlong(p2));
  }
}

// frozen atoms keep zero force and velocity (freeze_atoms, src/utils.c:131-150)
__global__ void k_freeze(int n, const int *__restrict__ frozen, double *__restrict__ f,
                         double *__restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !frozen[i]) return;
  f[i] = f[n + i] = f[2 * (size_t)n + i] = 0.;
  v[i] = v[n + i] = v[2 * (size_t)n + i] = 0.;
}

// Berendsen scaling of vv_nvt_b (src/integrate.c:1722-1733): every thread
// derives lambda from the kinetic energy summed on the device.
__global__ void k_berendsen(int n, double dtOverTau, double kinTemp0,
                            const long long *__restrict__ kfix, double *__restrict__ vx,
                            double *__restrict__ vy, double *__restrict__ vz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double kin = (double)(*kfix) / kEnergyScale;
  if (!(kin > 0.)) return;
  const double lambda = sqrt(1.0 + dtOverTau * (kinTemp0 / kin - 1.0));
  vx[i] *= lambda;
  vy[i] *= lambda;
  vz[i] *= lambda;
}

// --- graph-only kernels: the rebuild decision and the per-step record -----
// Set the rebuild condition (hB) from the largest squared displacement since
// the build, or from MDBas's fixed cadence "list N" (step % N == 0) when
// update > 0, and the prune condition (hP: a rebuild, or the displacement
// since the last prune past halfIn2; never when prune = 0); advance the
// device step counter.
__global__ void k_decide(cudaGraphConditionalHandle hB, cudaGraphConditionalHandle hP,
                         const unsigned long long *__restrict__ bitsB,
                         const unsigned long long *__restrict__ bitsP, double half2,
                         double halfIn2, int update, int prune,
                         long long *__restrict__ stepDev) {
  if (threadIdx.x != 0) return;
  const long long st = stepDev[0] + 1;
  stepDev[0] = st;
  const bool rebuild = update > 0 ? (st % update) == 0
                                  : __longlong_as_double((long long)bitsB[0]) > half2;
  const bool pr = prune && (rebuild || __longlong_as_double((long long)bitsP[0]) > halfIn2);
  cudaGraphSetConditional(hB, rebuild ? 1u : 0u);
  if (prune) cudaGraphSetConditional(hP, pr ? 1u : 0u);
}

__global__ void k_count(long long *__restrict__ c) {
  if (threadIdx.x == 0) c[0] += 1;
}

// Fixed-point energies of the step (elec direct, elec corr, vdw, kinetic) and
// the accumulated error bits.
// row = {direct, correction, vdw, kinetic, bonded, reciprocal} in fixed
// point (2^-24)
__global__ void k_md_row(long long *__restrict__ row, const long long *__restrict__ acc,
                         const long long *__restrict__ kin, const long long *__restrict__ bonded,
                         const long long *__restrict__ kspace, long long *__restrict__ flags) {
  if (threadIdx.x != 0) return;
  row[0] = acc[ACC_E_DIR];
  row[1] = acc[ACC_E_CORR];
  row[2] = acc[ACC_E_VDW];
  row[3] = kin[0];
  row[4] = bonded ? bonded[0] : 0;
  row[5] = kspace ? kspace[0] : 0;
  flags[0] |= acc[ACC_FLAGS];
}

}  // namespace
}  // namespace mdbas

// every replica's box and the atom -> replica map, as the MD kernels take them
#define BOXES(e) (e)->boxesDev.as<DevBox>(), (e)->atomRepPtr()

#define MD_TRY(expr)                                                           \
  do {                                                                         \
    int s__ = (expr);                                                          \
    if (s__ != MDBAS_NB_OK) {                                                  \
      set_last_status(s__, nullptr);                                           \
      return s__;                                                              \
    }                                                                          \
  } while (0)

namespace {

// Slots of the engine's MD word buffer (int64 each).
enum MdWord {
  W_DISP = 0,     // largest squared displacement since the last build (bits)
  W_FLAGS = 1,    // OR of the fixed-point error bits of the recorded steps
  W_KIN = 2,      // kinetic energy, fixed point (2^-24)
  W_SHAKE = 4,    // two ints: SHAKE error bits, largest iteration count
  W_STEP = 6,     // device step counter (graph form)
  W_BUILDS = 7,   // list builds inside the graph since the last read
  W_DISP2 = 3,    // largest squared displacement since the last prune (bits)
  W_PRUNES = 8,   // prunes inside the graph since the last read
  W_COUNT = 10
};

constexpr int kRowWords = 6;  // k_md_row's row length

// Fixed-point bonded energy of the last md_forces (null without bonded terms).
const long long *md_bonded_fix(const mdbas_nb_engine *e) {
  return e->bonded.nTerms() > 0 ? e->bonded.sums.as<long long>() + BS_FIX : nullptr;
}

// Fixed-point reciprocal + non-neutral energy of the last md_forces (null
// without k-space).
const long long *md_kspace_fix(const mdbas_nb_engine *e) {
  return e->kspaceKind != 0 ? e->kspaceFix.as<long long>() : nullptr;
}

// FP64 forces of the last compute, caller order, into e->mdF (3n); then the
// bonded terms in MDBas's order (energy(), src/energy.c:167-190) and the
// frozen atoms (freeze_atoms, src/energy.c:198-201).
int md_forces(mdbas_nb_engine *e, cudaStream_t s) {
  const int n = e->n;
  double *f = e->mdF.as<double>();
  if (e->cfg.precision == 0) {
    MDB_CUDA(cudaMemcpyAsync(f, e->f64.p, sizeof(double) * 3 * (size_t)n,
                             cudaMemcpyDeviceToDevice, s));
  } else {
    MDB_TRY(forces_out_launch(e->cl, n, 0, f, f + n, f + 2 * (size_t)n, s));
  }
  MDB_TRY(md_kspace(e, f, s));
  if (e->bonded.nTerms() > 0)
    MDB_TRY(bonded_eval(e->bonded, BOXES(e), e->x.as<double>(), e->y.as<double>(),
                        e->z.as<double>(), f, s));
  if (e->hasFrozen)
    MDB_LAUNCH(k_freeze, grid_for(n, 256), 256, 0, s, n, e->frozen.as<int>(), f,
               e->mdV.as<double>());
  return MDBAS_NB_OK;
}

int md_save_build_positions(mdbas_nb_engine *e, cudaStream_t s) {
  const size_t bytes = sizeof(double) * (size_t)e->n;
  double *xb = e->mdXb.as<double>();
  MDB_CUDA(cudaMemcpyAsync(xb, e->x.p, bytes, cudaMemcpyDeviceToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(xb + e->n, e->y.p, bytes, cudaMemcpyDeviceToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(xb + 2 * (size_t)e->n, e->z.p, bytes, cudaMemcpyDeviceToDevice, s));
  return MDBAS_NB_OK;
}

// Synchronising list build (either precision) at the current positions.
int md_build(mdbas_nb_engine *e) {
  MD_TRY(mdbas_nb_engine_build(e));
  MD_TRY(engine_resolve_build(e));  // the step uses the list right away
  MD_TRY(md_save_build_positions(e, e->stream));
  e->mdRebuilds += 1;
  return MDBAS_NB_OK;
}

// stage 1 of vv_nve: constraint vectors, half kick + drift, SHAKE on positions
int md_stage1(mdbas_nb_engine *e, cudaStream_t s) {
  const int n = e->n, nc = e->mdNCons;
  double *x = e->x.as<double>(), *y = e->y.as<double>(), *z = e->z.as<double>();
  double *vx = e->mdV.as<double>(), *vy = vx + n, *vz = vy + n;
  const double *fx = e->mdF.as<double>(), *fy = fx + n, *fz = fy + n;
  double *ddx = e->mdDd.as<double>(), *ddy = ddx + nc, *ddz = ddy + nc;
  if (e->mdTri) {
    // rigid triangles: vectors, kick, drift and SHAKE fused per molecule;
    // the atom kernel integrates the unconstrained atoms only
    if (e->mdNTri < n)
      MDB_LAUNCH(k_vv_stage1, grid_for(n, 256), 256, 0, s, n, e->mdDt, fx, fy, fz,
                 e->mdRmass.as<double>(), vx, vy, vz, x, y, z, e->mdNAt.as<int>());
    MDB_LAUNCH(k_tri_stage1, grid_for(e->mdNMol, 128), 128, 0, s, e->mdNMol, BOXES(e), e->mdDt,
               e->mdTol, e->mdMaxCycle, e->mdTriAtoms.as<int4>(), e->mdTriLen2.as<double4>(),
               fx, fy, fz, e->mdRmass.as<double>(), x, y, z, vx, vy, vz,
               reinterpret_cast<int *>(e->mdWord.as<long long>() + W_SHAKE));
    return MDBAS_NB_OK;
  }
  if (nc > 0)
    MDB_LAUNCH(k_cons_vectors, grid_for(nc, 256), 256, 0, s, nc, BOXES(e), e->mdCa.as<int>(),
               e->mdCb.as<int>(), x, y, z, ddx, ddy, ddz);
  MDB_LAUNCH(k_vv_stage1, grid_for(n, 256), 256, 0, s, n, e->mdDt, fx, fy, fz,
             e->mdRmass.as<double>(), vx, vy, vz, x, y, z, nullptr);
  if (nc > 0) {
    auto shake = e->mdMolClass == 0   ? k_shake_positions<kMolTinyAtoms, kMolTinyCons>
                 : e->mdMolClass == 1 ? k_shake_positions<kMolSmallAtoms, kMolSmallCons>
                                      : k_shake_positions<kMolMaxAtoms, kMolMaxCons>;
    MDB_LAUNCH(shake, grid_for(e->mdNMol, 128), 128, 0, s, e->mdNMol, BOXES(e),
               e->mdDt, e->mdTol, e->mdMaxCycle, e->mdMol.as<int>(), e->mdCa.as<int>(),
               e->mdCb.as<int>(), e->mdRc2.as<double>(), ddx, ddy, ddz, e->mdRmass.as<double>(),
               e->mdNAt.as<int>(), x, y, z, vx, vy, vz,
               reinterpret_cast<int *>(e->mdWord.as<long long>() + W_SHAKE));
  }
  return MDBAS_NB_OK;
}

bool md_prune_on(const mdbas_nb_engine *e) {
  return e->cfg.precision == 1 && e->mdPruneBuf > 0.;
}

int md_max_disp(mdbas_nb_engine *e, cudaStream_t s) {
  const int n = e->n;
  long long *word = e->mdWord.as<long long>();
  const double *xb = e->mdXb.as<double>();
  const double *xp = md_prune_on(e) ? e->mdXp.as<double>() : nullptr;
  MDB_CUDA(cudaMemsetAsync(word + W_DISP, 0, sizeof(long long), s));
  MDB_CUDA(cudaMemsetAsync(word + W_DISP2, 0, sizeof(long long), s));
  MDB_LAUNCH(k_max_disp, grid_for(n, 256), 256, 0, s, n, BOXES(e), e->x.as<double>(),
             e->y.as<double>(), e->z.as<double>(), xb, xb + n, xb + 2 * (size_t)n, xp,
             xp ? xp + n : nullptr, xp ? xp + 2 * (size_t)n : nullptr,
             reinterpret_cast<unsigned long long *>(word + W_DISP),
             reinterpret_cast<unsigned long long *>(word + W_DISP2));
  return MDBAS_NB_OK;
}

// Inner radius of the pruned list: the cut-off plus the prune buffer, with the
// list radius's FP32 margin.
float md_rin2(const mdbas_nb_engine *e) {
  const double rin = e->cfg.cutOff + e->mdPruneBuf;
  return (float)(rin * rin * (1.0 + 1e-5));
}

// Prune the list at the current (refreshed) layout and save the positions.
int md_prune(mdbas_nb_engine *e, cudaStream_t s) {
  MDB_TRY(cluster_prune(e->cl, md_rin2(e), s));
  const size_t bytes = sizeof(double) * (size_t)e->n;
  double *xp = e->mdXp.as<double>();
  MDB_CUDA(cudaMemcpyAsync(xp, e->x.p, bytes, cudaMemcpyDeviceToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(xp + e->n, e->y.p, bytes, cudaMemcpyDeviceToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(xp + 2 * (size_t)e->n, e->z.p, bytes, cudaMemcpyDeviceToDevice, s));
  return MDBAS_NB_OK;
}

// Host-driven prune (outside graphs): also switches the pair kernel over.
int md_prune_sync(mdbas_nb_engine *e) {
  MD_TRY(md_prune(e, e->stream));
  e->cl.useInner = true;
  e->mdPrunes += 1;
  return MDBAS_NB_OK;
}

// Nonbonded forces of the cluster form with no host interaction, on the
// current layout (refreshed by the caller): evaluate, convert to caller order.
int md_forces_cluster(mdbas_nb_engine *e, cudaStream_t s) {
  ClusterWork &w = e->cl;
  const int n = e->n;
  MDB_CUDA(cudaMemsetAsync(w.facc.p, 0, sizeof(long long) * 3 * (size_t)w.slotCap, s));
  MDB_CUDA(cudaMemsetAsync(w.acc.p, 0, sizeof(long long) * ACC_COUNT, s));
  MDB_TRY(pair_fp32_launch(w, e->pp, e->grid, e->block, s, e->variant));
  MDB_TRY(excl_fix_launch(w, n, e->pp, e->exclStartSym.as<int>(), e->exclFlatSym.as<int>(),
                          e->x.as<double>(), e->y.as<double>(), e->z.as<double>(),
                          e->q.as<double>(), s));
  return md_forces(e, s);
}

int md_refresh_cluster(mdbas_nb_engine *e, cudaStream_t s) {
  return cluster_refresh(e->cl, e->x.as<double>(), e->y.as<double>(), e->z.as<double>(),
                         e->q.as<double>(), sqrt(e->cfg.chargeConst), s);
}

// stage 2: half kick, RATTLE on velocities, kinetic energy (+ Berendsen),
// positions wrapped into the box
int md_stage2(mdbas_nb_engine *e, cudaStream_t s, bool kin, double tauT, double kinTemp0) {
  const int n = e->n, nc = e->mdNCons;
  double *x = e->x.as<double>(), *y = e->y.as<double>(), *z = e->z.as<double>();
  double *vx = e->mdV.as<double>(), *vy = vx + n, *vz = vy + n;
  const double *fx = e->mdF.as<double>(), *fy = fx + n, *fz = fy + n;
  double *ddx = e->mdDd.as<double>(), *ddy = ddx + nc, *ddz = ddy + nc;
  long long *word = e->mdWord.as<long long>();
  const int g = grid_for(n, 256);
  if (e->mdTri) {
    if (e->mdNTri < n)
      MDB_LAUNCH(k_vv_kick, g, 256, 0, s, n, e->mdDt, fx, fy, fz, e->mdRmass.as<double>(), vx,
                 vy, vz, e->mdNAt.as<int>());
    MDB_LAUNCH(k_tri_stage2, grid_for(e->mdNMol, 128), 128, 0, s, e->mdNMol, BOXES(e), e->mdDt,
               e->mdTol / e->mdDt, e->mdMaxCycle, e->mdTriAtoms.as<int4>(), fx, fy, fz,
               e->mdRmass.as<double>(), x, y, z, vx, vy, vz,
               reinterpret_cast<int *>(word + W_SHAKE));
  } else {
    MDB_LAUNCH(k_vv_kick, g, 256, 0, s, n, e->mdDt, fx, fy, fz, e->mdRmass.as<double>(), vx, vy,
               vz, nullptr);
  }
  if (nc > 0 && !e->mdTri) {
    // stage 2 takes the constraint vectors at the new positions
    MDB_LAUNCH(k_cons_vectors, grid_for(nc, 256), 256, 0, s, nc, BOXES(e), e->mdCa.as<int>(),
               e->mdCb.as<int>(), x, y, z, ddx, ddy, ddz);
    auto rattle = e->mdMolClass == 0   ? k_shake_velocities<kMolTinyAtoms, kMolTinyCons>
                  : e->mdMolClass == 1 ? k_shake_velocities<kMolSmallAtoms, kMolSmallCons>
                                       : k_shake_velocities<kMolMaxAtoms, kMolMaxCons>;
    MDB_LAUNCH(rattle, grid_for(e->mdNMol, 128), 128, 0, s, e->mdNMol, e->mdDt,
               e->mdTol / e->mdDt, e->mdMaxCycle, e->mdMol.as<int>(), e->mdCa.as<int>(),
               e->mdCb.as<int>(), ddx, ddy, ddz, e->mdRmass.as<double>(), e->mdNAt.as<int>(), vx,
               vy, vz, reinterpret_cast<int *>(word + W_SHAKE));
  }
  const bool thermo = tauT > 0.;
  if (kin || thermo) {
    MDB_CUDA(cudaMemsetAsync(word + W_KIN, 0, sizeof(long long), s));
    MDB_LAUNCH(k_kinetic, g, 256, 0, s, n, e->mdMass.as<double>(), vx, vy, vz,
               4611686018427387904.0 / (double)(n > 0 ? n : 1), word + W_KIN, word + W_FLAGS);
  }
  if (thermo)
    MDB_LAUNCH(k_berendsen, g, 256, 0, s, n, e->mdDt / tauT, kinTemp0, word + W_KIN, vx, vy,
               vz);
  // positions back into the box (image_update, src/integrate.c:1626)
  MDB_LAUNCH(k_wrap, g, 256, 0, s, n, BOXES(e), x, y, z);
  return MDBAS_NB_OK;
}

double md_kin_row(double kin, double dt, double tauT, double kinTemp0) {
  if (tauT > 0. && kin > 0.) kin *= 1.0 + dt / tauT * (kinTemp0 / kin - 1.0);
  return kin;
}

int md_check_shake(mdbas_nb_engine *e, const int st[2]) {
  e->mdShakeIter = std::max<long long>(e->mdShakeIter, st[1]);
  if (st[0] & 1) {
    set_last_status(MDBAS_NB_ERR_UNSUPPORTED, "SHAKE did not converge (CONVERG_SHAKE_ERROR)");
    return MDBAS_NB_ERR_UNSUPPORTED;
  }
  if (st[0] & 2) {
    set_last_status(MDBAS_NB_ERR_UNSUPPORTED, "a constrained molecule exceeds 16 atoms or 32 constraints");
    return MDBAS_NB_ERR_UNSUPPORTED;
  }
  return MDBAS_NB_OK;
}

// --- the graph form ------------------------------------------------------------
struct CaptureCount {
  long long main = 0, body = 0, prune = 0;
};

void md_graph_free(mdbas_nb_engine *e) {
  if (e->mdExec) cudaGraphExecDestroy(e->mdExec);
  if (e->mdGraph) cudaGraphDestroy(e->mdGraph);
  e->mdExec = nullptr;
  e->mdGraph = nullptr;
  e->mdGraphK = 0;
  e->mdGraphStale = true;
}

// The rebuild body: synchronisation-free cluster build, build positions
// saved, build counter advanced.
int md_capture_rebuild_body(mdbas_nb_engine *e, cudaGraph_t body, long long *counter) {
  cudaStream_t side = e->mdSideStream;
  MDB_CUDA(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed));
  g_launch_counter = counter;
  const int *frozen = e->hasFrozen ? e->frozen.as<int>() : nullptr;
  int st = cluster_build(e->cl, e->n, e->nRep, e->repBoxes.data(), e->repOff.data(),
                         e->cfg.cutOff, e->cfg.delr, engine_list_rule(e),
                         sqrt(e->cfg.chargeConst), e->x.as<double>(), e->y.as<double>(),
                         e->z.as<double>(), e->q.as<double>(), e->eps.as<double>(),
                         e->sig.as<double>(), frozen, e->exclStartSym.as<int>(),
                         e->exclFlatSym.as<int>(), side, false);
  if (st == MDBAS_NB_OK) st = md_save_build_positions(e, side);
  if (st == MDBAS_NB_OK) {
    k_count<<<1, 32, 0, side>>>(e->mdWord.as<long long>() + W_BUILDS);
    ++(*counter);
    if (cudaGetLastError() != cudaSuccess) st = MDBAS_NB_ERR_CUDA;
  }
  cudaGraph_t out = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(side, &out);
  if (st != MDBAS_NB_OK) return st;
  MDB_CUDA(ce);
  return MDBAS_NB_OK;
}

// Add an IF node on the capture stream's current dependencies and return its
// body graph; the stream continues after the node.
int md_add_if(cudaStream_t cs, cudaGraphConditionalHandle h, cudaGraph_t *body,
              cudaGraphNode_t *node) {
  cudaStreamCaptureStatus cst;
  cudaGraph_t capG = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  MDB_CUDA(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &capG, &deps, &nd));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  MDB_CUDA(cudaGraphAddNode(node, capG, deps, nd, &cp));
  *body = cp.conditional.phGraph_out[0];
  return MDBAS_NB_OK;
}

// The prune body: prune at the refreshed layout, save the positions, count.
int md_capture_prune_body(mdbas_nb_engine *e, cudaGraph_t body, long long *counter) {
  cudaStream_t side = e->mdSideStream;
  MDB_CUDA(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed));
  g_launch_counter = counter;
  int st = md_prune(e, side);
  if (st == MDBAS_NB_OK) {
    k_count<<<1, 32, 0, side>>>(e->mdWord.as<long long>() + W_PRUNES);
    ++(*counter);
    if (cudaGetLastError() != cudaSuccess) st = MDBAS_NB_ERR_CUDA;
  }
  cudaGraph_t out = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(side, &out);
  if (st != MDBAS_NB_OK) return st;
  MDB_CUDA(ce);
  return MDBAS_NB_OK;
}

int md_capture_steps(mdbas_nb_engine *e, int K, double tauT, double kinTemp0,
                     CaptureCount &cc) {
  cudaStream_t cs = e->mdCapStream;
  long long *word = e->mdWord.as<long long>();
  const double half2 = 0.25 * e->cfg.delr * e->cfg.delr;
  const double halfIn2 = 0.25 * e->mdPruneBuf * e->mdPruneBuf;
  const bool prune = md_prune_on(e);
  for (int k = 0; k < K; ++k) {
    g_launch_counter = &cc.main;
    MDB_TRY(md_stage1(e, cs));
    // the rebuild and prune decisions, on the device
    cudaStreamCaptureStatus cst;
    cudaGraph_t capG = nullptr;
    MDB_CUDA(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &capG, nullptr, nullptr));
    // (a handle that no conditional node uses makes the graph invalid: the
    // prune handle exists only with pruning on, else k_decide leaves it alone)
    cudaGraphConditionalHandle hB, hP;
    MDB_CUDA(cudaGraphConditionalHandleCreate(&hB, capG, 0, cudaGraphCondAssignDefault));
    hP = hB;
    if (prune)
      MDB_CUDA(cudaGraphConditionalHandleCreate(&hP, capG, 0, cudaGraphCondAssignDefault));
    if (e->mdListUpdate == 0 || prune) MDB_TRY(md_max_disp(e, cs));
    MDB_LAUNCH(k_decide, 1, 32, 0, cs, hB, hP,
               reinterpret_cast<const unsigned long long *>(word + W_DISP),
               reinterpret_cast<const unsigned long long *>(word + W_DISP2), half2, halfIn2,
               e->mdListUpdate, prune ? 1 : 0, word + W_STEP);
    cudaGraph_t body;
    cudaGraphNode_t node;
    MDB_TRY(md_add_if(cs, hB, &body, &node));
    long long bodyCount = 0;
    MDB_TRY(md_capture_rebuild_body(e, body, &bodyCount));
    cc.body = bodyCount;
    MDB_CUDA(cudaStreamUpdateCaptureDependencies(cs, &node, 1,
                                                 cudaStreamSetCaptureDependencies));
    g_launch_counter = &cc.main;
    MDB_TRY(md_refresh_cluster(e, cs));
    if (prune) {
      MDB_TRY(md_add_if(cs, hP, &body, &node));
      long long pruneCount = 0;
      MDB_TRY(md_capture_prune_body(e, body, &pruneCount));
      cc.prune = pruneCount;
      MDB_CUDA(cudaStreamUpdateCaptureDependencies(cs, &node, 1,
                                                   cudaStreamSetCaptureDependencies));
      g_launch_counter = &cc.main;
    }
    MDB_TRY(md_forces_cluster(e, cs));
    MDB_TRY(md_stage2(e, cs, true, tauT, kinTemp0));
    MDB_LAUNCH(k_md_row, 1, 32, 0, cs, e->mdRows.as<long long>() + kRowWords * (size_t)k,
               e->cl.acc.as<long long>(), word + W_KIN, md_bonded_fix(e), md_kspace_fix(e),
               word + W_FLAGS);
  }
  return MDBAS_NB_OK;
}

int md_capture(mdbas_nb_engine *e, int K, double targetTemp, double tauT, double kinTemp0) {
  md_graph_free(e);
  if (!e->mdCapStream)
    MDB_CUDA(cudaStreamCreateWithFlags(&e->mdCapStream, cudaStreamNonBlocking));
  if (!e->mdSideStream)
    MDB_CUDA(cudaStreamCreateWithFlags(&e->mdSideStream, cudaStreamNonBlocking));
  MDB_TRY(e->mdRows.ensure(sizeof(long long) * kRowWords * (size_t)K));
  // everything the capture reads from the host must be final: finish the
  // engine stream's work first
  MDB_CUDA(cudaStreamSynchronize(e->stream));
  long long *const saved = g_launch_counter;
  CaptureCount cc;
  MDB_CUDA(cudaStreamBeginCapture(e->mdCapStream, cudaStreamCaptureModeThreadLocal));
  const int st = md_capture_steps(e, K, tauT, kinTemp0, cc);
  g_launch_counter = saved;
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(e->mdCapStream, &graph);
  if (st != MDBAS_NB_OK || ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (st != MDBAS_NB_OK) return st;
    return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  if (ie != cudaSuccess) {
    cudaGraphDestroy(graph);
    return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
  }
  e->mdGraph = graph;
  e->mdExec = exec;
  e->mdGraphK = K;
  e->mdGraphTau = tauT;
  e->mdGraphTemp = targetTemp;
  e->mdGraphStale = false;
  e->mdGraphMainK = cc.main / K;
  e->mdGraphBodyK = cc.body;
  e->mdGraphPruneK = cc.prune;
  return MDBAS_NB_OK;
}

int md_snapshot(mdbas_nb_engine *e, bool restore) {
  const size_t n = (size_t)e->n, b = sizeof(double) * n;
  double *snap = e->mdSnap.as<double>();
  double *parts[4] = {e->x.as<double>(), e->y.as<double>(), e->z.as<double>(), nullptr};
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  cudaStream_t s = e->stream;
  for (int i = 0; i < 3; ++i) {
    if (restore) MDB_CUDA(cudaMemcpyAsync(parts[i], snap + i * n, b, k, s));
    else MDB_CUDA(cudaMemcpyAsync(snap + i * n, parts[i], b, k, s));
  }
  double *packed[3] = {e->mdV.as<double>(), e->mdF.as<double>(), e->mdXb.as<double>()};
  for (int i = 0; i < 3; ++i) {
    if (restore) MDB_CUDA(cudaMemcpyAsync(packed[i], snap + (3 + 3 * i) * n, 3 * b, k, s));
    else MDB_CUDA(cudaMemcpyAsync(snap + (3 + 3 * i) * n, packed[i], 3 * b, k, s));
  }
  return MDBAS_NB_OK;
}

void md_write_row(double *energies, int row, long long gstep, double pot, double kin) {
  energies[4 * row + 0] = (double)gstep;
  energies[4 * row + 1] = pot;
  energies[4 * row + 2] = kin;
  energies[4 * row + 3] = pot + kin;
}

// Steps [done, done + K*chunks) through the graph.  Returns the number of
// rows written through *outRow.
int md_run_graph(mdbas_nb_engine *e, int chunks, int energyEvery, double targetTemp,
                 double tauT, double kinTemp0, double *energies, int *outRow) {
  const int K = e->mdGraphSteps;
  cudaStream_t s = e->stream;
  long long *word = e->mdWord.as<long long>();
  if (e->mdGraphStale || e->mdGraphK != K || e->mdGraphTau != tauT ||
      e->mdGraphTemp != targetTemp)
    MD_TRY(md_capture(e, K, targetTemp, tauT, kinTemp0));
  MD_TRY(e->mdSnap.ensure(sizeof(double) * 12 * (size_t)e->n));
  std::vector<long long> rows(kRowWords * (size_t)K);
  int growths = 0;
  for (int c = 0; c < chunks;) {
    const long long step0 = e->mdSteps;
    MDB_CUDA(cudaMemcpyAsync(word + W_STEP, &step0, sizeof(long long), cudaMemcpyHostToDevice,
                             s));
    MDB_CUDA(cudaMemsetAsync(word + W_BUILDS, 0, sizeof(long long), s));
    MDB_CUDA(cudaMemsetAsync(word + W_PRUNES, 0, sizeof(long long), s));
    MDB_CUDA(cudaMemsetAsync(e->cl.sticky.p, 0, sizeof(long long), s));
    MD_TRY(md_snapshot(e, false));
    MDB_CUDA(cudaGraphLaunch(e->mdExec, s));
    long long w[W_COUNT], sticky = 0;
    MDB_CUDA(cudaMemcpyAsync(w, word, sizeof(w), cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaMemcpyAsync(&sticky, e->cl.sticky.p, sizeof(sticky), cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaMemcpyAsync(rows.data(), e->mdRows.p, sizeof(long long) * rows.size(),
                             cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaStreamSynchronize(s));
    e->launches += e->mdGraphMainK * K + e->mdGraphBodyK * w[W_BUILDS] +
                   e->mdGraphPruneK * w[W_PRUNES];
    if (sticky & CL_NONFINITE) {
      set_last_status(MDBAS_NB_ERR_NONFINITE, "non-finite positions during dynamics");
      return MDBAS_NB_ERR_NONFINITE;
    }
    if (sticky & CL_OVERFLOW) {
      // a rebuild inside the chunk outgrew the pair list: go back to the
      // chunk's start, enlarge the list and capture again
      if (++growths > 3) return MDBAS_NB_ERR_CAPACITY;
      MD_TRY(md_snapshot(e, true));
      e->cl.entryCap = (long long)(e->cl.entryCap * 1.5) + 4096;
      e->cl.itemCap = (long long)(e->cl.itemCap * 1.5) + 1024;
      MD_TRY(md_build(e));
      if (md_prune_on(e)) {
        MD_TRY(md_refresh_cluster(e, s));
        MD_TRY(md_prune_sync(e));
      }
      MD_TRY(md_capture(e, K, targetTemp, tauT, kinTemp0));
      continue;
    }
    const int st2[2] = {(int)(w[W_SHAKE] & 0xffffffff), (int)(w[W_SHAKE] >> 32)};
    MD_TRY(md_check_shake(e, st2));
    if (w[W_FLAGS] & FLAG_OVERFLOW) {
      set_last_status(MDBAS_NB_ERR_OVERFLOW, "fixed-point overflow (forces or kinetic energy)");
      return MDBAS_NB_ERR_OVERFLOW;
    }
    if (w[W_FLAGS] & FLAG_STAGE) {
      set_last_status(MDBAS_NB_ERR_CUDA, "a bulk copy into shared memory timed out");
      return MDBAS_NB_ERR_CUDA;
    }
    e->mdRebuilds += w[W_BUILDS];
    e->mdPrunes += w[W_PRUNES];
    for (int k = 0; k < K; ++k) {
      const long long gstep = step0 + k + 1;
      if (energies && energyEvery > 0 && gstep % energyEvery == 0) {
        const long long *r = &rows[kRowWords * (size_t)k];
        const double pot = (double)(r[0] + r[1] + r[2] + r[4] + r[5]) / kEnergyScale + e->selfE;
        const double kin = md_kin_row((double)r[3] / kEnergyScale, e->mdDt, tauT, kinTemp0);
        md_write_row(energies, (*outRow)++, gstep, pot, kin);
      }
    }
    e->mdSteps = step0 + K;
    ++c;
  }
  return MDBAS_NB_OK;
}

}  // namespace

void mdbas::md_release(mdbas_nb_engine *e) {
  md_graph_free(e);
  if (e->mdCapStream) cudaStreamDestroy(e->mdCapStream);
  if (e->mdSideStream) cudaStreamDestroy(e->mdSideStream);
  e->mdCapStream = e->mdSideStream = nullptr;
}

extern "C" {

int mdbas_nb_engine_md_init(mdbas_nb_engine *e, const double *mass, const double *vx,
                            const double *vy, const double *vz, double timeStep, int listUpdate,
                            int nConst, const int *constAtoms, const double *constLen2,
                            double tolShake, int maxCycle) {
  if (!e || !mass || !(timeStep > 0.) || listUpdate < 0 || nConst < 0) return MDBAS_NB_ERR_ARG;
  if (!e->topoSet || !e->posSet) return MDBAS_NB_ERR_STATE;
  if (nConst > 0 && (!constAtoms || !constLen2)) return MDBAS_NB_ERR_ARG;
  MDB_CUDA(cudaSetDevice(e->device));
  MD_TRY(engine_resolve_build(e));
  e->accCached = false;
  const int n = e->n;
  std::vector<double> rm(n);
  for (int i = 0; i < n; ++i) {
    if (!(mass[i] > 0.)) return MDBAS_NB_ERR_ARG;
    rm[i] = 1.0 / mass[i];
  }
  md_graph_free(e);
  MD_TRY(e->mdMass.ensure(sizeof(double) * n));
  MD_TRY(e->mdRmass.ensure(sizeof(double) * n));
  MD_TRY(e->mdV.ensure(sizeof(double) * 3 * (size_t)n));
  MD_TRY(e->mdF.ensure(sizeof(double) * 3 * (size_t)n));
  MD_TRY(e->mdXb.ensure(sizeof(double) * 3 * (size_t)n));
  MD_TRY(e->mdWord.ensure(sizeof(long long) * W_COUNT));
  cudaStream_t s = e->stream;
  MDB_CUDA(cudaMemsetAsync(e->mdWord.p, 0, sizeof(long long) * W_COUNT, s));
  MDB_CUDA(cudaMemcpyAsync(e->mdMass.p, mass, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  MDB_CUDA(cudaMemcpyAsync(e->mdRmass.p, rm.data(), sizeof(double) * n, cudaMemcpyHostToDevice,
                           s));
  double *v = e->mdV.as<double>();
  if (vx && vy && vz) {
    MDB_CUDA(cudaMemcpyAsync(v, vx, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaMemcpyAsync(v + n, vy, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaMemcpyAsync(v + 2 * (size_t)n, vz, sizeof(double) * n, cudaMemcpyHostToDevice,
                             s));
  } else {
    MDB_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * 3 * (size_t)n, s));
  }
  // constraints grouped by molecule (connected components)
  e->mdNCons = nConst;
  e->mdNMol = 0;
  e->mdTri = false;
  e->mdNTri = 0;
  if (nConst > 0) {
    std::vector<int> parent(n);
    for (int i = 0; i < n; ++i) parent[i] = i;
    auto find = [&](int a) {
      while (parent[a] != a) a = parent[a] = parent[parent[a]];
      return a;
    };
    std::vector<int> cnt(n, 0);
    for (int k = 0; k < nConst; ++k) {
      const int a = constAtoms[2 * k], b = constAtoms[2 * k + 1];
      if (a < 0 || a >= n || b < 0 || b >= n || a == b || !(constLen2[k] > 0.))
        return MDBAS_NB_ERR_ARG;
      parent[find(a)] = find(b);
      cnt[a]++;
      cnt[b]++;
    }
    std::vector<int> order(nConst), molKey(nConst), rootMol(n, -1);
    int nMol = 0;
    for (int k = 0; k < nConst; ++k) {
      const int r = find(constAtoms[2 * k]);
      if (rootMol[r] < 0) rootMol[r] = nMol++;
      molKey[k] = rootMol[r];
      order[k] = k;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return molKey[a] < molKey[b]; });
    std::vector<int> ca(nConst), cb(nConst), molStart(nMol + 1, 0);
    std::vector<double> r2(nConst);
    for (int t = 0; t < nConst; ++t) {
      const int k = order[t];
      ca[t] = constAtoms[2 * k];
      cb[t] = constAtoms[2 * k + 1];
      r2[t] = constLen2[k];
      molStart[molKey[k] + 1]++;
    }
    for (int m = 0; m < nMol; ++m) molStart[m + 1] += molStart[m];
    // molecule sizes: atoms and constraints of the largest molecule
    std::vector<int> molAtoms(nMol, 0);
    for (int i = 0; i < n; ++i)
      if (cnt[i] > 0) molAtoms[rootMol[find(i)]]++;
    int maxAtoms = 0, maxCons = 0;
    for (int m = 0; m < nMol; ++m) {
      maxAtoms = std::max(maxAtoms, molAtoms[m]);
      maxCons = std::max(maxCons, molStart[m + 1] - molStart[m]);
    }
    if (maxAtoms > kMolMaxAtoms || maxCons > kMolMaxCons) {
      set_last_status(MDBAS_NB_ERR_UNSUPPORTED,
                      "a constrained molecule exceeds 16 atoms or 32 constraints");
      return MDBAS_NB_ERR_UNSUPPORTED;
    }
    // every molecule a rigid triangle (3 atoms, the 3 pairs constrained)?
    bool allTri = true;
    std::vector<int> triAtoms;
    std::vector<double> triLen2;
    if (maxAtoms == 3 && maxCons == 3) {
      triAtoms.resize(4 * (size_t)nMol);
      triLen2.resize(4 * (size_t)nMol);
      for (int m = 0; m < nMol && allTri; ++m) {
        const int c0 = molStart[m];
        if (molStart[m + 1] - c0 != 3) { allTri = false; break; }
        // a0 = the first constraint's first atom, a1 its second, a2 the other
        const int a0 = ca[c0], a1 = cb[c0];
        int a2 = -1;
        for (int k = 1; k < 3; ++k)
          for (int v : {ca[c0 + k], cb[c0 + k]})
            if (v != a0 && v != a1) a2 = v;
        if (a2 < 0) { allTri = false; break; }
        double l01 = -1, l02 = -1, l12 = -1;
        for (int k = 0; k < 3; ++k) {
          const int u = std::min(ca[c0 + k], cb[c0 + k]), v = std::max(ca[c0 + k], cb[c0 + k]);
          if (u == std::min(a0, a1) && v == std::max(a0, a1)) l01 = r2[c0 + k];
          else if (u == std::min(a0, a2) && v == std::max(a0, a2)) l02 = r2[c0 + k];
          else if (u == std::min(a1, a2) && v == std::max(a1, a2)) l12 = r2[c0 + k];
        }
        if (l01 < 0 || l02 < 0 || l12 < 0) { allTri = false; break; }
        triAtoms[4 * m + 0] = a0;
        triAtoms[4 * m + 1] = a1;
        triAtoms[4 * m + 2] = a2;
        triAtoms[4 * m + 3] = 0;
        triLen2[4 * m + 0] = l01;
        triLen2[4 * m + 1] = l02;
        triLen2[4 * m + 2] = l12;
        triLen2[4 * m + 3] = 0.;
      }
    } else {
      allTri = false;
    }
    e->mdTri = allTri;
    e->mdNTri = allTri ? 3 * nMol : 0;
    if (allTri) {
      MD_TRY(e->mdTriAtoms.ensure(sizeof(int4) * (size_t)nMol));
      MD_TRY(e->mdTriLen2.ensure(sizeof(double4) * (size_t)nMol));
      MDB_CUDA(cudaMemcpyAsync(e->mdTriAtoms.p, triAtoms.data(), sizeof(int4) * (size_t)nMol,
                               cudaMemcpyHostToDevice, s));
      MDB_CUDA(cudaMemcpyAsync(e->mdTriLen2.p, triLen2.data(), sizeof(double4) * (size_t)nMol,
                               cudaMemcpyHostToDevice, s));
    }
    e->mdMolClass = (maxAtoms <= kMolTinyAtoms && maxCons <= kMolTinyCons)     ? 0
                    : (maxAtoms <= kMolSmallAtoms && maxCons <= kMolSmallCons) ? 1
                                                                               : 2;
    e->mdNMol = nMol;
    MD_TRY(e->mdCa.ensure(sizeof(int) * nConst));
    MD_TRY(e->mdCb.ensure(sizeof(int) * nConst));
    MD_TRY(e->mdRc2.ensure(sizeof(double) * nConst));
    MD_TRY(e->mdMol.ensure(sizeof(int) * (nMol + 1)));
    MD_TRY(e->mdNAt.ensure(sizeof(int) * n));
    MD_TRY(e->mdDd.ensure(sizeof(double) * 3 * (size_t)nConst));
    MDB_CUDA(cudaMemcpyAsync(e->mdCa.p, ca.data(), sizeof(int) * nConst, cudaMemcpyHostToDevice,
                             s));
    MDB_CUDA(cudaMemcpyAsync(e->mdCb.p, cb.data(), sizeof(int) * nConst, cudaMemcpyHostToDevice,
                             s));
    MDB_CUDA(cudaMemcpyAsync(e->mdRc2.p, r2.data(), sizeof(double) * nConst,
                             cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaMemcpyAsync(e->mdMol.p, molStart.data(), sizeof(int) * (nMol + 1),
                             cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaMemcpyAsync(e->mdNAt.p, cnt.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    MDB_CUDA(cudaStreamSynchronize(s));
  }
  int nFrozen = 0;
  if (e->hasFrozen) {
    std::vector<int> fr(n);
    MDB_CUDA(cudaMemcpyAsync(fr.data(), e->frozen.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    MDB_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < n; ++i) nFrozen += fr[i] != 0;
  }
  // degrees of freedom (get_degfree, src/utils.c:569-581)
  e->mdDegFree = 3 * (n - nFrozen) - 3 * e->nRep - nConst;  // centre of mass per replica
  e->mdDt = timeStep;
  e->mdListUpdate = listUpdate;
  e->mdTol = tolShake > 0. ? tolShake : 1e-8;          // src/io.c:95
  e->mdMaxCycle = maxCycle > 0 ? maxCycle : 150;       // src/io.c:96
  e->mdSteps = 0;
  e->mdRebuilds = 0;
  e->mdShakeIter = 0;
  if (e->grid <= 0) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
    e->grid = sms * 8;
    e->block = 256;
  }
  // forces at the initial positions
  LaunchScope ls(e);
  e->mdPrunes = 0;
  if (md_prune_on(e)) MD_TRY(e->mdXp.ensure(sizeof(double) * 3 * (size_t)n));
  // the search writes the inner list at the pruning radius (or, without
  // pruning, at the cut-off for the build's own positions only)
  e->cl.rin2 = md_prune_on(e) ? md_rin2(e) : 0.f;
  MD_TRY(md_build(e));
  if (e->cfg.precision == 1) MD_TRY(mdbas_nb_engine_refresh(e));
  if (md_prune_on(e)) MD_TRY(md_prune_sync(e));
  MD_TRY(mdbas_nb_engine_compute(e));
  MD_TRY(md_forces(e, e->stream));
  MDB_CUDA(cudaStreamSynchronize(s));
  e->mdReady = true;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_md_set_graph(mdbas_nb_engine *e, int stepsPerLaunch) {
  if (!e || stepsPerLaunch < 0 || stepsPerLaunch > 1000) return MDBAS_NB_ERR_ARG;
  if (stepsPerLaunch != e->mdGraphSteps) {
    e->mdGraphSteps = stepsPerLaunch;
    e->mdGraphStale = true;
  }
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_md_run(mdbas_nb_engine *e, int nSteps, int energyEvery, double targetTemp,
                           double tauT, double *energies) {
  if (!e || nSteps < 0) return MDBAS_NB_ERR_ARG;
  if (!e->mdReady) return MDBAS_NB_ERR_STATE;
  MDB_CUDA(cudaSetDevice(e->device));
  MD_TRY(engine_resolve_build(e));
  e->accCached = false;  // the steps evaluate again
  LaunchScope ls(e);
  cudaStream_t s = e->stream;
  long long *word = e->mdWord.as<long long>();
  const double half2 = 0.25 * e->cfg.delr * e->cfg.delr;
  const double halfIn2 = 0.25 * e->mdPruneBuf * e->mdPruneBuf;
  // kinTemp0 of the Berendsen bath (src/utils.c:555-581)
  const double kinTemp0 = 0.5 * targetTemp * (double)e->mdDegFree * 0.83144621;
  MDB_CUDA(cudaMemsetAsync(word + W_SHAKE, 0, sizeof(long long), s));
  MDB_CUDA(cudaMemsetAsync(word + W_FLAGS, 0, sizeof(long long), s));
  int outRow = 0;
  int done = 0;
  // whole graph launches first (mixed precision only)
  const int K = e->mdGraphSteps;
  if (e->cfg.precision == 1 && K > 0 && nSteps >= K) {
    const int chunks = nSteps / K;
    MD_TRY(md_run_graph(e, chunks, energyEvery, targetTemp, tauT, kinTemp0, energies, &outRow));
    done = chunks * K;
  }
  for (int step = done; step < nSteps; ++step) {
    const long long gstep = e->mdSteps + 1;
    MD_TRY(md_stage1(e, s));
    // list: fixed cadence or half-skin displacement; inner list: a rebuild
    // or half the prune buffer since the last prune (k_decide's rules)
    const bool prune = md_prune_on(e);
    double d2 = 0., p2 = 0.;
    if (e->mdListUpdate == 0 || prune) {
      MD_TRY(md_max_disp(e, s));
      unsigned long long bits[2] = {0, 0};
      MDB_CUDA(cudaMemcpyAsync(&bits[0], word + W_DISP, sizeof(bits[0]), cudaMemcpyDeviceToHost,
                               s));
      MDB_CUDA(cudaMemcpyAsync(&bits[1], word + W_DISP2, sizeof(bits[1]),
                               cudaMemcpyDeviceToHost, s));
      MDB_CUDA(cudaStreamSynchronize(s));
      memcpy(&d2, &bits[0], sizeof(d2));
      memcpy(&p2, &bits[1], sizeof(p2));
    }
    const bool rebuild = e->mdListUpdate > 0 ? (gstep % e->mdListUpdate) == 0 : d2 > half2;
    if (rebuild) MD_TRY(md_build(e));
    if (e->cfg.precision == 1) MD_TRY(mdbas_nb_engine_refresh(e));
    if (prune && (rebuild || p2 > halfIn2)) MD_TRY(md_prune_sync(e));
    MD_TRY(mdbas_nb_engine_compute(e));
    MD_TRY(md_forces(e, s));
    const bool wantE = energies && energyEvery > 0 && (gstep % energyEvery) == 0;
    MD_TRY(md_stage2(e, s, wantE, tauT, kinTemp0));
    if (wantE) {
      long long kfix = 0;
      MDB_CUDA(cudaMemcpyAsync(&kfix, word + W_KIN, sizeof(kfix), cudaMemcpyDeviceToHost, s));
      long long bfix = 0, kfixr = 0;
      if (const long long *b = md_bonded_fix(e))
        MDB_CUDA(cudaMemcpyAsync(&bfix, b, sizeof(bfix), cudaMemcpyDeviceToHost, s));
      if (const long long *k = md_kspace_fix(e))
        MDB_CUDA(cudaMemcpyAsync(&kfixr, k, sizeof(kfixr), cudaMemcpyDeviceToHost, s));
      mdbas_nb_energies en;
      MD_TRY(mdbas_nb_engine_energies(e, &en));  // synchronises the stream
      const double pot = en.elec_direct + en.elec_corr + en.elec_self + en.vdw +
                         (double)(bfix + kfixr) / kEnergyScale;
      md_write_row(energies, outRow++, gstep,
                   pot, md_kin_row((double)kfix / kEnergyScale, e->mdDt, tauT, kinTemp0));
    }
    e->mdSteps = gstep;
  }
  // constraint status
  long long w[W_COUNT];
  MDB_CUDA(cudaMemcpyAsync(w, word, sizeof(w), cudaMemcpyDeviceToHost, s));
  MDB_CUDA(cudaStreamSynchronize(s));
  const int st2[2] = {(int)(w[W_SHAKE] & 0xffffffff), (int)(w[W_SHAKE] >> 32)};
  MD_TRY(md_check_shake(e, st2));
  if (w[W_FLAGS] & FLAG_OVERFLOW) {
    set_last_status(MDBAS_NB_ERR_OVERFLOW, "fixed-point kinetic energy overflow");
    return MDBAS_NB_ERR_OVERFLOW;
  }
  e->computed = true;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_md_stats(mdbas_nb_engine *e, long long out[6]) {
  if (!e || !out) return MDBAS_NB_ERR_ARG;
  out[0] = e->mdSteps;
  out[1] = e->mdRebuilds;
  out[2] = e->mdShakeIter;
  out[3] = e->mdNMol;
  out[4] = e->mdPrunes;
  out[5] = e->cl.useInner ? 1 : 0;
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_md_set_prune(mdbas_nb_engine *e, double buffer) {
  if (!e || buffer < 0. || buffer > e->cfg.delr) return MDBAS_NB_ERR_ARG;
  e->mdPruneBuf = buffer;
  e->mdGraphStale = true;
  e->mdReady = false;  // md_init sets the lists up for the new setting
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_get_positions(mdbas_nb_engine *e, double *x, double *y, double *z,
                                  int device_ptrs) {
  if (!e || !x || !y || !z) return MDBAS_NB_ERR_ARG;
  MDB_CUDA(cudaSetDevice(e->device));
  const cudaMemcpyKind k = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t bytes = sizeof(double) * (size_t)e->n;
  MDB_CUDA(cudaMemcpyAsync(x, e->x.p, bytes, k, e->stream));
  MDB_CUDA(cudaMemcpyAsync(y, e->y.p, bytes, k, e->stream));
  MDB_CUDA(cudaMemcpyAsync(z, e->z.p, bytes, k, e->stream));
  MDB_CUDA(cudaStreamSynchronize(e->stream));
  return MDBAS_NB_OK;
}

int mdbas_nb_engine_get_velocities(mdbas_nb_engine *e, double *vx, double *vy, double *vz,
                                   int device_ptrs) {
  if (!e || !vx || !vy || !vz) return MDBAS_NB_ERR_ARG;
  if (!e->mdReady) return MDBAS_NB_ERR_STATE;
  MDB_CUDA(cudaSetDevice(e->device));
  const cudaMemcpyKind k = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t bytes = sizeof(double) * (size_t)e->n;
  const double *v = e->mdV.as<double>();
  MDB_CUDA(cudaMemcpyAsync(vx, v, bytes, k, e->stream));
  MDB_CUDA(cudaMemcpyAsync(vy, v + e->n, bytes, k, e->stream));
  MDB_CUDA(cudaMemcpyAsync(vz, v + 2 * (size_t)e->n, bytes, k, e->stream));
  MDB_CUDA(cudaStreamSynchronize(e->stream));
  return MDBAS_NB_OK;
}

}  // extern "C"
