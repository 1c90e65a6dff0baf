// engine.cuh -- the device-resident engine object behind mdbas_nb_engine_*.
#pragma once

#include <vector>

#include "bonded.cuh"
#include "cluster.cuh"
#include "kspace.cuh"
#include "list_ref.cuh"

struct mdbas_nb_engine {
  mdbas_nb_engine_config cfg{};
  int n = 0;
  int device = 0;
  PBC hostBox{};
  mdbas::DevBox box{};          // replica 0's box
  // batch of independent boxes (a single system is a batch of one)
  int nRep = 1;
  std::vector<mdbas::DevBox> repBoxes;  // nRep
  std::vector<int> repOff;              // nRep + 1 atom offsets
  mdbas::DBuf boxesDev;                 // DevBox[nRep]
  mdbas::DBuf atomRepDev;               // atom -> replica (nRep > 1)
  const int *atomRepPtr() const { return nRep > 1 ? atomRepDev.as<int>() : nullptr; }
  mdbas::PairParams pp{};
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  // topology (caller's atom order)
  mdbas::DBuf q, eps, sig, frozen, exclStart, exclFlat;
  // the exclusion rows made symmetric (each excluded pair in both atoms'
  // rows, once), as the cluster search reads them
  mdbas::DBuf exclStartSym, exclFlatSym;
  std::vector<int> hExclStartSym, hExclFlatSym;
  bool hasFrozen = false;
  bool topoSet = false;
  double selfE = 0.0;
  // positions (FP64, caller's atom order)
  mdbas::DBuf x, y, z;
  bool posSet = false;
  // precision 0: MDBas-format list + FP64 accumulators
  mdbas::RefListWork ref;
  mdbas::DBuf f64, acc64;
  // precision 1: cluster layout + fixed-point accumulators
  mdbas::ClusterWork cl;
  mdbas::DBuf fout;
  int grid = 0, block = 0;
  int variant = 7;  // pair kernel variant (kPairHalfLean)
  // export scratch
  mdbas::DBuf exportBuf, exportCount;
  // adjoint scratch (adjoint.cu)
  mdbas::DBuf adjBuf;
  // bonded terms (bonded.cu), added to the dynamics forces
  mdbas::BondedTerms bonded;
  mdbas::DBuf bondedF;
  // reciprocal space of the dynamics (md_kspace.cu): 0 none, 1 explicit
  // Ewald (m-range kspaceM), 2 SPME (grid kspaceM, order kspaceOrder)
  int kspaceKind = 0;
  int kspaceM[3] = {0, 0, 0};
  int kspaceOrder = 0;
  double kspaceSystq = 0.0, kspaceSumq2 = 0.0;
  mdbas::EwaldWork *kEwald = nullptr;
  mdbas::SpmeWork *kSpme = nullptr;
  mdbas::DBuf kspaceFix, kspaceF;  // int64 energy word; scratch forces (3n)
  // bookkeeping
  bool built = false, computed = false;
  // a build ran without reading its counts back (precision 1, same grid and
  // capacities as the build before): its error bits wait in cl.sticky until
  // the next call that returns results (engine_resolve_build)
  bool buildPending = false;
  // energy accumulators read back with the forces (same synchronisation);
  // energies() uses them until the next evaluation
  bool accCached = false;
  long long accCache[8] = {};
  double acc64Cache[8] = {};
  long long launches = 0;
  bool timing = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // second stream of compute(): the exclusion correction runs beside the
  // pair kernel (both add into the same fixed-point words)
  cudaStream_t side = nullptr;
  cudaEvent_t evFork = nullptr, evJoin = nullptr;
  double pairMs = 0.0;
  long long pairCount = 0;
  // velocity-Verlet state (md.cu)
  mdbas::DBuf mdMass, mdRmass, mdV, mdF, mdXb, mdWord;
  mdbas::DBuf mdCa, mdCb, mdRc2, mdMol, mdNAt, mdDd;
  int mdNCons = 0, mdNMol = 0, mdListUpdate = 0, mdMaxCycle = 150, mdDegFree = 0;
  double mdDt = 0.0, mdTol = 1e-8;
  long long mdSteps = 0, mdRebuilds = 0, mdShakeIter = 0;
  bool mdReady = false;
  bool mdTri = false;   // every constrained molecule a rigid triangle (fused kernels)
  int mdNTri = 0;       // atoms in those triangles
  mdbas::DBuf mdTriAtoms, mdTriLen2;  // int4 / double4 per molecule
  int mdMolClass = 0;  // SHAKE kernel class: 0 <= 3 atoms/3 constraints, 1 <= 4/6, 2 <= 16/32
  // CUDA graph of mdGraphSteps whole steps (precision 1); rebuilt when stale
  int mdGraphSteps = 20, mdGraphK = 0;
  long long mdGraphMainK = 0, mdGraphBodyK = 0;  // kernels per step / per rebuild
  long long mdGraphPruneK = 0;                   // kernels per prune
  double mdPruneBuf = 0.0;  // inner-list buffer (A) of the mixed form; 0 = no pruning
  mdbas::DBuf mdXp;         // positions at the last prune
  long long mdPrunes = 0;
  bool mdGraphStale = true;
  double mdGraphTau = 0.0, mdGraphTemp = 0.0;
  cudaGraph_t mdGraph = nullptr;
  cudaGraphExec_t mdExec = nullptr;
  cudaStream_t mdCapStream = nullptr, mdSideStream = nullptr;
  mdbas::DBuf mdRows, mdSnap;
};

namespace mdbas {
// Counts the library's kernel launches into an engine for the lifetime of
// the scope; nested scopes restore the outer counter.
struct LaunchScope {
  long long *prev;
  explicit LaunchScope(mdbas_nb_engine *e) : prev(g_launch_counter) {
    g_launch_counter = &e->launches;
  }
  ~LaunchScope() { g_launch_counter = prev; }
};
int engine_check_device(int device);
// Releases the dynamics graph and its streams (md.cu).
void md_release(mdbas_nb_engine *e);
// Reciprocal forces added to f (3n, caller order) and the reciprocal plus
// non-neutral energy into kspaceFix (md_kspace.cu); no-op when off.
int md_kspace(mdbas_nb_engine *e, double *f, cudaStream_t s);
// Settle a pending build (see buildPending): read its error bits; on an
// overflowing list build again with room, synchronously, and redo the
// evaluation if one ran on the empty list; non-finite positions are an error.
int engine_resolve_build(mdbas_nb_engine *e);
// Settle a pending build whose error word (already read) holds a failure.
int engine_settle_build(mdbas_nb_engine *e, long long sticky);
// The engine's side stream and its fork/join events (created once, outside
// any stream capture).
int engine_side_stream(mdbas_nb_engine *e);
void kspace_release(mdbas_nb_engine *e);
// MDBas's choice of list builder for this engine (cluster_build's listRule).
inline int engine_list_rule(const mdbas_nb_engine *e) {
  return list_rule(e->cfg.linkRatio, e->cfg.noLink);
}
PairParams make_params(double cutOff, double cutOn, double alpha, double chargeConst,
                       int vdwSwitch, int elecType);
}  // namespace mdbas
