// cluster.cuh -- cell-sorted 8-atom cluster layout and cluster-pair list.
#pragma once

#include <vector>

#include "common.cuh"

namespace mdbas {

constexpr int kClusterSize = 8;
constexpr int kItemMax = 32;  // j-clusters per work item of the pair kernel
constexpr int kZBins = 64;    // z bins per column of the search's cluster lookup table

// Geometry of the column grid (x-y cells, atoms sorted by z inside a cell).
//
// The list keeps exactly the pairs MDBas's list builder keeps.  Pair
// distances are tested in FP32 against a band around the list radius:
// r2 <= rlo2 is in, r2 > rhi2 is out, and a pair inside the band is decided
// by MDBas's own FP64 expression (listMode 1: link cells, fractional
// coordinates of src/list.c:1932-1936 and 2051-2057; listMode 0: all pairs,
// dist() of src/utils.c:38-80) against cutnb2 = (rc + delr)^2.  The band
// (2e-5 relative, ~0.004 A^2 at 14 A) is ten times the FP32 error of the
// cluster-relative distances.
struct ClusterGeom {
  int ncx, ncy;       // cells per side in x and y
  int Dx, Dy;         // cell offsets searched on each side
  double Lx, Ly, Lz;  // orthorhombic box edges
  double invLx, invLy, invLz;  // 1 / edge (the FP64 quotient the device would form)
  double wx, wy;      // cell widths
  float rlist2;       // candidate test: rhi2
  float rlo2, rhi2;   // FP32 band around the list radius
  double cutnb2;      // MDBas's list radius squared (FP64)
  int listMode;       // 1: MDBas's link-cell list, 0: its all-pairs list
};

// One entry of the inner list: a 4-atom half of a j cluster (jh = 2 j + h,
// atoms 4h..4h+3) with the cluster pair's FP32 shift; its 32-bit mask holds
// bit i + 8 k for i atom i and half atom k.
struct HalfEntry {
  int jh;
  float sx, sy, sz;
};

// One cluster-pair entry: j cluster and the FP32 shift vector
// (o_j + S - o_i, computed in FP64 from the cluster origins).
struct CPairEntry {
  int j;
  float sx, sy, sz;
};

// The layout holds a batch of independent boxes ("replicas"): replica r owns
// atoms [atomOff[r], atomOff[r+1]) of the concatenated arrays and columns
// [colOff[r], colOff[r+1]) of the global column numbering, hence a
// contiguous run of slots and clusters; cluster-pair entries name global
// clusters, so one pair-kernel launch serves every replica.  A single system
// is a batch of one.
struct ClusterWork {
  // grid
  int nRep = 0;
  std::vector<ClusterGeom> geomH;  // per replica
  std::vector<int> colOffH;        // nRep + 1
  std::vector<int> atomOffH;       // nRep + 1
  DBuf geoms;         // ClusterGeom[nRep]
  DBuf colOff;        // int[nRep + 1]
  DBuf boxes;         // DevBox[nRep]
  DBuf atomRep;       // atom -> replica (nRep > 1 only)
  DBuf clusterRep;    // cluster -> replica (nRep > 1 only)
  ClusterGeom geom{}; // replica 0's grid (single-system callers)
  int nCols = 0;      // columns of all replicas
  DBuf colRank;       // colOff[r] + (cy*ncx+cx) -> global column, Morton order inside r
  DBuf colXY;         // global column -> cx | cy << 16
  DBuf colCount, colFill, colStart, colPadStart;
  DBuf atomCol, tmpIdx;
  DBuf atomZ;         // wrapped fractional z (FP64)
  // layout.  Slot-indexed buffers hold slotCap = n + 7 * nCols slots (rounded
  // up to a whole cluster), the most that per-column padding can produce, so
  // a rebuild never reallocates and kernels read the actual count on the
  // device (colPadStart[nCols]).  nSlots/nClusters are host copies, valid
  // after a synchronising build or cluster_read_counts.
  int slotCap = 0, clCap = 0;
  int nSlots = 0, nClusters = 0;
  DBuf slotAtom;      // slot -> atom (-1 for padding)
  DBuf slotOf;        // atom -> slot
  DBuf clusterXY;     // cluster -> cx | cy << 16
  DBuf colClStart;    // column slot -> first cluster (nCols + 1)
  DBuf zTab;          // int[nCols * (kZBins + 1)]: per column and z bin b, the first
                      // cluster whose origin z is at least -Lz/2 + b Lz / kZBins
  DBuf origin;        // double4 per cluster (FP64 origin)
  DBuf originF;       // float4 per cluster (FP32 origin, w = real atoms)
  DBuf hmax;          // int[4 * nRep]: largest half extent per axis (float bits)
  DBuf half;          // float4 per cluster (bbox half extents, w = real atoms)
  DBuf xq;            // float4 per slot: position - origin, q*sqrt(C)
  DBuf lj;            // float2 per slot: 2*eps_i, sig_i
  // The same slot data paired for packed (f32x2) arithmetic: for cluster c
  // and h = 0..3 the atoms a = h and b = h + 4 sit side by side,
  //   xp[2(4c+h)]   = (x_a, x_b, y_a, y_b), xp[2(4c+h)+1] = (z_a, z_b, q_a, q_b),
  //   ljp[4c+h]     = (2eps_a, 2eps_b, sig_a, sig_b),
  // so one lane's two j atoms load as float2 pairs.
  DBuf xp;            // float4[8 per cluster]
  DBuf ljp;           // float4[4 per cluster]
  // pair list
  DBuf entries;       // CPairEntry
  DBuf masks;         // uint2 (64 interaction bits)
  DBuf items;         // int4: i cluster, first entry, entry count, 0
  DBuf counters;      // int64[8]: entries, items, overflow flag, candidates, the search's
                      // packed count (items << 40 | entries taken), entries kept, -,
                      // search warps finished
  long long entryCap = 0, itemCap = 0;
  long long nEntries = 0, nItems = 0;
  // Inner list: the j-cluster halves of the list above that hold a pair
  // within the inner radius (rin2), with 32-bit masks of those pairs, written
  // by the search at build time and by the prune pass during dynamics.  The
  // half-cluster pair kernel reads it while useInner is set, the full list
  // otherwise.  Items hold up to 2 * kItemMax half entries.
  DBuf entriesIn;     // HalfEntry
  DBuf masksIn;       // uint32
  DBuf itemsIn;       // int4: i cluster, first half entry, count, 0
  DBuf countersIn;    // int64[8]: entries, items, overflow flag, warp steps, pairs
                      // within the inner radius, the search's packed count
  long long inEntryCap = 0, inItemCap = 0;
  float rin2 = 0.f;   // radius^2 of the inner list the search writes (0: the
                      // pair kernel's own FP32 rc^2, an exact inner list)
  float innerRin2 = 0.f;  // radius^2 of the inner list as last written
  long long nInEntries = 0, nInItems = 0, nInSteps = 0;  // host copies (synchronising builds)
  bool useInner = false;
  DBuf sticky;        // int64: OR of every build's error bits since last read
  // stage timing of a synchronising build (cluster_build_stages): events
  // after binning, the grid scans, the scatter, the column sort, the cluster
  // layout and the search
  bool timeStages = false;
  cudaEvent_t stageEv[7] = {};
  // accumulators
  DBuf facc;          // int64 fixed-point forces, SoA [3][slotCap]
  DBuf acc;           // int64[ACC_COUNT]
  ~ClusterWork() {
    for (cudaEvent_t ev : stageEv)
      if (ev) cudaEventDestroy(ev);
  }
  const int *nSlotsDev() const { return colPadStart.as<int>() + nCols; }
  const int *atomRepDev() const { return nRep > 1 ? atomRep.as<int>() : nullptr; }
  const int *clusterRepDev() const { return nRep > 1 ? clusterRep.as<int>() : nullptr; }
};

// Bits of ClusterWork::counters[2] and ::sticky.
enum ClusterFlag { CL_OVERFLOW = 1, CL_NONFINITE = 2 };

// Sort atoms into cells/clusters and build the cluster-pair list.
// sync = true: the host reads the counts back, grows the pair-list capacity
// and searches again when it overflowed.  sync = false: no host interaction
// and no allocation (the form captured into CUDA graphs); the layout must
// have been set up by an earlier synchronising build of the same geometry,
// and an overflow only raises CL_OVERFLOW in `sticky`.
// Batch form: nRep boxes, atomOff[nRep + 1] atom ranges (host arrays).
// listRule: MDBas's makelist choice of list builder (bits 0-2 linkRatio,
// bit 3 noLink), which decides the FP64 expression that settles pairs at the
// list radius.  Exclusion rows must be symmetric (cluster_symmetric_excl).
// The inner list is written at w.rin2 (0: rc^2 with a 1e-5 margin).
int cluster_build(ClusterWork &w, int n, int nRep, const DevBox *boxes, const int *atomOff,
                  double cutOff, double delr, int listRule, double sqrtC, const double *x,
                  const double *y, const double *z, const double *q, const double *eps,
                  const double *sig, const int *frozen, const int *exclStart,
                  const int *exclFlat, cudaStream_t s, bool sync = true);
// Single box.
int cluster_build(ClusterWork &w, int n, const DevBox &b, double cutOff, double delr,
                  int listRule, double sqrtC, const double *x, const double *y,
                  const double *z, const double *q, const double *eps, const double *sig,
                  const int *frozen, const int *exclStart, const int *exclFlat, cudaStream_t s,
                  bool sync = true);
// Exclusion rows as the cluster search reads them: each excluded pair in
// both atoms' rows, once (MDBas's all-pairs builder keeps half rows).
void cluster_symmetric_excl(int n, const int *start, const int *flat, std::vector<int> &outStart,
                            std::vector<int> &outFlat);
inline int list_rule(int linkRatio, int noLink) { return (linkRatio & 7) | (noLink ? 8 : 0); }
// Prune the list into the inner list: keep the pairs within sqrt(rin2) at the
// current layout (after cluster_refresh), drop entries left without pairs.
// No host interaction (graph-capturable); requires a synchronising build.
int cluster_prune(ClusterWork &w, float rin2, cudaStream_t s);
// A synchronising build with CUDA events between its stages; ms[0..5] =
// binning, grid scans, scatter, column sort, cluster layout, search.
int cluster_build_stages(ClusterWork &w, int n, int nRep, const DevBox *boxes,
                         const int *atomOff, double cutOff, double delr, int listRule,
                         double sqrtC, const double *x, const double *y, const double *z,
                         const double *q, const double *eps, const double *sig,
                         const int *frozen, const int *exclStart, const int *exclFlat,
                         cudaStream_t s, double ms[6]);
// Host copies of the list counts (synchronises the stream).
int cluster_read_counts(ClusterWork &w, cudaStream_t s);
// Refresh xq from the current FP64 positions (list kept).
int cluster_refresh(ClusterWork &w, const double *x, const double *y, const double *z,
                    const double *q, double sqrtC, cudaStream_t s);

}  // namespace mdbas
