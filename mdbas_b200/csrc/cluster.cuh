// cluster.cuh -- cell-sorted 8-atom cluster layout and cluster-pair list.
#pragma once

#include "common.cuh"

namespace mdbas {

constexpr int kClusterSize = 8;
constexpr int kItemMax = 32;  // j-clusters per work item of the pair kernel

// Geometry of the column grid (x-y cells, atoms sorted by z inside a cell).
struct ClusterGeom {
  int ncx, ncy;       // cells per side in x and y
  int Dx, Dy;         // cell offsets searched on each side
  double Lx, Ly, Lz;  // orthorhombic box edges
  double wx, wy;      // cell widths
  float rlist2;       // (rc + delr)^2 with a small safety margin
};

// One cluster-pair entry: j cluster and the FP32 shift vector
// (o_j + S - o_i, computed in FP64 from the cluster origins).
struct CPairEntry {
  int j;
  float sx, sy, sz;
};

struct ClusterWork {
  // grid
  ClusterGeom geom{};
  int nCols = 0;
  DBuf colRank;       // (cy*ncx+cx) -> column slot in Morton order
  DBuf colXY;         // column slot -> cx | cy << 16
  DBuf colCount, colFill, colStart, colPad, colPadStart;
  DBuf atomCol, tmpIdx;
  DBuf atomZ;         // wrapped fractional z (FP64)
  DBuf scanTmp;
  // layout
  int nSlots = 0, nClusters = 0;
  DBuf slotAtom;      // slot -> atom (-1 for padding)
  DBuf slotOf;        // atom -> slot
  DBuf clusterXY;     // cluster -> cx | cy << 16
  DBuf colClStart;    // column slot -> first cluster (nCols + 1)
  DBuf origin;        // double4 per cluster (FP64 origin)
  DBuf originF;       // float4 per cluster (FP32 origin, w = real atoms)
  DBuf hmax;          // int[4]: largest half extent per axis (float bits)
  DBuf half;          // float4 per cluster (bbox half extents, w = real atoms)
  DBuf xq;            // float4 per slot: position - origin, q*sqrt(C)
  DBuf lj;            // float2 per slot: 2*eps_i, sig_i
  // pair list
  DBuf entries;       // CPairEntry
  DBuf masks;         // uint2 (64 interaction bits)
  DBuf items;         // int4: i cluster, first entry, entry count, 0
  DBuf counters;      // int64[4]: entries, items, overflow flag, candidates
  long long entryCap = 0, itemCap = 0;
  long long nEntries = 0, nItems = 0;
  // accumulators
  DBuf facc;          // int64 fixed-point forces, SoA [3][nSlots]
  DBuf acc;           // int64[ACC_COUNT]
};

// Sort atoms into cells/clusters and build the cluster-pair list.
int cluster_build(ClusterWork &w, int n, const DevBox &b, double cutOff, double delr,
                  double sqrtC, const double *x, const double *y, const double *z,
                  const double *q, const double *eps, const double *sig, const int *frozen,
                  const int *exclStart, const int *exclFlat, cudaStream_t s);
// Refresh xq from the current FP64 positions (list kept).
int cluster_refresh(ClusterWork &w, int n, const DevBox &b, const double *x, const double *y,
                    const double *z, const double *q, double sqrtC, cudaStream_t s);

}  // namespace mdbas
