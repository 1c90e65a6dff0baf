// list_ref.cuh -- MDBas-format list builders and their workspace.
#pragma once

#include "common.cuh"

namespace mdbas {

struct RefListWork {
  // outputs (device)
  DBuf list;        // neighList entries (int32)
  DBuf neighPair;   // per atom (int32)
  DBuf order;       // neighOrder (int32)
  DBuf off;         // entry offset of each neighOrder position (int64, n+1)
  long long entries = 0;
  int linkCells = 0;
  int nlc[3] = {0, 0, 0};
  int ncell = 0;
  // scratch
  DBuf xu, yu, zu, xs, ys, zs, fs, cellOf, posOf, tmpIdx, cellCount, cellFill, cellStart, cnt,
      scanTmp, flags;
};

int image_update_device(int n, const DevBox &b, double *x, double *y, double *z, cudaStream_t s);
int link_cell_dims(const DevBox &b, double cutOff, double delr, int linkRatio, int nlc[3]);
int makelist_uses_link_cells(const DevBox &b, double cutOff, double delr, int linkRatio,
                             int noLink);
// Build MDBas's half list on the device.  x/y/z (device, FP64) must already be
// wrapped when restating the first link-cell build.  frozen may be null.
// exclStart/exclFlat: CSR exclusion rows on the device (MDBas's rows).
int build_ref_list(RefListWork &w, int n, const DevBox &b, double cutOff, double delr,
                   int linkRatio, int linkCells, const double *x, const double *y,
                   const double *z, const int *frozen, const int *exclStart,
                   const int *exclFlat, cudaStream_t s);
// Offsets of a caller-supplied list already copied into w.neighPair/w.order.
int ref_list_offsets(RefListWork &w, int n, cudaStream_t s);

}  // namespace mdbas
