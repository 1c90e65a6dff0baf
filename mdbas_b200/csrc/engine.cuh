// engine.cuh -- the device-resident engine object behind mdbas_nb_engine_*.
#pragma once

#include "cluster.cuh"
#include "list_ref.cuh"

struct mdbas_nb_engine {
  mdbas_nb_engine_config cfg{};
  int n = 0;
  int device = 0;
  PBC hostBox{};
  mdbas::DevBox box{};
  mdbas::PairParams pp{};
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  // topology (caller's atom order)
  mdbas::DBuf q, eps, sig, frozen, exclStart, exclFlat;
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
  int variant = 0;  // pair kernel variant (kPairDense)
  // export scratch
  mdbas::DBuf exportBuf, exportCount;
  // bookkeeping
  bool built = false, computed = false;
  long long launches = 0;
  bool timing = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double pairMs = 0.0;
  long long pairCount = 0;
};

namespace mdbas {
int engine_check_device(int device);
PairParams make_params(double cutOff, double cutOn, double alpha, double chargeConst,
                       int vdwSwitch, int elecType);
}  // namespace mdbas
