// bonded.cuh -- MDBas's bonded terms (src/internal.c) on the device.
#pragma once

#include <vector>

#include "common.cuh"

namespace mdbas {

// Kinds in the order MDBas's energy() evaluates them (src/energy.c:167-190).
enum BondedKind { KIND_BOND = 0, KIND_ANGLE = 1, KIND_UB = 2, KIND_DIHEDRAL = 3,
                  KIND_IMPROPER = 4, KIND_COUNT = 5 };

// Energy slots of BondedTerms::sums: the five energies in kind order, then
// the bond and Urey-Bradley virials; slot 7 holds the total energy in fixed
// point (2^-24 units, int64 bits).
enum BondedSum { BS_VIRBOND = 5, BS_VIRUB = 6, BS_FIX = 7, BS_COUNT = 8 };

// One topology's bonded terms, device resident.  Each term writes its force
// on each of its atoms into its own contribution slot (no atomics); a gather
// pass then adds an atom's slots to its force in slot order.  Slots are
// numbered kind by kind, term by term, atom by atom, which is exactly the
// order in which MDBas's loops add into fx[i], so every force component is
// accumulated in MDBas's order.  Energies and virials are summed per block
// and then over blocks in a fixed order: deterministic, run to run.
struct BondedTerms {
  int nAtom = 0;
  int count[KIND_COUNT] = {};
  int termBase[KIND_COUNT + 1] = {};  // flat term index of each kind's first term
  int slotBase[KIND_COUNT + 1] = {};  // first contribution slot of each kind
  DBuf terms[KIND_COUNT];             // MDBas structs (BOND/ANGLE/BOND/DIHE/DIHE)
  DBuf contrib;                       // 3 * nSlots doubles (x block, y block, z block)
  DBuf atomStart, atomSlot;           // per-atom slot lists (CSR)
  DBuf part;                          // per-block partial sums
  DBuf sums;                          // BS_COUNT doubles
  std::vector<char> hostCopy;         // terms as last uploaded (drop-in cache)
  int nTerms() const { return termBase[KIND_COUNT]; }
  int nSlots() const { return slotBase[KIND_COUNT]; }
};

// Upload terms (host arrays of MDBas structs, indexed by kind) for nAtom
// atoms and build the slot lists.  Every atom index must lie in [0, nAtom).
int bonded_set(BondedTerms &t, int nAtom, const int count[KIND_COUNT],
               const void *const terms[KIND_COUNT], cudaStream_t s);
// Forces added in place to f (3 * nAtom: x block, y block, z block, device)
// and the energy sums into t.sums, at positions x, y, z (device).  boxes /
// atomRep: the per-replica boxes and atom -> replica map (atomRep may be null
// for a single box).
int bonded_eval(BondedTerms &t, const DevBox *boxes, const int *atomRep, const double *x,
                const double *y, const double *z, double *f, cudaStream_t s);

}  // namespace mdbas
