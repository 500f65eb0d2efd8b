// CudaBondedForce<long long int, float>: the bonded terms of a ForceManager
// (bond, Urey-Bradley, angle, proper and improper dihedral) as a force
// object: the reference's include/CudaBondedForce.h:38-200
// (calc_force(xyzq, calcEnergy, calcVirial), getForce, clear,
// setBoxDimensions), energies "bond" "angle" "ureyb" "dihe" "imdihe".  The
// 1-4 pairs belong to CudaPMEDirectForce, as in the reference.
#pragma once

#include <memory>
#include <type_traits>

#include "apocharmm/ForcePart.h"

template <typename AT = long long int, typename CT = float>
class CudaBondedForce : public ForcePart {
  static_assert(std::is_same<AT, long long int>::value && std::is_same<CT, float>::value,
                "CudaBondedForce: the library accumulates in long long int from float coordinates");

 public:
  explicit CudaBondedForce(std::shared_ptr<ForceManager> fm)
      : ForcePart(std::move(fm), 1 | 8, {"bond", "angle", "ureyb", "dihe", "imdihe"}) {}
};
