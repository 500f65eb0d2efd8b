// CudaPMEDirectForce<long long int, float>: the direct-space part of a
// ForceManager's PME force field as a force object: the reference's
// include/CudaPMEDirectForce.h:109-420 (calc_force(xyzq, calcEnergy,
// calcVirial), resetNeighborList, getForce, clear, setBoxDimensions).
// Terms: real-space Ewald electrostatics and force-switched Lennard-Jones
// over the tile list, the 1-4 pairs, and the Ewald exclusion corrections;
// energies "elec" "vdw" "ewex".
#pragma once

#include <memory>
#include <type_traits>

#include "apocharmm/ForcePart.h"

template <typename AT = long long int, typename CT = float>
class CudaPMEDirectForce : public ForcePart {
  static_assert(std::is_same<AT, long long int>::value && std::is_same<CT, float>::value,
                "CudaPMEDirectForce: the library accumulates in long long int from float "
                "coordinates");

 public:
  explicit CudaPMEDirectForce(std::shared_ptr<ForceManager> fm)
      : ForcePart(std::move(fm), 2 | 8, {"elec", "vdw", "ewex"}) {}
};
