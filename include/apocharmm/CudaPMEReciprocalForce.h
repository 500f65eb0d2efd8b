// CudaPMEReciprocalForce: the reciprocal-space part of a ForceManager's PME
// force field as a force object: the reference's
// include/CudaPMEReciprocalForce.h:21-240 (calc_force(xyzq, calcEnergy,
// calcVirial), getForce, clear, setBoxDimensions).  B-spline charge spread,
// 3-D FFT, influence function, gather; energies "ewks" (reciprocal sum) and
// "ewse" (self energy).  Grid and spline order are the manager's
// (ForceManager::setFFTGrid / setPmeSplineOrder).
#pragma once

#include <memory>

#include "apocharmm/ForcePart.h"

class CudaPMEReciprocalForce : public ForcePart {
 public:
  explicit CudaPMEReciprocalForce(std::shared_ptr<ForceManager> fm)
      : ForcePart(std::move(fm), 4, {"ewks", "ewse"}) {}
};
