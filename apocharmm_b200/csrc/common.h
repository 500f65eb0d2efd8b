// Shared definitions of the B200 force/step engine.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace apo {

// Physical constants, as used throughout CHARMM and the reference engine
// (src/CudaDirectForceKernels.cu:59, include/Constants.h).
constexpr double kCcelec = 332.0716;
constexpr double kBoltz = 1.987191e-3;
constexpr double kTimfac = 0.0488882129;  // AKMA time unit in ps

// Fixed-point scales.  Gradients: 2^40 (the reference's FORCE_SCALE,
// include/gpu_utils.h:21) so a component of up to 8.4e6 kcal/mol/A is
// representable with 1e-12 resolution.  Energies: 2^32.  PME charge grid:
// int32 at 2^28 (|rho| < 8 e per grid point, resolution 3.7e-9 e).
constexpr double kForceScale = 1099511627776.0;     // 2^40
constexpr double kInvForceScale = 1.0 / 1099511627776.0;
constexpr double kEnergyScale = 4294967296.0;       // 2^32
constexpr double kInvEnergyScale = 1.0 / 4294967296.0;
constexpr float kGridScale = 268435456.0f;          // 2^28
constexpr float kInvGridScale = 1.0f / 268435456.0f;

// Energy term slots of the fixed-point energy accumulator.  Names are the
// keys of ForceManager::getEnergyComponents (src/ForceManager.cu:278-296).
enum EnergyTerm : int {
  kEBond = 0, kEAngle, kEUreyb, kEDihe, kEImdihe,
  kEEwks, kEEwse, kEEwex, kEElec, kEVdw, kNumEnergyTerms
};
static const char *const kEnergyNames[kNumEnergyTerms] = {
    "bond", "angle", "ureyb", "dihe", "imdihe",
    "ewks", "ewse", "ewex", "elec", "vdw"};

// Nonbonded tile geometry: clusters of 32 atoms (one warp).
constexpr int kTile = 32;

// Device-side error word bits (polled by the host after launches).
enum DeviceError : unsigned {
  kErrNone = 0,
  kErrTileOverflow = 1u << 0,     // neighbour tile list larger than allocated
  kErrColumnOverflow = 1u << 1,   // a cell column exceeded the sort capacity
  kErrWorkOverflow = 1u << 2,     // nonbonded work list larger than allocated
  kErrNaN = 1u << 3,              // non-finite coordinates
  kErrCopyTimeout = 1u << 4,      // an asynchronous tensor copy did not complete in time
};

struct CudaError : public std::runtime_error {
  explicit CudaError(const std::string &m) : std::runtime_error(m) {}
};

inline void cuda_check(cudaError_t e, const char *what, const char *file,
                       int line) {
  if (e != cudaSuccess) {
    throw CudaError(std::string("CUDA error '") + cudaGetErrorString(e) +
                    "' in " + what + " at " + file + ":" +
                    std::to_string(line));
  }
}

}  // namespace apo

#define APO_CUDA(x) ::apo::cuda_check((x), #x, __FILE__, __LINE__)
#define APO_LAUNCH_CHECK() \
  ::apo::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)
