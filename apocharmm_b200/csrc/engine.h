// ForceManager and CharmmContext: the host orchestration of one system.
//
// Mirrors the reference's classes of the same names (include/ForceManager.h:115-694,
// include/CharmmContext.h:36-469) for the P1 / VDW_VFSW / EWALD path:
// same setters, defaults (kappa 0.34, cutnb 14, ctonnb 12, ctofnb 10, spline
// order 4, FFT grid 2*floor(L/2)), energy-term names, gradient sign and
// exceptions on bad input.  Differences by design:
//   * one int64 fixed-point gradient buffer in neighbour-list slot order is
//     shared by the bonded, reciprocal and direct parts (the reference keeps
//     three and adds them into a fourth on the host's command);
//   * energies are 64-bit fixed-point sums, so the total is order-free;
//   * a force evaluation issues no host synchronisation, so it can be
//     captured in a CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "bonded.h"
#include "charmm_io.h"
#include "common.h"
#include "force_plugins.h"
#include "nblist.h"
#include "nonbonded.h"
#include "pme.h"
#include "topology.h"

namespace apo {

enum class PBC { P1 = 0, P21 = 1 };
enum VdwModel { VDW_VSH = 1, VDW_VSW = 2, VDW_VFSW = 3, VDW_VGSH = 4, VDW_CUT = 5 };

template <typename T>
struct DeviceArray {
  T *p = nullptr;
  size_t n = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray &) = delete;
  DeviceArray &operator=(const DeviceArray &) = delete;
  ~DeviceArray() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    reset();
    n = count;
    if (count) APO_CUDA(cudaMalloc(&p, count * sizeof(T)));
  }
  void upload(const std::vector<T> &v) {
    alloc(v.size());
    if (!v.empty())
      APO_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  }
  std::vector<T> download() const {
    std::vector<T> v(n);
    if (n) APO_CUDA(cudaMemcpy(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost));
    return v;
  }
};

// One system of a multi-system force manager (replicas, lambda windows, or
// unrelated molecules advanced together): its files, box and nonbonded/PME
// settings.  All systems of one manager share the spline order, the
// precision form and the tiles per work item.
struct SystemSpec {
  std::shared_ptr<CharmmPSF> psf;
  std::shared_ptr<CharmmParameters> prm;
  std::array<double, 3> box{{0.0, 0.0, 0.0}};
  double kappa = 0.34, cutnb = 14.0, ctonnb = 12.0, ctofnb = 10.0;
  std::array<int, 3> nfft{{-1, -1, -1}};  // -1: 2 floor(L/2)
  uint64_t seed = 0;                      // velocities and Langevin noise of this system
  // the system's topology built beforehand from psf and prm (build_topology),
  // or null to build it during initialisation
  std::shared_ptr<const Topology> topology;
};

class ForceManager {
 public:
  ForceManager(std::shared_ptr<CharmmPSF> psf, std::shared_ptr<CharmmParameters> prm);
  // several independent systems, concatenated in order, evaluated with one
  // launch per stage; initialised on construction
  explicit ForceManager(const std::vector<SystemSpec> &systems, int order = 4,
                        int tilesPerWork = 8, bool precise = false);
  ~ForceManager();
  bool isMulti() const { return m_Multi; }
  int numSystems() const { return m_Multi ? (int)m_Specs.size() : 1; }
  const std::vector<SystemSpec> &systemSpecs() const { return m_Specs; }
  // first atom of every system and the total (numSystems() + 1 entries)
  const std::vector<int> &atomOffsets() const { return m_AtomOff; }
  const std::vector<Topology> &systemTopologies() const { return m_SysTop; }
  // device: atom -> system, per-system box (x, y, z, 0)
  const int *sysOfAtom() { return m_Nbl.sys_of_atom; }
  const double4 *systemBoxes() const { return m_Boxes.p; }
  // energies of one system (multi-system managers)
  std::map<std::string, double> getEnergyComponents(int sys, cudaStream_t s);
  std::vector<double> getVirial(int sys, cudaStream_t s);

  void setBoxDimensions(const std::array<double, 3> &box);
  // a box that changes every step (pressure control, one system): the
  // direct-space set-up, the list's box and the reciprocal box follow it
  // without a new initialisation; the list is rebuilt at the next
  // evaluation and graphs captured with the old box are dropped.  The
  // caller has synchronised the context's stream.
  void updateBoxDimensions(const std::array<double, 3> &box);
  // device-resident box (one system): PME and image centering read the box
  // from deviceBox(), so kernels that change the box on the device (the
  // Langevin piston) need no host round trip; they write deviceBox(), the
  // direct-space set-up (deviceSetup()) and the list's dims (deviceListDims())
  void useDeviceBox();
  bool hasDeviceBox() const { return m_DevBox.p != nullptr; }
  double4 *deviceBox() { return m_DevBox.p; }
  NbSetup *deviceSetup() { return m_Setup.p; }
  NbSysDims *deviceListDims() { return m_Nbl.device_dims(); }
  // the host copies of a box the device already holds (after such kernels)
  void adoptDeviceBox(const std::array<double, 3> &box);
  void setKappa(double k) { m_Kappa = k; m_Initialized = false; }
  void setCutoff(double c) { m_Cutoff = c; m_Initialized = false; }
  void setCtonnb(double c) { m_Ctonnb = c; m_Initialized = false; }
  void setCtofnb(double c) { m_Ctofnb = c; m_Initialized = false; }
  void setFFTGrid(int nx, int ny, int nz);
  void setPmeSplineOrder(int order) { m_Order = order; m_Initialized = false; }
  void setVdwType(int type);
  void setPeriodicBoundaryCondition(PBC pbc);
  // precision form: per-pair fixed-point accumulation, FP64 influence function
  void setPrecisionMode(bool precise) { m_Precise = precise; }
  bool getPrecisionMode() const { return m_Precise; }
  void setTilesPerWork(int t) { m_TilesPerWork = t; m_Initialized = false; }
  // work items a warp of the direct-space kernel takes before it retires
  // (0: persistent grid, every warp until the list is done)
  void setWorkItemsPerWarp(int k) { m_ItemsPerWarp = k < 0 ? 0 : k; }
  int getWorkItemsPerWarp() const { return m_ItemsPerWarp; }
  // direct-space kernel form (kNbTileBatches or kNbGroupedQueues, nonbonded.h)
  void setDirectKernel(int v);
  int getDirectKernel() const { return m_NbVariant; }
  // evaluated parts: 1 bonded (with the 1-4 pairs and exclusion corrections
  // unless kComponent14WithDirect is set), 2 direct space, 4 reciprocal space
  void setComponentMask(int mask) { m_ComponentMask = mask; }
  int getComponentMask() const { return m_ComponentMask; }
  // the 1-4 pairs and the exclusion corrections go with the direct space, as
  // the reference splits CudaBondedForce and CudaPMEDirectForce
  static constexpr int kComponent14WithDirect = 8;
  // extra force terms evaluated with every force call, their energies
  // reported under `tag` (ForceManager::subscribe/unsubscribe,
  // include/ForceManager.h:420-475); one system only
  void subscribe(std::shared_ptr<ForcePlugin> force, const std::string &tag);
  bool unsubscribe(const std::string &tag);
  bool unsubscribe(const ForcePlugin *force);
  // changes whenever the set of plug-ins or a device buffer the force path
  // reads changes (captured graphs are then stale)
  int pluginGeneration() const { return m_PluginGen; }
  // tile capacity of the neighbour list (work items follow); a list that
  // outgrows it during propagate() is grown and the segment run again
  void setListCapacity(int tiles);
  int getListCapacity() const { return m_Nbl.dims().tile_cap; }
  // after a device-side list overflow: rebuild the list at the current
  // coordinates with capacities that hold it, clear the error word (sync);
  // true when the buffers moved
  bool growNeighborList(const float4 *d_xyzq, cudaStream_t s);
  // z-pencil slabs moved by tiled tensor copies (default) or by plain loads
  void setPmeTensorCopies(bool on);
  bool getPmeTensorCopies() const { return m_Pme.tensor_copies(); }
  // calcForce with clear = true, then a synchronisation; a list that
  // overflowed on the way is grown and the forces evaluated again
  void calcForceChecked(const float4 *d_xyzq, bool calcEnergy, bool calcVirial, cudaStream_t s);
  static constexpr int kMaxPlugins = 16;

  const std::array<double, 3> &getBoxDimensions() const { return m_Box; }
  double getKappa() const { return m_Kappa; }
  double getCutoff() const { return m_Cutoff; }
  double getCtonnb() const { return m_Ctonnb; }
  double getCtofnb() const { return m_Ctofnb; }
  std::array<int, 3> getFFTGrid() const { return {m_Nfft[0], m_Nfft[1], m_Nfft[2]}; }
  int getPmeSplineOrder() const { return m_Order; }
  int getNumAtoms() const { return m_Multi ? m_Top.natom : m_Psf->getNumAtoms(); }
  bool isInitialized() const { return m_Initialized; }
  bool isListBuilt() const { return m_ListBuilt; }
  std::shared_ptr<CharmmPSF> getPsf() const { return m_Psf; }
  const Topology &topology() const { return m_Top; }
  std::array<int, 3> computeFFTGridSize() const;

  void initialize();
  // image-wrapped rebuild of the tile list from global-order coordinates
  void resetNeighborList(const float4 *d_xyzq, cudaStream_t s);
  // gradients into the slot-order fixed-point buffer (cleared first unless
  // clear == false); energies into the fixed-point energy slots
  void calcForce(const float4 *d_xyzq, bool calcEnergy, bool calcVirial, cudaStream_t s,
                 bool clear = true);
  // FP64 state coordinates (x, y, z, q) in atom order, read by the bonded
  // terms; set by the CharmmContext that owns them
  void setStateCoordinates(const double4 *c) {
    m_StateCoords = c;
    m_Nbl.set_state_coordinates(c);
  }
  // The reference's ForceManager::calcForce(xyzq, reset, calcEnergy,
  // calcVirial) (include/ForceManager.h:424, src/ForceManager.cu:821) on
  // caller-owned single-precision coordinates and charges (device float4,
  // atom order): the FP64 state the kernels read is formed from them, the
  // list is rebuilt when `reset` (or when none exists yet), and `components`
  // selects the parts as setComponentMask does, for this call only.
  void calcForceXyzq(const float4 *d_xyzq, bool reset, bool calcEnergy, bool calcVirial,
                     int components, cudaStream_t s);

  std::map<std::string, double> getEnergyComponents(cudaStream_t s);
  double getPotentialEnergy(cudaStream_t s);
  // internal virial of the last evaluation made with calcVirial, row-major
  // 3x3 (kcal/mol): W = -sum r (x) dU/dr over direct, reciprocal, bonded,
  // 1-4 and exclusion terms (ForceManager::getVirial, src/ForceManager.cu:393)
  std::vector<double> getVirial(cudaStream_t s);
  // total gradient, global atom order, (N,3) row-major
  void getForces(std::vector<double> &out, cudaStream_t s);
  // the same into a caller's device buffer of x/y/z planes `stride` apart,
  // in FP64 or in the 2^40 fixed point it is summed in (stream-ordered on s)
  void getForcesDevice(double *d_out, int stride, cudaStream_t s);
  void getForceFixedDevice(long long *d_out, int stride, cudaStream_t s);

  // device state used by the integrators
  long long *forceFixed() const { return m_Force.p; }
  int forceStride() const { return m_Stride; }
  long long *energyFixed() const { return m_Energy.p; }
  NeighborList &neighborList() { return m_Nbl; }
  Pme &pme() { return m_Pme; }
  // the virial slots of the last evaluation made with calcVirial (3x3 row
  // major, 2^32 fixed point; one system)
  const long long *deviceVirial() const { return m_Energy.p + kNumEnergyTerms; }
  double selfEnergy() const { return m_SelfEnergy; }
  unsigned readDeviceError(cudaStream_t s);
  // CUDA-event timing of every direct-space launch (on the stream it runs
  // on); events of a captured graph are replayed with the graph, so the
  // cursor is rewound at the start of every integration segment
  void setKernelTiming(bool on);
  void rewindKernelTimers() { m_TimerCursor = 0; }
  // sum (ms) over the launches recorded since the last rewind
  double kernelTimeMs(int &launches);

 private:
  void initializeMulti();
  void createStreams();
  std::shared_ptr<CharmmPSF> m_Psf;
  std::shared_ptr<CharmmParameters> m_Prm;
  bool m_Multi = false;
  std::vector<SystemSpec> m_Specs;
  std::vector<Topology> m_SysTop;
  std::vector<int> m_AtomOff;
  std::vector<double> m_SelfEnergies;
  int m_EStride = 0;  // energy slots per system (energies + virial)
  PmeMulti m_PmeMulti;
  DeviceArray<double4> m_Boxes;
  DeviceArray<double4> m_DevBox;  // one system's box in device memory (useDeviceBox)
  std::array<double, 3> m_Box{{-9999.9999, -9999.9999, -9999.9999}};
  double m_Kappa = 0.34, m_Cutoff = 14.0, m_Ctonnb = 12.0, m_Ctofnb = 10.0;
  int m_Nfft[3] = {-1, -1, -1};
  int m_Order = 4;
  int m_VdwType = VDW_VFSW;
  bool m_VirialValid = false;
  bool m_Precise = false;
  bool m_Initialized = false;
  bool m_ListBuilt = false;
  bool m_ListDirty = false;  // buffers replaced: rebuild before the next use
  bool m_PmeTensorCopies = true;
  int m_TilesPerWork = 8;
  int m_ItemsPerWarp = 0;
  int m_NbVariant = kNbTileBatches;
  int m_ComponentMask = 7;
  int m_EvalMask = 7;  // parts of the last evaluation
  double m_SelfEnergy = 0.0;
  const double4 *m_StateCoords = nullptr;
  DeviceArray<double4> m_XyzqState;  // FP64 state formed by calcForceXyzq
  std::vector<std::pair<std::string, std::shared_ptr<ForcePlugin>>> m_Plugins;
  DeviceArray<long long> m_PluginEnergy;  // kMaxPlugins fixed-point slots
  int m_PluginGen = 0;
  Topology m_Top;

  NeighborList m_Nbl;
  Pme m_Pme;
  int m_Stride = 0;
  DeviceArray<long long> m_Force, m_Energy;
  DeviceArray<int> m_VdwTypeD;
  DeviceArray<float2> m_Vdw, m_Vdw14;
  DeviceArray<NbSetup> m_Setup;
  NbSetup m_HostSetup{};
  DeviceArray<int2> m_BondIJ, m_UbIJ, m_In14, m_Ex14, m_DiheTerms;
  DeviceArray<float2> m_BondP, m_UbP, m_AngleP, m_ImpP;
  DeviceArray<int4> m_AngleIJK, m_DiheIJKL, m_ImpIJKL;
  DeviceArray<float4> m_DiheCoef;
  DeviceArray<double> m_Scratch;
  bool m_Timing = false;
  int m_TimerCursor = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> m_Timers;
  cudaStream_t m_SNb = nullptr, m_SPme = nullptr, m_SBond = nullptr;
  cudaEvent_t m_EvFork = nullptr, m_EvNb = nullptr, m_EvPme = nullptr, m_EvBond = nullptr;
};

class CharmmContext {
 public:
  explicit CharmmContext(std::shared_ptr<ForceManager> fm);
  ~CharmmContext();

  void setCoordinates(const std::vector<double> &xyz);
  void setCoordinates(const CharmmCrd &crd) { setCoordinates(crd.getCoordinates()); }
  std::vector<double> getCoordinates();
  void setVelocities(const std::vector<double> &v);
  std::vector<double> getVelocities();
  // the same four transfers on a caller's x,y,z-interleaved host array of
  // 3N doubles (pinned memory gives full-bandwidth copies): one copy
  // through a device staging array and one pack/unpack kernel each
  // (first, count) restricts a transfer to an atom range (one system of a
  // multi-system context); count < 0 means to the last atom
  // rebuild = false: the list is marked stale and rebuilt before the next
  // force evaluation (lets several systems be loaded before the first build)
  void setCoordinatesXyz(const double *xyz, int first = 0, int count = -1, bool rebuild = true);
  void getCoordinatesXyz(double *xyz, int first = 0, int count = -1);
  void setVelocitiesXyz(const double *v, int first = 0, int count = -1);
  void getVelocitiesXyz(double *v, int first = 0, int count = -1);
  // device-resident copy of an atom range's state: coordinates (x, y, z,
  // charge) then velocities (with the mass term), 2 x count double4 at dst,
  // and back; stream-ordered on the context's stream (a load marks the list
  // stale and refreshes the single-precision coordinates)
  void saveStateDevice(double4 *dst, int first, int count);
  void loadStateDevice(const double4 *src, int first, int count);
  void setRandomSeedForVelocities(uint64_t seed) { m_Seed = seed; }
  void assignVelocitiesAtTemperature(double temperature);
  void useHolonomicConstraints(bool flag);
  bool isUsingHolonomicConstraints() const { return m_Holonomic; }
  int getDegreesOfFreedom() const { return m_Ndegf; }
  // per system (one entry for a single-system context)
  const std::vector<int> &systemDegreesOfFreedom() const { return m_SysNdegf; }
  // instantaneous temperature of every system from the on-step velocities
  std::vector<double> systemTemperatures();
  int getNumAtoms() const { return m_N; }
  double computeTemperature();
  double getKineticEnergy();

  void imageCentering(cudaStream_t s);
  void resetNeighborList(cudaStream_t s);
  // rebuild now (synchronously usable, outside any capture) if the list was
  // never built or coordinates were loaded without a rebuild
  void ensureNeighborList();
  // the list's buffers exist (the first build sizes them, synchronously); a
  // list that is merely stale is left for the caller's next rebuild
  void ensureListBuffers();
  void calculateForces(bool reset, bool calcEnergy, bool calcVirial);
  double calculatePotentialEnergy(bool reset, bool print);

  std::shared_ptr<ForceManager> getForceManager() const { return m_Fm; }
  cudaStream_t stream() const { return m_Stream; }
  // device state: coordinates+charge (double4), velocity + inverse mass
  // (double4), single-precision coordinates+charge in atom order (float4)
  double4 *coords() const { return m_Coords.p; }
  double4 *velMass() const { return m_VelMass.p; }
  float4 *xyzq() const { return m_Xyzq.p; }
  const int2 *groups() const { return m_Groups.p; }
  int numGroups() const { return (int)m_Groups.n; }

 private:
  std::shared_ptr<ForceManager> m_Fm;
  int m_N = 0;
  uint64_t m_Seed = 0;
  bool m_Holonomic = true;
  int m_Ndegf = 0;
  std::vector<int> m_SysNdegf;
  DeviceArray<long long> m_SysKe;
  bool m_HasCoords = false;
  bool m_ListStale = false;
  cudaStream_t m_Stream = nullptr;
  DeviceArray<double4> m_Coords, m_VelMass;
  DeviceArray<float4> m_Xyzq;
  DeviceArray<double> m_Stage;    // 3N doubles: host transfers
  DeviceArray<int> m_BadAtom;     // first non-finite coordinate, or INT_MAX
  DeviceArray<int2> m_Groups;
  int m_NumBigGroups = 0;  // leading components taken by a warp each
};

// device helpers shared with the integrators
// groups: bonded components (first, last atom), the nbig components of more
// than kSmallComponent atoms first (order_components sorts them so)
void launch_image_centering(double4 *coords, float4 *xyzq, const int2 *groups, int ngroups,
                            int nbig, double Lx, double Ly, double Lz, cudaStream_t s,
                            const int *sys_of_atom = nullptr, const double4 *boxes = nullptr);
// stable reorder: components of more than `small` atoms first; returns their count
int order_components(std::vector<int2> &groups, int small);
void launch_coords_to_xyzq(const double4 *coords, float4 *xyzq, int n, cudaStream_t s);

}  // namespace apo
