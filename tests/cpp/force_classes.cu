// Drives the C++ class surface (include/apocharmm/) the way a user of the
// reference's C++ classes would, and writes what it computed for the test
// to compare:
//   force_classes PSF PRM XYZQ.bin BOX KAPPA CUTNB CTONNB CTOFNB NX NY NZ ORDER OUTDIR
// XYZQ.bin: float32 (x, y, z, q) per atom.  Writes OUTDIR/<name>.bin
// (float64 atom-major gradients) and OUTDIR/results.txt (energies, counts).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "apocharmm/CudaBondedForce.h"
#include "apocharmm/CudaNeighborList.h"
#include "apocharmm/CudaPMEDirectForce.h"
#include "apocharmm/CudaPMEReciprocalForce.h"
#include "apocharmm/ForceManager.h"

namespace {

// E = k sum_i |r_i|^2 on the float coordinates the manager hands over:
// gradient 2 k r_i in 2^40 fixed point, energy into the first term
__global__ void well_kernel(int n, const float4 *xyzq, double k, long long *f, int stride,
                            double *energy) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = xyzq[i];
  const double g[3] = {2.0 * k * p.x, 2.0 * k * p.y, 2.0 * k * p.z};
  for (int d = 0; d < 3; ++d) f[d * stride + i] = llrint(g[d] * 1099511627776.0);
  atomicAdd(energy, k * ((double)p.x * p.x + (double)p.y * p.y + (double)p.z * p.z));
}

// a user-defined force with the ForceView members
class WellForce {
 public:
  WellForce(double k, cudaStream_t s) : m_K(k), m_S(s) {
    m_Ev = std::make_shared<CudaEnergyVirial>();
    m_Ev->insert("well");
  }
  void initialize(int numAtoms, const std::vector<double> &) {
    m_F = std::make_shared<Force<long long int>>(numAtoms);
    m_N = numAtoms;
    ++initialized;
  }
  void clear() {
    m_F->clear(m_S);
    m_Ev->clear(m_S);
  }
  void calcForce(const float4 *xyzq, bool, bool) {
    well_kernel<<<(m_N + 127) / 128, 128, 0, m_S>>>(m_N, xyzq, m_K, m_F->xyz(), m_F->stride(),
                                                   m_Ev->getEnergyPointer("well"));
    ++calls;
  }
  void setBoxDimensions(const std::vector<double> &) {}
  std::shared_ptr<Force<long long int>> getForce() { return m_F; }
  std::shared_ptr<CudaEnergyVirial> getEnergyVirial() { return m_Ev; }
  int initialized = 0, calls = 0;

 private:
  double m_K;
  cudaStream_t m_S;
  int m_N = 0;
  std::shared_ptr<Force<long long int>> m_F;
  std::shared_ptr<CudaEnergyVirial> m_Ev;
};

void save(const std::string &path, const std::vector<double> &v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char *>(v.data()), v.size() * sizeof(double));
}

std::vector<double> from_fixed(Force<long long int> &f) {
  auto v = f.getXYZ();
  std::vector<double> out(v.size());
  for (size_t k = 0; k < v.size(); ++k) out[k] = (double)v[k] / 1099511627776.0;
  return out;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 14) {
    std::fprintf(stderr, "usage: %s PSF PRM XYZQ BOX KAPPA CUTNB CTONNB CTOFNB NX NY NZ ORDER OUT\n",
                 argv[0]);
    return 2;
  }
  const std::string out = argv[13];
  const double box = std::stod(argv[4]);
  try {
    auto psf = std::make_shared<CharmmPSF>(argv[1]);
    auto prm = std::make_shared<CharmmParameters>(std::vector<std::string>{argv[2]});
    const int n = psf->getNumAtoms();
    std::vector<float> h(4 * (size_t)n);
    {
      std::ifstream f(argv[3], std::ios::binary);
      f.read(reinterpret_cast<char *>(h.data()), h.size() * sizeof(float));
      if (!f) throw std::runtime_error("short coordinate file");
    }
    float4 *d_xyzq = nullptr;
    apocharmm_detail::cuda_check(cudaMalloc(&d_xyzq, (size_t)n * sizeof(float4)), "malloc");
    apocharmm_detail::cuda_check(
        cudaMemcpy(d_xyzq, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice), "copy");

    auto fm = std::make_shared<ForceManager>(psf, prm);
    fm->setBoxDimensions({box, box, box});
    fm->setKappa(std::stof(argv[5]));
    fm->setCutoff(std::stof(argv[6]));
    fm->setCtonnb(std::stof(argv[7]));
    fm->setCtofnb(std::stof(argv[8]));
    fm->setFFTGrid(std::stoi(argv[9]), std::stoi(argv[10]), std::stoi(argv[11]));
    fm->setPmeSplineOrder(std::stoi(argv[12]));
    fm->initialize();

    std::ofstream res(out + "/results.txt");
    res.precision(17);

    // the whole force field: calcForce(xyzq, reset, calcEnergy, calcVirial)
    fm->calcForce(d_xyzq, true, true, true);
    save(out + "/total.bin", fm->getForces()->getXYZ());
    for (auto &kv : fm->getEnergyComponents()) res << "total " << kv.first << " " << kv.second << "\n";
    auto w = fm->getVirial();
    res << "virial";
    for (double x : w) res << " " << x;
    res << "\n";

    // the three parts as force objects
    CudaBondedForce<long long int, float> bonded(fm);
    CudaPMEDirectForce<long long int, float> direct(fm);
    CudaPMEReciprocalForce recip(fm);
    bonded.calc_force(d_xyzq, true, false);
    direct.calc_force(d_xyzq, true, false);
    recip.calc_force(d_xyzq, true, false);
    save(out + "/bonded.bin", from_fixed(*bonded.getForce()));
    save(out + "/direct.bin", from_fixed(*direct.getForce()));
    save(out + "/recip.bin", from_fixed(*recip.getForce()));
    for (auto *p : {static_cast<ForcePart *>(&bonded), static_cast<ForcePart *>(&direct),
                    static_cast<ForcePart *>(&recip)}) {
      auto ev = p->getEnergyVirial();
      for (auto &name : ev->getNames())
        res << "part " << p->getComponents() << " " << name << " " << ev->getEnergy(name) << "\n";
    }

    // the tile list
    CudaNeighborList<32> nl(fm);
    nl.build(d_xyzq);
    res << "list " << nl.getNumList() << " " << nl.getNumSlots() << " " << nl.getNumTiles() << " "
        << nl.getNumWorkItems() << "\n";
    std::vector<int> glo2loc(n), perm(nl.getNumSlots());
    apocharmm_detail::cuda_check(cudaMemcpy(glo2loc.data(), nl.get_glo2loc(), n * sizeof(int),
                                            cudaMemcpyDeviceToHost), "copy");
    apocharmm_detail::cuda_check(cudaMemcpy(perm.data(), nl.get_ind_sorted(),
                                            perm.size() * sizeof(int), cudaMemcpyDeviceToHost),
                                 "copy");
    int roundtrip = 1;
    for (int i = 0; i < n; ++i)
      if (glo2loc[i] < 0 || glo2loc[i] >= (int)perm.size() || perm[glo2loc[i]] != i) roundtrip = 0;
    res << "glo2loc_roundtrip " << roundtrip << "\n";
    auto pairs = nl.getPairs(std::stod(argv[8]));
    size_t excluded = 0;
    for (auto &p : pairs) excluded += p[2];
    res << "pairs " << pairs.size() << " " << excluded << "\n";

    // a user force through ForceView, on a stream of its own
    auto fstream = std::shared_ptr<cudaStream_t>(new cudaStream_t(nullptr), [](cudaStream_t *s) {
      if (*s) cudaStreamDestroy(*s);
      delete s;
    });
    apocharmm_detail::cuda_check(cudaStreamCreateWithFlags(fstream.get(), cudaStreamNonBlocking),
                                 "stream");
    auto well = std::make_shared<WellForce>(0.05, *fstream);
    fm->subscribe(well, "well", fstream, well->getForce(), well->getEnergyVirial());
    fm->calcForce(d_xyzq, false, true, false);
    save(out + "/with_well.bin", fm->getForces()->getXYZ());
    auto e = fm->getEnergyComponents();
    res << "well_energy " << e["well"] << "\n";
    res << "well_calls " << well->initialized << " " << well->calls << "\n";
    fm->unsubscribe("well");
    fm->calcForce(d_xyzq, false, true, false);
    save(out + "/after_unsubscribe.bin", fm->getForces()->getXYZ());
    e = fm->getEnergyComponents();
    res << "after_unsubscribe_has_well " << (int)e.count("well") << "\n";

    // an error raised by the library reaches the caller as an exception
    int threw = 0;
    try {
      fm->setCutoff((float)box);  // above half the box edge
      fm->initialize();
    } catch (const std::invalid_argument &) {
      threw = 1;
    } catch (const std::runtime_error &) {
      threw = 2;
    }
    res << "bad_cutoff_exception " << threw << "\n";
    cudaFree(d_xyzq);
    res << "done\n";
  } catch (const std::exception &ex) {
    std::fprintf(stderr, "error: %s\n", ex.what());
    return 1;
  }
  return 0;
}
