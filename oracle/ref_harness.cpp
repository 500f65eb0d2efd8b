// Harness that drives the reference engine's own build (oracle/_ref,
// compiled by oracle/Makefile.ref) through its public C++ API.
//
// TEST / MEASUREMENT INFRASTRUCTURE ONLY: used by the parity tests and the
// reference arm of the benchmark on a machine with a GPU, never by the product.
//
//   ref_harness forces <psf> <prm> <crd> <L> <kappa> <cutnb> <ctonnb> <ctofnb>
//               <nx> <ny> <nz> <order> <out>
//     one energy/force evaluation (CharmmContext::calculatePotentialEnergy);
//     writes the 10 energy terms on the first line and the N gradients.
//   ref_harness md <psf> <prm> <crd> <L> <kappa> <cutnb> <ctonnb> <ctofnb>
//               <nx> <ny> <nz> <order> <warmup> <steps> <seed> <friction>
//               [langevin|leapfrog|nosehoover]
//     dynamics at 300 K, dt 2 fs (Langevin by default, `friction` in 1/ps);
//     prints one JSON line with the time of `steps` steps after `warmup`
//     steps, taken on the host between two device-wide synchronisations.
//   ref_harness relax <psf> <prm> <crd> <L> <kappa> <cutnb> <ctonnb> <ctofnb>
//               <nx> <ny> <nz> <order> <iterations> <max_step> <out>
//     deterministic steepest descent on the reference's forces: each
//     iteration moves every atom along -gradient, the largest move
//     `max_step` Angstrom; writes the final x y z per line.
//   ref_harness traj <psf> <prm> <crd> <L> <kappa> <cutnb> <ctonnb> <ctofnb>
//               <nx> <ny> <nz> <order> <langevin|leapfrog|nosehoover> <steps>
//               <seed> <friction> <velocities> <out>
//     takes the velocities (3N values, A per AKMA time unit) from a text file
//     (CharmmContext::assignVelocities), runs `steps` steps of the named
//     integrator at 300 K with dt 2 fs and writes per atom the FP64 state
//     x y z, the single-precision x y z (the only copy the reference's
//     leapfrog advances) and vx vy vz.
//   ref_harness nblist <psf> <prm> <crd> <L> <kappa> <cutnb> <ctonnb> <ctofnb>
//               <nx> <ny> <nz> <order> <radius> <out>
//     builds the neighbour list (CharmmContext::resetNeighborList) and writes
//     every atom pair of its tiles whose distance (FP64, from the sorted
//     coordinates and the tile's image shift) is below `radius` as int32
//     triples (global i, global j, exclusion bit) to a binary file.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <exception>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "CharmmContext.h"
#include "CharmmCrd.h"
#include "CharmmPSF.h"
#include "CharmmParameters.h"
#include "CudaLangevinPistonIntegrator.h"
#include "CudaLangevinThermostatIntegrator.h"
#include "CudaLeapFrogIntegrator.h"
#include "CudaNeighborList.h"
#include "CudaNoseHooverIntegrator.h"
#include "CudaPMEDirectForce.h"
#include "ForceManager.h"

namespace {

// White-box access to the list the reference's direct-space force builds:
// pointers to protected members, formed in a class derived from the owner,
// applied to the owner's object (no change to the reference's classes).
struct FmPeek : ForceManager {
  static CudaPMEDirectForce<long long int, float> *direct(ForceManager &f) {
    return (f.*(&FmPeek::m_DirectForcePtr)).get();
  }
};
struct DirectPeek : CudaPMEDirectForce<long long int, float> {
  using D = CudaPMEDirectForce<long long int, float>;
  static CudaNeighborList<32> &list(D &d) { return *(d.*(&DirectPeek::neighborList)); }
  static const float4 *sorted(D &d) {
    return (d.*(&DirectPeek::xyzq_sorted)).getDeviceArray().data();
  }
  static const int *l2g(D &d) { return d.*(&DirectPeek::loc2glo); }
};

template <typename T>
std::vector<T> from_device(const T *p, size_t n) {
  std::vector<T> h(n);
  if (n) cudaMemcpy(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost);
  return h;
}

struct Setup {
  std::vector<double4> xyz;
  std::shared_ptr<CharmmParameters> prm;
  std::shared_ptr<CharmmPSF> psf;
  std::shared_ptr<ForceManager> fm;
  std::shared_ptr<CharmmContext> ctx;
};

Setup make(char **a) {
  Setup s;
  s.prm = std::make_shared<CharmmParameters>(std::string(a[1]));
  s.psf = std::make_shared<CharmmPSF>(std::string(a[0]));
  s.fm = std::make_shared<ForceManager>(s.psf, s.prm);
  const double L = std::atof(a[3]);
  s.fm->setBoxDimensions({L, L, L});
  s.fm->setKappa((float)std::atof(a[4]));
  s.fm->setCutoff((float)std::atof(a[5]));
  s.fm->setCtonnb((float)std::atof(a[6]));
  s.fm->setCtofnb((float)std::atof(a[7]));
  s.fm->setFFTGrid(std::atoi(a[8]), std::atoi(a[9]), std::atoi(a[10]));
  s.fm->setPmeSplineOrder(std::atoi(a[11]));
  s.ctx = std::make_shared<CharmmContext>(s.fm);
  auto crd = std::make_shared<CharmmCrd>(std::string(a[2]));
  s.ctx->setCoordinates(crd);
  s.xyz = crd->getCoordinatesD();
  return s;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: ref_harness forces|md ...\n");
    return 2;
  }
  const std::string mode = argv[1];
  if (mode == "forces" && argc == 15) {
    Setup s = make(argv + 2);
    s.ctx->calculatePotentialEnergy(true, false);
    auto e = s.fm->getEnergyComponents();
    const int n = s.ctx->getNumAtoms();
    auto f = s.ctx->getForces();
    std::vector<double> fx(n), fy(n), fz(n);
    cudaMemcpy(fx.data(), f->x(), n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(fy.data(), f->y(), n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(fz.data(), f->z(), n * sizeof(double), cudaMemcpyDeviceToHost);
    FILE *out = std::fopen(argv[14], "w");
    if (!out) return 3;
    for (const char *k : {"bond", "angle", "ureyb", "dihe", "imdihe", "ewks", "ewse", "ewex",
                          "elec", "vdw"})
      std::fprintf(out, "%.12e ", e[k]);
    std::fprintf(out, "\n");
    for (int i = 0; i < n; ++i) std::fprintf(out, "%.12e %.12e %.12e\n", fx[i], fy[i], fz[i]);
    std::fclose(out);
    return 0;
  }
  if (mode == "relax" && argc == 17) {
    Setup s = make(argv + 2);
    const int iters = std::atoi(argv[14]);
    const double max_step = std::atof(argv[15]);
    const int n = s.ctx->getNumAtoms();
    std::vector<double4> x(s.xyz.begin(), s.xyz.begin() + n);
    std::vector<double> gx(n), gy(n), gz(n);
    for (int it = 0; it < iters; ++it) {
      s.ctx->calculatePotentialEnergy(true, false);
      auto f = s.ctx->getForces();
      cudaMemcpy(gx.data(), f->x(), n * sizeof(double), cudaMemcpyDeviceToHost);
      cudaMemcpy(gy.data(), f->y(), n * sizeof(double), cudaMemcpyDeviceToHost);
      cudaMemcpy(gz.data(), f->z(), n * sizeof(double), cudaMemcpyDeviceToHost);
      double gmax = 0.0;
      for (int i = 0; i < n; ++i)
        gmax = std::max(gmax, std::max(std::fabs(gx[i]), std::max(std::fabs(gy[i]), std::fabs(gz[i]))));
      if (!(gmax > 0.0) || !std::isfinite(gmax)) break;
      const double c = max_step / gmax;
      for (int i = 0; i < n; ++i) {
        x[i].x -= c * gx[i];
        x[i].y -= c * gy[i];
        x[i].z -= c * gz[i];
      }
      s.ctx->setCoordinates(x);
    }
    FILE *out = std::fopen(argv[16], "w");
    if (!out) return 3;
    for (int i = 0; i < n; ++i) std::fprintf(out, "%.10f %.10f %.10f\n", x[i].x, x[i].y, x[i].z);
    std::fclose(out);
    return 0;
  }
  if (mode == "md" && (argc == 18 || argc == 19)) {
    Setup s = make(argv + 2);
    const int warmup = std::atoi(argv[14]), steps = std::atoi(argv[15]);
    const unsigned long long seed = std::strtoull(argv[16], nullptr, 10);
    const std::string kind = argc == 19 ? argv[18] : "langevin";
    s.ctx->setRandomSeedForVelocities(seed);
    s.ctx->assignVelocitiesAtTemperature(300.0f);
    std::shared_ptr<CudaIntegrator> integ;
    if (kind == "langevin") {
      auto lg = std::make_shared<CudaLangevinThermostatIntegrator>(0.002);
      lg->setThermostatFriction(std::atof(argv[17]));
      lg->setReferenceTemperature(300.0);
      lg->setThermostatRngSeed(seed);
      integ = lg;
    } else if (kind == "leapfrog") {
      integ = std::make_shared<CudaLeapFrogIntegrator>(0.002);
    } else if (kind == "nosehoover") {
      auto nh = std::make_shared<CudaNoseHooverIntegrator>(0.002);
      nh->setReferenceTemperature(300.0);
      integ = nh;
    } else if (kind == "piston") {
      auto lp = std::make_shared<CudaLangevinPistonIntegrator>(0.002);
      lp->setCrystalType(CRYSTAL::CUBIC);
      lp->setReferenceTemperature(300.0);
      lp->setLangevinPistonFriction(std::atof(argv[17]));
      lp->setLangevinPistonFrictionSeed(seed);
      integ = lp;
    } else {
      std::fprintf(stderr, "unknown integrator %s\n", kind.c_str());
      return 2;
    }
    integ->setCharmmContext(s.ctx);
    integ->propagate(warmup);
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    integ->propagate(steps);
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    const double sec = std::chrono::duration<double>(t1 - t0).count();
    double temp = -1.0;
    try {
      temp = s.ctx->computeTemperature();
    } catch (const std::exception &) {
    }
    std::printf("{\"steps\": %d, \"seconds\": %.6f, \"ns_per_day\": %.4f, "
                "\"integrator\": \"%s\", \"temperature_end\": %.3f}\n",
                steps, sec, 86400.0 * steps / sec * 0.002 * 1e-3, kind.c_str(), temp);
    return 0;
  }
  if (mode == "traj" && argc == 20) {
    Setup s = make(argv + 2);
    const std::string kind = argv[14];
    const int steps = std::atoi(argv[15]);
    const unsigned long long seed = std::strtoull(argv[16], nullptr, 10);
    const double friction = std::atof(argv[17]);
    const int n = s.ctx->getNumAtoms();
    std::vector<double> vel;
    {
      FILE *in = std::fopen(argv[18], "r");
      if (!in) return 3;
      double v;
      while (std::fscanf(in, "%lf", &v) == 1) vel.push_back(v);
      std::fclose(in);
    }
    if ((int)vel.size() != 3 * n) {
      std::fprintf(stderr, "velocity file holds %zu values, expected %d\n", vel.size(), 3 * n);
      return 2;
    }
    s.ctx->assignVelocities(vel);
    std::shared_ptr<CudaIntegrator> integ;
    if (kind == "langevin") {
      auto lg = std::make_shared<CudaLangevinThermostatIntegrator>(0.002);
      lg->setThermostatFriction(friction);
      lg->setReferenceTemperature(300.0);
      lg->setThermostatRngSeed(seed);
      integ = lg;
    } else if (kind == "leapfrog") {
      integ = std::make_shared<CudaLeapFrogIntegrator>(0.002);
    } else if (kind == "nosehoover") {
      auto nh = std::make_shared<CudaNoseHooverIntegrator>(0.002);
      nh->setReferenceTemperature(300.0);
      integ = nh;
    } else if (kind.rfind("piston", 0) == 0) {
      // Langevin piston at 1 atm with its Nose-Hoover thermostat at 300 K
      // ("piston": cubic; "piston_tetra", "piston_ortho": those crystal
      // types; "piston_nonh": cubic without the thermostat); `friction` is
      // the piston's, `seed` its noise seed
      auto lp = std::make_shared<CudaLangevinPistonIntegrator>(0.002);
      lp->setCrystalType(kind == "piston_tetra"   ? CRYSTAL::TETRAGONAL
                         : kind == "piston_ortho" ? CRYSTAL::ORTHORHOMBIC
                                                  : CRYSTAL::CUBIC);
      lp->setReferenceTemperature(300.0);
      lp->setLangevinPistonFriction(friction);
      lp->setLangevinPistonFrictionSeed(seed);
      if (kind == "piston_nonh") lp->useNoseHooverThermostat(false);
      integ = lp;
    } else {
      std::fprintf(stderr, "unknown integrator %s\n", kind.c_str());
      return 2;
    }
    integ->setCharmmContext(s.ctx);
    if (steps > 0) integ->propagate(steps);
    if (kind.rfind("piston", 0) == 0) {
      const std::vector<double> b = s.fm->getBoxDimensions();
      FILE *bf = std::fopen((std::string(argv[19]) + ".box").c_str(), "w");
      if (!bf) return 3;
      std::fprintf(bf, "%.17g %.17g %.17g\n", b[0], b[1], b[2]);
      std::fclose(bf);
    }
    cudaDeviceSynchronize();
    auto x = from_device(s.ctx->getCoordinatesCharges().getDeviceArray().data(), n);
    auto xf = from_device(s.ctx->getXYZQ().getDeviceArray().data(), n);
    auto v = from_device(s.ctx->getVelocityMass().getDeviceArray().data(), n);
    FILE *out = std::fopen(argv[19], "w");
    if (!out) return 3;
    for (int i = 0; i < n; ++i)
      std::fprintf(out, "%.17g %.17g %.17g %.9g %.9g %.9g %.17g %.17g %.17g\n", x[i].x, x[i].y,
                   x[i].z, xf[i].x, xf[i].y, xf[i].z, v[i].x, v[i].y, v[i].z);
    std::fclose(out);
    return 0;
  }
  if (mode == "nblist" && argc == 16) {
    Setup s = make(argv + 2);
    const double radius = std::atof(argv[14]);
    s.ctx->resetNeighborList();
    s.ctx->calculatePotentialEnergy(true, false);
    cudaDeviceSynchronize();
    auto *direct = FmPeek::direct(*s.fm);
    if (!direct) {
      std::fprintf(stderr, "no direct-space force\n");
      return 2;
    }
    auto &nl = DirectPeek::list(*direct);
    auto &b = nl.getBuilder(0);
    const int n = s.ctx->getNumAtoms();
    const int ne = b.get_n_ientry(), nt = b.get_n_tile();
    auto ientry = from_device(b.get_ientry(), ne);
    auto indj = from_device(b.get_tile_indj(), nt);
    auto excl = from_device(b.get_tile_excl(), nt);
    auto xs = from_device(DirectPeek::sorted(*direct), n);
    auto l2g = from_device(DirectPeek::l2g(*direct), n);
    const double L = std::atof(argv[5]);
    const double r2 = radius * radius;
    std::vector<int> out3;
    for (const ientry_t &e : ientry) {
      int ish = e.ish;
      const double shz = (ish / 9 - 1) * L;
      ish -= (ish / 9) * 9;
      const double shy = (ish / 3 - 1) * L;
      ish -= (ish / 3) * 3;
      const double shx = (ish - 1) * L;
      for (int t = e.tileStart; t <= e.tileEnd; ++t) {
        for (int wid = 0; wid < 32; ++wid) {
          const int j = indj[t] + wid;
          if (j >= n) continue;
          const unsigned word = excl[t].excl[wid];
          for (int k = 0; k < 32; ++k) {
            const int i = e.iatomStart + (wid + k) % 32;
            if (i >= n) continue;
            const double dx = (double)xs[i].x + shx - (double)xs[j].x;
            const double dy = (double)xs[i].y + shy - (double)xs[j].y;
            const double dz = (double)xs[i].z + shz - (double)xs[j].z;
            if (dx * dx + dy * dy + dz * dz >= r2) continue;
            out3.push_back(l2g[i]);
            out3.push_back(l2g[j]);
            out3.push_back((int)((word >> k) & 1u));
          }
        }
      }
    }
    FILE *out = std::fopen(argv[15], "wb");
    if (!out) return 3;
    std::fwrite(out3.data(), sizeof(int), out3.size(), out);
    std::fclose(out);
    std::printf("{\"ientries\": %d, \"tiles\": %d, \"pairs\": %zu}\n", ne, nt, out3.size() / 3);
    return 0;
  }
  std::fprintf(stderr, "bad arguments\n");
  return 2;
}
