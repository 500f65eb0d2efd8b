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
#include "CudaLangevinThermostatIntegrator.h"
#include "CudaLeapFrogIntegrator.h"
#include "CudaNoseHooverIntegrator.h"
#include "ForceManager.h"

namespace {

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
  std::fprintf(stderr, "bad arguments\n");
  return 2;
}
