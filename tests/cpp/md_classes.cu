// Drives a Langevin run through the C++ context, integrator and subscriber
// classes (include/apocharmm/CharmmContext.h, CudaIntegrator.h) the way the
// reference's C++ drivers do, and writes the end state for the test to
// compare with the same run made through the Python API:
//   md_classes PSF PRM CRD BOX KAPPA CUTNB CTONNB CTOFNB NX NY NZ ORDER NSTEPS OUTDIR
// Writes OUTDIR/{coords,velocities,forces}.bin (float64, atom-major),
// OUTDIR/traj.dcd, OUTDIR/run.rst and OUTDIR/results.txt.
#include <cstdio>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "apocharmm/CharmmContext.h"
#include "apocharmm/CudaIntegrator.h"

namespace {

void save(const std::string &path, const std::vector<double> &v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char *>(v.data()), v.size() * sizeof(double));
}

std::vector<double> flatten(const std::vector<std::vector<double>> &a) {
  std::vector<double> out;
  out.reserve(3 * a.size());
  for (auto &r : a) out.insert(out.end(), r.begin(), r.end());
  return out;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 15) {
    std::fprintf(stderr,
                 "usage: %s PSF PRM CRD BOX KAPPA CUTNB CTONNB CTOFNB NX NY NZ ORDER NSTEPS OUT\n",
                 argv[0]);
    return 2;
  }
  const std::string out = argv[14];
  const double box = std::stod(argv[4]);
  const int nsteps = std::stoi(argv[13]);
  try {
    auto psf = std::make_shared<CharmmPSF>(argv[1]);
    auto prm = std::make_shared<CharmmParameters>(std::vector<std::string>{argv[2]});
    auto fm = std::make_shared<ForceManager>(psf, prm);
    fm->setBoxDimensions({box, box, box});
    fm->setKappa(std::stof(argv[5]));
    fm->setCutoff(std::stof(argv[6]));
    fm->setCtonnb(std::stof(argv[7]));
    fm->setCtofnb(std::stof(argv[8]));
    fm->setFFTGrid(std::stoi(argv[9]), std::stoi(argv[10]), std::stoi(argv[11]));
    fm->setPmeSplineOrder(std::stoi(argv[12]));

    auto ctx = std::make_shared<CharmmContext>(fm);
    auto crd = std::make_shared<CharmmCrd>(argv[3]);
    ctx->setCoordinates(crd);
    ctx->setRandomSeedForVelocities(314159);
    ctx->assignVelocitiesAtTemperature(300.0f);

    std::ofstream res(out + "/results.txt");
    res.precision(17);
    res << "crd_atoms " << crd->getNumAtoms() << " " << ctx->getNumAtoms() << "\n";
    res << "ndegf " << ctx->getDegreesOfFreedom() << "\n";

    auto integrator = std::make_shared<CudaLangevinThermostatIntegrator>(0.002);
    integrator->setThermostatFriction(5.0);
    integrator->setReferenceTemperature(300.0);
    integrator->setThermostatRngSeed(1234);
    integrator->setCharmmContext(ctx);
    auto dcd = std::make_shared<DcdSubscriber>(out + "/traj.dcd", 10);
    auto rst = std::make_shared<RestartSubscriber>(out + "/run.rst", nsteps);
    auto spare = std::make_shared<DcdSubscriber>(out + "/spare.dcd");
    integrator->subscribe({dcd, rst, spare});
    spare->setReportFrequency(5);
    res << "report_frequency " << dcd->getReportFrequency() << " " << rst->getReportFrequency() << " "
        << spare->getReportFrequency() << "\n";
    integrator->unsubscribe(spare);
    res << "subscribers " << integrator->getSubscribers().size() << "\n";
    integrator->propagate(nsteps);

    res << "step " << integrator->getCurrentPropagatedStep() << "\n";
    res << "rngpos " << integrator->getRngSequencePos() << "\n";
    res << "temperature " << ctx->computeTemperature() << "\n";
    save(out + "/coords.bin", flatten(ctx->getCoordinates()));
    save(out + "/velocities.bin", ctx->getVelocities());

    ctx->calculatePotentialEnergy(true, false);
    for (auto &kv : ctx->getEnergyComponents()) res << "energy " << kv.first << " " << kv.second << "\n";
    res << "epot " << ctx->getPotentialEnergies() << "\n";
    save(out + "/forces.bin", ctx->getForces()->getXYZ());

    // the same context driven on by a second integrator kind
    CudaLeapFrogIntegrator leap(0.001);
    leap.setCharmmContext(ctx);
    leap.propagate(5);
    res << "leapfrog_step " << leap.getCurrentPropagatedStep() << "\n";

    // and at constant pressure (cubic Langevin piston, 1 atm)
    CudaLangevinPistonIntegrator piston(0.001);
    piston.setCrystalType(CRYSTAL::CUBIC);
    piston.setReferenceTemperature(300.0);
    piston.setLangevinPistonFriction(10.0);
    piston.setLangevinPistonFrictionSeed(5);
    piston.setCharmmContext(ctx);
    piston.propagate(5);
    const auto b = ctx->getBoxDimensions();
    res << "piston_box " << b[0] << " " << b[1] << " " << b[2] << "\n";
    res << "piston_pressure " << piston.getInstantaneousPressureScalar() << " "
        << piston.getLangevinPistonMass().size() << " " << piston.getRngSequencePos() << "\n";
    res << "done\n";
  } catch (const std::exception &ex) {
    std::fprintf(stderr, "error: %s\n", ex.what());
    return 1;
  }
  return 0;
}
