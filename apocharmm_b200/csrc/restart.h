// CHARMM-style restart files as apoCHARMM writes and reads them.
//
// Layout of the reference writer src/RestartSubscriber.cu:39-445: header
// "REST" + version 50 + crystal tag + "APO" at column 30, a two-line title,
// " !CRYSTAL PARAMETERS" (lower-triangle cell, HDOT, Nose-Hoover piston
// PNH/PNHV/PNHF, the UC and GRAD blocks), " !NATOM,NPRIV,NSTEP,NSAVC,NSAVV,
// JHSTRT,NDEGF,SEED,NSAVL" (seven 12-wide integers, the 22-wide thermostat
// seed, then the RNG sequence position), " !ENERGIES and STATISTICS", and
// the per-atom sections " !XOLD, YOLD, ZOLD" (current coordinates),
// " !VX, VY, VZ" (velocities) and " !X, Y, Z" (the position-Verlet delta of
// the last step).  Real numbers sit in 22-character columns read back by
// column (src/CudaLangevinThermostatIntegrator.cu:307-316, 446-500).
//
// The reference prints 16 significant digits, which does not give back the
// same double.  This writer prints 17 significant digits wherever they fit
// in the 22 columns (every value whose exponent has one digit, every
// non-negative value with a two-digit exponent), dropping the exponent's
// "+" sign and leading zero for negative values ("-1.2345678901234567D-3");
// both the reference's reader (replace D by e, std::stod) and Fortran D
// editing read that form.  Only a negative value with a two-digit negative
// exponent (|x| < 1e-9) falls back to 16 digits.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace apo {

struct RestartRecord {
  std::array<double, 3> box{};       // orthorhombic cell edges (A)
  // crystal tag of the header ("CUBI", "TETR", "ORTH"); empty: from the box
  // edges when writing, as the reference does for its thermostats
  std::string crystal;
  std::array<double, 3> hdot{};      // Langevin piston displacement (HDOT)
  double pnhv = 0.0, pnhf = 0.0;     // Nose-Hoover piston velocity and force
  int natom = 0;
  long long npriv = 0;               // steps taken since the run began
  long long nstep = 0;               // steps of the run that wrote the file
  int nsavc = 0;                     // report frequency of the writer
  int ndegf = 0;
  uint64_t seed = 0;                 // Langevin thermostat or piston seed
  bool has_rng = false;              // RNG position present (Langevin thermostat or piston)
  unsigned long long rngpos = 0;     // Philox sequence position
  double avetem = 0.0;               // running average temperature
  bool apo = true;                   // header carries the "APO" tag
  std::vector<double> xold, vel, delta;  // natom x 3 each
};

// one value in the 22-column form described above
std::string restartDouble(double v);
double parseRestartDouble(const std::string &field);

void writeRestartFile(const std::string &path, const RestartRecord &r);
RestartRecord readRestartFile(const std::string &path);

}  // namespace apo
