// CHARMM topology (PSF), parameter (PRM/STR) and coordinate (CRD) readers.
//
// Host-side C++ mirroring the reference's file classes so the C-ABI can take
// the same files:  CharmmPSF (include/CharmmPSF.h, src/CharmmPSF.cu:387-706),
// CharmmParameters (src/CharmmParameters.cu:57-345), CharmmCrd
// (src/CharmmCrd.cu).
#pragma once

#include <array>
#include <map>
#include <set>
#include <string>
#include <tuple>
#include <vector>

namespace apo {

struct Bond { int i, j; };
struct Angle { int i, j, k; };
struct Dihedral { int i, j, k, l; };

class CharmmPSF {
 public:
  CharmmPSF() = default;
  explicit CharmmPSF(const std::string &path);

  int getNumAtoms() const { return (int)m_Charges.size(); }
  int getNumBonds() const { return (int)m_Bonds.size(); }
  int getNumAngles() const { return (int)m_Angles.size(); }
  int getNumDihedrals() const { return (int)m_Dihedrals.size(); }
  int getNumImpropers() const { return (int)m_Impropers.size(); }
  int getNumCrossTerms() const { return m_NumCrossTerms; }
  const std::vector<std::string> &getSegmentIdentifiers() const { return m_Segids; }
  const std::vector<int> &getResidueIdentifiers() const { return m_Resids; }
  const std::vector<std::string> &getResidueNames() const { return m_Resnames; }
  const std::vector<std::string> &getAtomNames() const { return m_AtomNames; }
  const std::vector<std::string> &getAtomTypes() const { return m_AtomTypes; }
  const std::vector<double> &getCharges() const { return m_Charges; }
  const std::vector<double> &getMasses() const { return m_Masses; }
  const std::vector<Bond> &getBonds() const { return m_Bonds; }
  const std::vector<Angle> &getAngles() const { return m_Angles; }
  const std::vector<Dihedral> &getDihedrals() const { return m_Dihedrals; }
  const std::vector<Dihedral> &getImpropers() const { return m_Impropers; }
  double getNetCharge() const;
  double getTotalMass() const;
  const std::string &getFileName() const { return m_FileName; }

  // TIP3 waters: consecutive OT, HT, HT (src/CharmmPSF.cu:281-296)
  std::vector<std::array<int, 3>> getWaterMolecules() const;
  // Bonded components as contiguous [first,last] atom ranges
  // (src/CharmmPSF.cu:302-329)
  std::vector<std::array<int, 2>> getConnectedComponents() const;

  // programmatic construction (used by the batch/serving front-ends)
  void setAtoms(const std::vector<std::string> &types,
                const std::vector<double> &charges,
                const std::vector<double> &masses);
  std::vector<Bond> &bonds() { return m_Bonds; }
  std::vector<Angle> &angles() { return m_Angles; }
  std::vector<Dihedral> &dihedrals() { return m_Dihedrals; }
  std::vector<Dihedral> &impropers() { return m_Impropers; }

 private:
  std::string m_FileName;
  std::vector<std::string> m_Segids, m_Resnames, m_AtomNames, m_AtomTypes;
  std::vector<int> m_Resids;
  std::vector<double> m_Charges, m_Masses;
  std::vector<Bond> m_Bonds;
  std::vector<Angle> m_Angles;
  std::vector<Dihedral> m_Dihedrals, m_Impropers;
  int m_NumCrossTerms = 0;
};

struct BondParam { float kb, b0; };
struct AngleParam { float ktheta, theta0; };       // theta0 in radians
struct DihedralTerm { float k; int n; float delta; };  // delta in degrees
struct ImproperParam { float kpsi, psi0; };        // psi0 in degrees
struct VdwParam { double eps, rmin2; };            // eps as written (<0)
struct NbfixParam { double emin, rmin, emin14, rmin14; };

using Key2 = std::pair<std::string, std::string>;
using Key3 = std::tuple<std::string, std::string, std::string>;
using Key4 = std::tuple<std::string, std::string, std::string, std::string>;

class CharmmParameters {
 public:
  CharmmParameters() = default;
  explicit CharmmParameters(const std::string &path);
  explicit CharmmParameters(const std::vector<std::string> &paths);
  void read(const std::string &path);

  std::map<std::string, double> masses;
  std::map<Key2, BondParam> bonds;
  std::map<Key3, AngleParam> angles;
  std::map<Key3, BondParam> ureyb;
  std::map<Key4, std::vector<DihedralTerm>> dihedrals;
  std::map<Key4, ImproperParam> impropers;
  std::map<std::string, VdwParam> vdw, vdw14;
  std::map<Key2, NbfixParam> nbfix;
};

class CharmmCrd {
 public:
  CharmmCrd() = default;
  explicit CharmmCrd(const std::string &path);
  int getNumAtoms() const { return (int)m_Xyz.size() / 3; }
  const std::vector<double> &getCoordinates() const { return m_Xyz; }
  std::vector<double> &coordinates() { return m_Xyz; }

 private:
  std::vector<double> m_Xyz;
};

}  // namespace apo
