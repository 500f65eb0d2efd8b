// CHARMM file readers; see charmm_io.h.
#include "charmm_io.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <numeric>
#include <sstream>
#include <stdexcept>

namespace apo {
namespace {

std::vector<std::string> split_ws(const std::string &s) {
  std::vector<std::string> out;
  std::istringstream ss(s);
  std::string t;
  while (ss >> t) out.push_back(t);
  return out;
}

std::string upper(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

std::string strip_comment(const std::string &line) {
  auto p = line.find('!');
  std::string s = p == std::string::npos ? line : line.substr(0, p);
  auto b = s.find_first_not_of(" \t\r\n");
  if (b == std::string::npos) return "";
  auto e = s.find_last_not_of(" \t\r\n");
  return s.substr(b, e - b + 1);
}

std::vector<std::string> read_lines(const std::string &path) {
  std::ifstream f(path);
  if (!f.is_open()) throw std::invalid_argument("Cannot open file " + path);
  std::vector<std::string> lines;
  std::string l;
  while (std::getline(f, l)) lines.push_back(l);
  return lines;
}

// Canonical key orders used by the reference's lookup
// (src/CharmmParameters.cu:135-233, :378-600).
Key2 key2(std::string a, std::string b) {
  if (a > b) std::swap(a, b);
  return {a, b};
}
Key3 key3(std::string a, const std::string &b, std::string c) {
  if (a > c) std::swap(a, c);
  return {a, b, c};
}
Key4 key4(std::string a, std::string b, std::string c, std::string d) {
  if (a > d) {
    std::swap(a, d);
    std::swap(b, c);
  } else if (a == d && b > c) {
    std::swap(b, c);
  }
  return {a, b, c, d};
}

}  // namespace

// ---------------------------------------------------------------- PSF ------

CharmmPSF::CharmmPSF(const std::string &path) : m_FileName(path) {
  auto lines = read_lines(path);
  size_t p = 0;
  auto find_section = [&](const std::string &tag, bool required) -> long long {
    for (; p < lines.size(); ++p) {
      auto t = split_ws(lines[p]);
      if (t.size() >= 2 && t[1] == tag) {
        ++p;
        return std::stoll(t[0]);
      }
    }
    if (required)
      throw std::runtime_error("Could not find " + tag + " section in PSF \"" +
                               path + "\"");
    return -1;
  };
  long long ntitle = find_section("!NTITLE", true);
  p += (size_t)ntitle;
  long long natom = find_section("!NATOM", true);
  for (long long i = 0; i < natom; ++i, ++p) {
    if (p >= lines.size()) throw std::runtime_error("PSF truncated in atoms");
    auto t = split_ws(lines[p]);
    if (t.size() < 8) throw std::runtime_error("Malformed PSF atom line: " + lines[p]);
    m_Segids.push_back(t[1]);
    m_Resids.push_back(std::stoi(t[2]));
    m_Resnames.push_back(t[3]);
    m_AtomNames.push_back(t[4]);
    m_AtomTypes.push_back(t[5]);
    m_Charges.push_back(std::stod(t[6]));
    m_Masses.push_back(std::stod(t[7]));
  }
  auto read_ints = [&](long long count, int width) {
    std::vector<int> v;
    v.reserve((size_t)(count * width));
    while ((long long)v.size() < count * width && p < lines.size()) {
      for (auto &s : split_ws(lines[p])) v.push_back(std::stoi(s) - 1);
      ++p;
    }
    if ((long long)v.size() < count * width)
      throw std::runtime_error("PSF truncated in connectivity");
    return v;
  };
  long long nb = find_section("!NBOND:", true);
  auto vb = read_ints(nb, 2);
  for (long long i = 0; i < nb; ++i) m_Bonds.push_back({vb[2 * i], vb[2 * i + 1]});
  long long na = find_section("!NTHETA:", true);
  auto va = read_ints(na, 3);
  for (long long i = 0; i < na; ++i)
    m_Angles.push_back({va[3 * i], va[3 * i + 1], va[3 * i + 2]});
  long long nd = find_section("!NPHI:", true);
  auto vd = read_ints(nd, 4);
  for (long long i = 0; i < nd; ++i)
    m_Dihedrals.push_back({vd[4 * i], vd[4 * i + 1], vd[4 * i + 2], vd[4 * i + 3]});
  long long ni = find_section("!NIMPHI:", true);
  auto vi = read_ints(ni, 4);
  for (long long i = 0; i < ni; ++i)
    m_Impropers.push_back({vi[4 * i], vi[4 * i + 1], vi[4 * i + 2], vi[4 * i + 3]});
  long long nc = find_section("!NCRTERM:", false);
  m_NumCrossTerms = nc > 0 ? (int)nc : 0;
  for (auto &b : m_Bonds)
    if (b.i < 0 || b.j < 0 || b.i >= natom || b.j >= natom)
      throw std::runtime_error("PSF bond atom index out of range");
}

void CharmmPSF::setAtoms(const std::vector<std::string> &types,
                         const std::vector<double> &charges,
                         const std::vector<double> &masses) {
  size_t n = types.size();
  if (charges.size() != n || masses.size() != n)
    throw std::invalid_argument("setAtoms: inconsistent array lengths");
  m_AtomTypes = types;
  m_Charges = charges;
  m_Masses = masses;
  m_Segids.assign(n, "SYS");
  m_Resnames.assign(n, "UNK");
  m_AtomNames = types;
  m_Resids.resize(n);
  std::iota(m_Resids.begin(), m_Resids.end(), 1);
}

double CharmmPSF::getNetCharge() const {
  return std::accumulate(m_Charges.begin(), m_Charges.end(), 0.0);
}
double CharmmPSF::getTotalMass() const {
  return std::accumulate(m_Masses.begin(), m_Masses.end(), 0.0);
}

std::vector<std::array<int, 3>> CharmmPSF::getWaterMolecules() const {
  std::vector<std::array<int, 3>> w;
  int n = getNumAtoms();
  for (int i = 0; i + 2 < n; ++i) {
    if (m_AtomTypes[i] == "OT" && m_AtomTypes[i + 1] == "HT" &&
        m_AtomTypes[i + 2] == "HT") {
      w.push_back({i, i + 1, i + 2});
      i += 2;
    }
  }
  return w;
}

std::vector<std::array<int, 2>> CharmmPSF::getConnectedComponents() const {
  int n = getNumAtoms();
  std::vector<int> link(n);
  std::iota(link.begin(), link.end(), 0);
  auto find = [&](int x) {
    while (x != link[x]) x = link[x];
    return x;
  };
  for (auto &b : m_Bonds) {
    int r1 = find(b.i), r2 = find(b.j);
    if (r1 != r2) {
      if (r1 > r2) link[r2] = r1;
      else link[r1] = r2;
    }
  }
  std::vector<std::array<int, 2>> g;
  int s = 0;
  while (s < n) {
    int e = find(s);
    g.push_back({s, e});
    s = e + 1;
  }
  return g;
}

// ---------------------------------------------------------------- PRM ------

CharmmParameters::CharmmParameters(const std::string &path) { read(path); }
CharmmParameters::CharmmParameters(const std::vector<std::string> &paths) {
  for (auto &p : paths) read(p);
}

void CharmmParameters::read(const std::string &path) {
  auto lines = read_lines(path);
  enum class S { NONE, ATOMS, BONDS, ANGLES, DIHEDRALS, IMPROPERS, CMAP, NONBONDED, NBFIX, HBOND, RTF };
  S state = S::NONE;
  // A stream file carries a topology block first ("read rtf card"); the
  // parameters start after "read para".  Files without such lines are plain
  // parameter files.
  bool has_read_para = false;
  for (auto &l0 : lines) {
    auto l = upper(strip_comment(l0));
    if (l.find("READ") != std::string::npos && l.find("PARA") != std::string::npos)
      has_read_para = true;
  }
  if (has_read_para) state = S::RTF;
  for (size_t p = 0; p < lines.size(); ++p) {
    std::string line = upper(strip_comment(lines[p]));
    if (line.empty() || line[0] == '*') continue;
    if (state == S::RTF) {
      if (line.find("READ") != std::string::npos && line.find("PARA") != std::string::npos)
        state = S::NONE;
      continue;
    }
    auto tok = split_ws(line);
    const std::string &h = tok[0];
    if (h.rfind("ATOM", 0) == 0 && tok.size() == 1) { state = S::ATOMS; continue; }
    const bool alone = tok.size() == 1;
    if (alone && h.rfind("BOND", 0) == 0) { state = S::BONDS; continue; }
    if (alone && (h.rfind("ANGL", 0) == 0 || h.rfind("THET", 0) == 0)) { state = S::ANGLES; continue; }
    if (alone && (h.rfind("DIHE", 0) == 0 || h == "PHI")) { state = S::DIHEDRALS; continue; }
    if (alone && (h.rfind("IMPR", 0) == 0 || h.rfind("IMPH", 0) == 0)) { state = S::IMPROPERS; continue; }
    if (alone && h.rfind("CMAP", 0) == 0) { state = S::CMAP; continue; }
    if (h.rfind("NONB", 0) == 0 || h.rfind("NBON", 0) == 0) {
      state = S::NONBONDED;
      // option line, possibly continued with a trailing '-'
      while (!tok.empty() && tok.back() == "-" && p + 1 < lines.size()) {
        ++p;
        tok = split_ws(upper(strip_comment(lines[p])));
      }
      continue;
    }
    if (alone && h.rfind("NBFI", 0) == 0) { state = S::NBFIX; continue; }
    if (h.rfind("HBON", 0) == 0) { state = S::HBOND; continue; }
    if (h == "END") { state = S::NONE; continue; }
    if (h == "RETURN") break;
    try {
      switch (state) {
        case S::ATOMS:
          if (h == "MASS" && tok.size() >= 4) masses[tok[2]] = std::stod(tok[3]);
          break;
        case S::BONDS:
          if (tok.size() >= 4)
            bonds[key2(tok[0], tok[1])] = {std::stof(tok[2]), std::stof(tok[3])};
          break;
        case S::ANGLES:
          if (tok.size() >= 5) {
            auto k = key3(tok[0], tok[1], tok[2]);
            angles[k] = {std::stof(tok[3]),
                         (float)(std::stod(tok[4]) * M_PI / 180.0)};
            if (tok.size() >= 7)
              ureyb[k] = {std::stof(tok[5]), std::stof(tok[6])};
            else
              ureyb[k] = {0.0f, 0.0f};
          }
          break;
        case S::DIHEDRALS:
          if (tok.size() >= 7)
            dihedrals[key4(tok[0], tok[1], tok[2], tok[3])].push_back(
                {std::stof(tok[4]), std::stoi(tok[5]), std::stof(tok[6])});
          break;
        case S::IMPROPERS:
          if (tok.size() >= 7)
            impropers[key4(tok[0], tok[1], tok[2], tok[3])] = {std::stof(tok[4]),
                                                              std::stof(tok[6])};
          break;
        case S::NONBONDED:
          if (tok.size() == 4) {
            vdw[tok[0]] = {std::stod(tok[2]), std::stod(tok[3])};
          } else if (tok.size() == 7) {
            vdw[tok[0]] = {std::stod(tok[2]), std::stod(tok[3])};
            vdw14[tok[0]] = {std::stod(tok[5]), std::stod(tok[6])};
          } else {
            throw std::invalid_argument("Extra tokens in line " + line);
          }
          break;
        case S::NBFIX:
          if (tok.size() >= 4) {
            NbfixParam f;
            f.emin = std::fabs(std::stod(tok[2]));
            f.rmin = std::stod(tok[3]);
            f.emin14 = f.emin;
            f.rmin14 = f.rmin;
            if (tok.size() >= 6) {
              f.emin14 = std::fabs(std::stod(tok[4]));
              f.rmin14 = std::stod(tok[5]);
            }
            nbfix[key2(tok[0], tok[1])] = f;
          }
          break;
        default:
          break;
      }
    } catch (const std::invalid_argument &e) {
      throw std::invalid_argument(std::string("Parameter file ") + path +
                                  ": cannot parse line '" + line + "'");
    }
  }
}

// ---------------------------------------------------------------- CRD ------

CharmmCrd::CharmmCrd(const std::string &path) {
  auto lines = read_lines(path);
  size_t p = 0;
  while (p < lines.size() && !lines[p].empty() && lines[p][0] == '*') ++p;
  if (p >= lines.size()) throw std::runtime_error("Malformed CRD file " + path);
  auto t = split_ws(lines[p]);
  long long n = std::stoll(t[0]);
  bool ext = t.size() >= 2 && upper(t[1]) == "EXT";
  ++p;
  m_Xyz.resize((size_t)(3 * n));
  for (long long i = 0; i < n; ++i, ++p) {
    if (p >= lines.size()) throw std::runtime_error("CRD file truncated: " + path);
    const std::string &l = lines[p];
    size_t o = ext ? 40 : 20, w = ext ? 20 : 10;
    if (l.size() < o + 3 * w - 1) throw std::runtime_error("Malformed CRD line: " + l);
    for (int d = 0; d < 3; ++d) m_Xyz[3 * i + d] = std::stod(l.substr(o + d * w, w));
  }
}

}  // namespace apo
