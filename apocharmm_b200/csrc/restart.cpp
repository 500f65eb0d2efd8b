// Restart file writer and reader; see restart.h.
#include "restart.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace apo {

namespace {
constexpr int kWidth = 22;
constexpr int kVersion = 50;
constexpr int kLenEnp = 60, kLenEnt = 128, kLenEnv = 50;  // CHARMM energy table sizes

std::string pad_left(const std::string &s, int w) {
  return (int)s.size() >= w ? s : std::string(w - s.size(), ' ') + s;
}

// mantissa and exponent of the %.{digits-1}E form
void sci_parts(double v, int digits, std::string &mant, int &expo) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.*E", digits - 1, v);
  std::string s(buf);
  const size_t e = s.find('E');
  mant = s.substr(0, e);
  expo = std::atoi(s.c_str() + e + 1);
}

std::string with_exponent(const std::string &mant, int expo, bool compact) {
  char buf[16];
  if (compact) std::snprintf(buf, sizeof(buf), "D%d", expo);
  else std::snprintf(buf, sizeof(buf), "D%c%02d", expo < 0 ? '-' : '+', expo < 0 ? -expo : expo);
  return mant + buf;
}

std::string line_of(std::initializer_list<double> vals) {
  std::string s;
  for (double v : vals) s += restartDouble(v);
  return s + "\n";
}

bool getline_checked(std::istream &in, std::string &line) {
  if (!std::getline(in, line)) return false;
  if (!line.empty() && line.back() == '\r') line.pop_back();
  return true;
}

void find_section(std::istream &in, const std::string &title, const std::string &path) {
  std::string line;
  while (getline_checked(in, line))
    if (line == title) return;
  throw std::runtime_error("Could not find " + title.substr(1) + " section in restart file \"" +
                           path + "\"");
}

std::string field(const std::string &line, size_t pos, size_t len, const std::string &what) {
  if (line.size() < pos + 1) throw std::runtime_error("restart file: line too short for " + what);
  return line.substr(pos, len);
}

long long parse_int(const std::string &s, const std::string &what) {
  char *end = nullptr;
  const long long v = std::strtoll(s.c_str(), &end, 10);
  while (end && *end == ' ') ++end;
  if (end == s.c_str() || (end && *end)) throw std::runtime_error("restart file: bad " + what);
  return v;
}

void read_triples(std::istream &in, int n, std::vector<double> &out, const std::string &what) {
  out.resize((size_t)3 * n);
  std::string line;
  for (int i = 0; i < n; ++i) {
    if (!getline_checked(in, line))
      throw std::runtime_error("restart file: " + what + " section ends early");
    for (int d = 0; d < 3; ++d)
      out[(size_t)3 * i + d] = parseRestartDouble(field(line, (size_t)kWidth * d, kWidth, what));
  }
}
}  // namespace

std::string restartDouble(double v) {
  if (!std::isfinite(v)) throw std::invalid_argument("restart file: non-finite value");
  std::string mant;
  int expo = 0;
  sci_parts(v, 17, mant, expo);
  std::string s = with_exponent(mant, expo, false);
  if ((int)s.size() > kWidth) s = with_exponent(mant, expo, true);
  for (int digits = 16; (int)s.size() > kWidth && digits > 1; --digits) {
    sci_parts(v, digits, mant, expo);
    s = with_exponent(mant, expo, false);
  }
  return pad_left(s, kWidth);
}

double parseRestartDouble(const std::string &f) {
  std::string s = f;
  for (char &c : s)
    if (c == 'D' || c == 'd') c = 'e';
  char *end = nullptr;
  const double v = std::strtod(s.c_str(), &end);
  while (end && *end == ' ') ++end;
  if (end == s.c_str() || (end && *end))
    throw std::runtime_error("restart file: cannot read a number from \"" + f + "\"");
  return v;
}

void writeRestartFile(const std::string &path, const RestartRecord &r) {
  if ((int)r.xold.size() != 3 * r.natom || (int)r.vel.size() != 3 * r.natom ||
      (int)r.delta.size() != 3 * r.natom)
    throw std::invalid_argument("restart file: per-atom arrays must hold 3 x NATOM values");
  std::ostringstream o;
  const auto &b = r.box;
  std::string crystal = r.crystal;
  if (crystal.empty())
    crystal = (b[0] == b[1] && b[0] == b[2]) ? "CUBI" : (b[0] == b[1] ? "TETR" : "ORTH");
  if (crystal.size() != 4) throw std::invalid_argument("restart file: crystal tag must have 4 characters");
  o << "REST" << pad_left(std::to_string(kVersion), 6) << pad_left("1", 6) << "  " << crystal
    << "  " << "    " << "  " << "APO" << "\n\n";
  o << pad_left("2", 8) << " !NTITLE followed by title\n";
  o << "* APOCHARMM RESTART FILE\n";
  o << "* USED FOR CONTINUING MOLECULAR DYNAMICS TRAJECTORY\n\n";
  o << " !CRYSTAL PARAMETERS\n";
  o << line_of({b[0], 0.0, b[1]}) << line_of({0.0, 0.0, b[2]});
  o << line_of({r.hdot[0], r.hdot[1], r.hdot[2]}) << line_of({0.0, 0.0, 0.0});  // HDOT
  o << line_of({0.0, r.pnhv, r.pnhf});                              // PNH, PNHV, PNHF
  for (int k = 0; k < 8; ++k) o << line_of({0.0, 0.0, 0.0});        // UC1A..UC2B
  o << line_of({0.0, 0.0, 0.0}) << line_of({0.0}) << "\n";          // GRAD1A..GRAD2B
  o << " !NATOM,NPRIV,NSTEP,NSAVC,NSAVV,JHSTRT,NDEGF,SEED,NSAVL\n";
  o << pad_left(std::to_string(r.natom), 12) << pad_left(std::to_string(r.npriv), 12)
    << pad_left(std::to_string(r.nstep), 12) << pad_left(std::to_string(r.nsavc), 12)
    << pad_left("0", 12) << pad_left("0", 12) << pad_left(std::to_string(r.ndegf), 12)
    << pad_left(std::to_string(r.seed), 22) << "  ";
  if (r.has_rng) o << r.rngpos;
  o << "\n\n";
  o << " !ENERGIES and STATISTICS\n";
  o << std::string(kLenEnp, 'T') << "\n" << std::string(kLenEnt, 'T') << "\n";
  o << pad_left("0", 8) << restartDouble(0.0) << restartDouble(0.0) << restartDouble(r.avetem)
    << "\n";
  const std::string z3 = line_of({0.0, 0.0, 0.0}), z2 = line_of({0.0, 0.0});
  for (int i = 0; i < kLenEnp; ++i) o << z3;
  for (int i = 0; i < kLenEnp; ++i) o << z2;
  for (int i = 0; i < kLenEnt; ++i) o << z3;
  for (int i = 0; i < kLenEnt; ++i) o << z2;
  for (int i = 0; i < kLenEnv; ++i) o << z3;
  for (int i = 0; i < kLenEnv; ++i) o << z2;
  o << "\n";
  auto triples = [&](const char *title, const std::vector<double> &v) {
    o << title << "\n";
    for (int i = 0; i < r.natom; ++i)
      o << restartDouble(v[3 * (size_t)i]) << restartDouble(v[3 * (size_t)i + 1])
        << restartDouble(v[3 * (size_t)i + 2]) << "\n";
  };
  triples(" !XOLD, YOLD, ZOLD", r.xold);
  o << "\n";
  triples(" !VX, VY, VZ", r.vel);
  o << "\n";
  triples(" !X, Y, Z", r.delta);
  // the whole file is rewritten at every report, as the reference does
  std::ofstream f(path, std::ios::out | std::ios::trunc);
  if (!f) throw std::runtime_error("Could not open restart file \"" + path + "\" for writing");
  const std::string s = o.str();
  f.write(s.data(), (std::streamsize)s.size());
  if (!f) throw std::runtime_error("Could not write restart file \"" + path + "\"");
}

RestartRecord readRestartFile(const std::string &path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("Could not open file \"" + path + "\"");
  RestartRecord r;
  std::string line;
  if (!getline_checked(in, line) || line.compare(0, 4, "REST") != 0)
    throw std::runtime_error("\"" + path + "\" is not a restart file");
  r.apo = line.size() >= 33 && line.substr(30, 3) == "APO";
  if (line.size() >= 22) r.crystal = line.substr(18, 4);
  find_section(in, " !CRYSTAL PARAMETERS", path);
  std::vector<std::string> cry(5);
  for (auto &l : cry)
    if (!getline_checked(in, l)) throw std::runtime_error("restart file: crystal block ends early");
  r.box[0] = parseRestartDouble(field(cry[0], 0, kWidth, "XTLABC"));
  r.box[1] = parseRestartDouble(field(cry[0], 44, kWidth, "XTLABC"));
  r.box[2] = parseRestartDouble(field(cry[1], 44, kWidth, "XTLABC"));
  for (int k = 0; k < 3; ++k) r.hdot[k] = parseRestartDouble(field(cry[2], k * kWidth, kWidth, "HDOT"));
  r.pnhv = parseRestartDouble(field(cry[4], 22, kWidth, "PNHV"));
  r.pnhf = parseRestartDouble(field(cry[4], 44, kWidth, "PNHF"));
  find_section(in, " !NATOM,NPRIV,NSTEP,NSAVC,NSAVV,JHSTRT,NDEGF,SEED,NSAVL", path);
  if (!getline_checked(in, line)) throw std::runtime_error("restart file: NATOM line missing");
  r.natom = (int)parse_int(field(line, 0, 12, "NATOM"), "NATOM");
  r.npriv = parse_int(field(line, 12, 12, "NPRIV"), "NPRIV");
  r.nstep = parse_int(field(line, 24, 12, "NSTEP"), "NSTEP");
  r.nsavc = (int)parse_int(field(line, 36, 12, "NSAVC"), "NSAVC");
  r.ndegf = (int)parse_int(field(line, 72, 12, "NDEGF"), "NDEGF");
  r.seed = (uint64_t)std::strtoull(field(line, 84, 22, "SEED").c_str(), nullptr, 10);
  if (r.natom < 0) throw std::runtime_error("restart file: negative NATOM");
  if (line.size() > 106) {
    const std::string rest = line.substr(106);
    if (rest.find_first_not_of(' ') != std::string::npos) {
      r.rngpos = (unsigned long long)parse_int(rest, "RNG position");
      r.has_rng = true;
    }
  }
  find_section(in, " !ENERGIES and STATISTICS", path);
  for (int k = 0; k < 3; ++k)
    if (!getline_checked(in, line)) throw std::runtime_error("restart file: statistics end early");
  r.avetem = parseRestartDouble(field(line, 8 + 2 * kWidth, kWidth, "AVETEM"));
  find_section(in, " !XOLD, YOLD, ZOLD", path);
  read_triples(in, r.natom, r.xold, "XOLD");
  find_section(in, " !VX, VY, VZ", path);
  read_triples(in, r.natom, r.vel, "VX");
  find_section(in, " !X, Y, Z", path);
  read_triples(in, r.natom, r.delta, "X");
  return r;
}

}  // namespace apo
