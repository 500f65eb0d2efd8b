// Subscribers; see subscribers.h.
#include "subscribers.h"

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "common.h"
#include "engine.h"
#include "integrators.h"
#include "restart.h"

namespace apo {

Subscriber::Subscriber(int f) { setReportFrequency(f); }

void Subscriber::setReportFrequency(int f) {
  if (f <= 0) throw std::invalid_argument("report frequency must be positive");
  m_Freq = f;
}

DcdSubscriber::DcdSubscriber(const std::string &path, int f) : Subscriber(f), m_Path(path) {
  m_File = std::fopen(path.c_str(), "wb");
  if (!m_File) throw std::invalid_argument("Cannot open DCD file " + path);
}

DcdSubscriber::~DcdSubscriber() {
  if (m_File) std::fclose(m_File);
}

namespace {
void record(std::FILE *f, const void *data, int32_t bytes) {
  std::fwrite(&bytes, 4, 1, f);
  std::fwrite(data, 1, (size_t)bytes, f);
  std::fwrite(&bytes, 4, 1, f);
}
}  // namespace

void DcdSubscriber::writeHeader(int natom, long long step, double dtPs) {
  char hdr[84];
  std::memset(hdr, 0, sizeof(hdr));
  std::memcpy(hdr, "CORD", 4);
  int32_t *ic = reinterpret_cast<int32_t *>(hdr + 4);
  ic[0] = m_Frames;              // NSET, rewritten after every frame
  ic[1] = (int32_t)step;         // ISTART
  ic[2] = m_Freq;                // NSAVC
  ic[3] = m_Freq * std::max(1, m_Frames);
  float delta = (float)(dtPs / kTimfac);  // AKMA units
  std::memcpy(&ic[9], &delta, 4);
  ic[10] = 1;                    // unit cell present
  ic[19] = 24;                   // CHARMM version tag
  std::fseek(m_File, 0, SEEK_SET);
  record(m_File, hdr, 84);
  char title[4 + 80];
  int32_t ntitle = 1;
  std::memcpy(title, &ntitle, 4);
  std::memset(title + 4, ' ', 80);
  const char *t = "* TRAJECTORY WRITTEN BY THE B200 ENGINE";
  std::memcpy(title + 4, t, std::strlen(t));
  record(m_File, title, 84);
  int32_t n = natom;
  record(m_File, &n, 4);
}

void DcdSubscriber::update(CharmmContext &ctx, long long step, double dtPs) {
  const int n = ctx.getNumAtoms();
  auto xyz = ctx.getCoordinates();
  if (m_Frames == 0) writeHeader(n, step, dtPs);
  std::fseek(m_File, 0, SEEK_END);
  auto box = ctx.getForceManager()->getBoxDimensions();
  double cell[6] = {box[0], 90.0, box[1], 90.0, 90.0, box[2]};
  record(m_File, cell, 48);
  std::vector<float> c(n);
  for (int d = 0; d < 3; ++d) {
    for (int i = 0; i < n; ++i) c[i] = (float)xyz[3 * i + d];
    record(m_File, c.data(), 4 * n);
  }
  ++m_Frames;
  writeHeader(n, step - (long long)(m_Frames - 1) * m_Freq, dtPs);
  std::fflush(m_File);
}

RestartSubscriber::RestartSubscriber(const std::string &path, int f)
    : Subscriber(f), m_Path(path) {
  // fail at creation, not at the first report, when the path is unusable
  std::FILE *t = std::fopen(path.c_str(), "a");
  if (!t) throw std::invalid_argument("Cannot open restart file " + path);
  std::fclose(t);
}

void RestartSubscriber::update(CharmmContext &, long long, double) {
  if (!m_Integrator) throw std::runtime_error("RestartSubscriber: not subscribed to an integrator");
  RestartRecord r = m_Integrator->restartRecord();
  r.nsavc = m_Freq;
  writeRestartFile(m_Path, r);
  ++m_Writes;
}

}  // namespace apo
