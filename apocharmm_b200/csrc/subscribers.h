// Reporting subscribers called by CudaIntegrator::propagate every
// `reportFrequency` steps (reference: include/Subscriber.h:76,
// src/CudaIntegrator.cu:347-355, src/DcdSubscriber.cu,
// src/RestartSubscriber.cu).
#pragma once

#include <cstdio>
#include <memory>
#include <string>

namespace apo {

class CharmmContext;
class CudaIntegrator;

class Subscriber {
 public:
  explicit Subscriber(int reportFrequency = 1000);
  virtual ~Subscriber() = default;
  int getReportFrequency() const { return m_Freq; }
  void setReportFrequency(int f);
  virtual void update(CharmmContext &ctx, long long step, double timeStepPs) = 0;
  // the integrator that reports to this subscriber (set by subscribe())
  void attach(CudaIntegrator *it) { m_Integrator = it; }

 protected:
  int m_Freq;
  CudaIntegrator *m_Integrator = nullptr;
};

// CHARMM/X-PLOR DCD trajectory: single-precision frames with the unit cell
class DcdSubscriber : public Subscriber {
 public:
  explicit DcdSubscriber(const std::string &path, int reportFrequency = 1000);
  ~DcdSubscriber() override;
  void update(CharmmContext &ctx, long long step, double timeStepPs) override;
  int numFrames() const { return m_Frames; }

 private:
  void writeHeader(int natom, long long step, double dtPs);
  std::string m_Path;
  std::FILE *m_File = nullptr;
  int m_Frames = 0;
};

// restart file rewritten at every report (layout in restart.h); needs a
// Langevin thermostat or Nose-Hoover integrator
class RestartSubscriber : public Subscriber {
 public:
  explicit RestartSubscriber(const std::string &path, int reportFrequency = 1000);
  void update(CharmmContext &ctx, long long step, double timeStepPs) override;
  int numWrites() const { return m_Writes; }

 private:
  std::string m_Path;
  int m_Writes = 0;
};

}  // namespace apo
