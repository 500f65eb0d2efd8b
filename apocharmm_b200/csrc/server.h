// Request server with continuous batching.
//
// Clients submit MD-segment requests (a system, its coordinates, a step
// count and a seed) and energy/force requests.  A preparation thread builds
// each request's topology from its PSF and parameters as it arrives; a
// worker thread owns the GPU and advances every admitted MD request
// together in one batch (batch.h), 20 steps (one list-update segment, one
// CUDA graph) at a time.  Between segments it admits prepared requests
// while their estimated device memory fits a fraction of the free HBM
// measured at start, and drops finished ones; when the set changes the
// batch is re-formed from the prepared topologies, and every continuing
// system carries its coordinates, velocities and position-Verlet delta
// over device to device (through a compact device buffer, so the old and
// the new batch never coexist) together with its noise position.  A system
// therefore follows the same trajectory alone and among any others: its
// segments always start at its own steps 0, 20, 40, ..., and a system whose
// step count ends inside a segment is held still (not advanced) for the
// rest of it, and for as long afterwards as it stays in the batch: done
// members leave at the next re-formation, which comes with the next
// admission or once they hold 30 % of the batch's atoms.  Energy/force
// requests join the batch at its next re-formation, are evaluated by one
// force call of the whole batch at their own coordinates, and are then done
// members like finished MD requests.
//
// No counterpart in the reference (it has no serving layer); the physics
// is the reference's per-system force/step path.
#pragma once

#include <array>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"

namespace apo {

struct ServeRequest {
  int kind = 0;                 // 0: MD segment, 1: energy and forces
  SystemSpec spec;
  std::vector<double> xyz;      // initial coordinates, N x 3
  long long steps = 0;          // MD segment length
};

struct ServeResult {
  int kind = 0;
  int status = 0;               // 0 pending, 1 done, 2 failed
  std::string error;
  std::vector<double> xyz, vel, forces;
  std::array<double, kNumEnergyTerms> energy{};
  double latency_s = 0.0;       // submission -> result
};

struct ServerStats {
  long long md_steps = 0;       // system-steps advanced
  double sim_ps = 0.0;          // simulated time over all requests
  long long rebuilds = 0;       // batch re-formations
  long long segments = 0;
  int max_active = 0;
  double busy_s = 0.0;          // time the worker spent on GPU work
  double reform_s = 0.0;        // of which re-forming the batch
  long long energy_evals = 0;   // force calls made for energy/force requests
};

class Server {
 public:
  // hbm_fraction: share of the free device memory (measured at start) that
  // admitted requests may occupy
  Server(double hbm_fraction, int order, bool precise, double dtPs, double frictionPerPs,
         double temperature, uint64_t seed);
  ~Server();
  int submit(ServeRequest r);
  // copies the result out when it is finished (returns false while pending)
  bool poll(int id, ServeResult *out);
  bool wait(int id, double timeout_s, ServeResult *out);
  void release(int id);
  ServerStats stats();
  void stop();
  static double bytesPerAtom() { return 1536.0; }  // admission estimate

 private:
  struct Job {
    int id;
    ServeRequest req;
    std::chrono::steady_clock::time_point t0;
    int natom = 0;
    long long done = 0;                  // steps taken
    unsigned long long rng = 0;          // noise position
    bool started = false;                // has been a member of a batch
    bool evaluated = false;              // energy/force request answered
  };
  void loop();
  void prepareLoop();
  void evaluateEnergies();
  void markIdle();
  void reform();
  void build(const std::map<int, size_t> &carried);
  void finish(const std::shared_ptr<Job> &j, ServeResult &&r);

  double m_Fraction;
  int m_Order;
  bool m_Precise;
  double m_Dt, m_Friction, m_Temp;
  uint64_t m_Seed;
  int m_Device = 0;
  size_t m_Budget = 0;

  std::mutex m_Mu;
  std::condition_variable m_Cv;
  bool m_Stop = false;
  int m_NextId = 1;
  std::deque<std::shared_ptr<Job>> m_Prepare;    // submitted, topology not built yet
  std::deque<std::shared_ptr<Job>> m_Queue;      // prepared, not admitted
  std::map<int, ServeResult> m_Results;
  ServerStats m_Stats;
  std::string m_Fatal;

  // worker-thread state
  std::vector<std::shared_ptr<Job>> m_Active;    // MD jobs running
  std::vector<std::shared_ptr<Job>> m_BatchJobs; // the jobs of m_Batch, in its order
  std::unique_ptr<Batch> m_Batch;
  DeviceArray<double4> m_Carry;                  // continuing systems' state during a re-formation
  bool m_Dirty = false;
  std::thread m_Thread, m_PrepThread;
};

}  // namespace apo
