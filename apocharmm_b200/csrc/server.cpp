// Request server with continuous batching; see server.h.
#include "server.h"

#include <algorithm>
#include <stdexcept>

namespace apo {

namespace {
constexpr int kSegment = 20;  // MD steps per list-update segment
constexpr double kIdleShare = 0.3;  // idle atoms in a batch that trigger a re-formation
double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

Server::Server(double fraction, int order, bool precise, double dt, double friction,
               double temperature, uint64_t seed)
    : m_Fraction(fraction), m_Order(order), m_Precise(precise), m_Dt(dt),
      m_Friction(friction), m_Temp(temperature), m_Seed(seed) {
  if (!(fraction > 0.0 && fraction <= 1.0))
    throw std::invalid_argument("Server: HBM fraction must be in (0, 1]");
  if (order != 4 && order != 6 && order != 8)
    throw std::invalid_argument("Server: spline order must be 4, 6 or 8");
  if (!(dt > 0.0)) throw std::invalid_argument("Server: time step must be positive");
  APO_CUDA(cudaGetDevice(&m_Device));
  size_t free_b = 0, total_b = 0;
  APO_CUDA(cudaMemGetInfo(&free_b, &total_b));
  m_Budget = (size_t)(fraction * (double)free_b);
  m_PrepThread = std::thread([this] { prepareLoop(); });
  m_Thread = std::thread([this] { loop(); });
}

Server::~Server() { stop(); }

void Server::stop() {
  {
    std::lock_guard<std::mutex> lk(m_Mu);
    m_Stop = true;
  }
  m_Cv.notify_all();
  if (m_PrepThread.joinable()) m_PrepThread.join();
  if (m_Thread.joinable()) m_Thread.join();
}

int Server::submit(ServeRequest r) {
  if (!r.spec.psf || !r.spec.prm) throw std::invalid_argument("Server: null PSF or parameters");
  const int n = r.spec.psf->getNumAtoms();
  if ((int)r.xyz.size() != 3 * n) throw std::invalid_argument("Server: coordinates must be 3 N");
  if (r.kind == 0 && r.steps <= 0) throw std::invalid_argument("Server: MD steps must be positive");
  if (r.kind != 0 && r.kind != 1) throw std::invalid_argument("Server: unknown request kind");
  auto j = std::make_shared<Job>();
  j->req = std::move(r);
  j->natom = n;
  j->t0 = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> lk(m_Mu);
  if (m_Stop) throw std::runtime_error("Server: stopped");
  if (!m_Fatal.empty()) throw std::runtime_error("Server: failed earlier: " + m_Fatal);
  j->id = m_NextId++;
  m_Results[j->id] = ServeResult{};
  m_Results[j->id].kind = j->req.kind;
  m_Prepare.push_back(j);
  m_Cv.notify_all();
  return j->id;
}

// builds each submitted request's topology off the worker thread, in
// submission order, and hands it on to admission
void Server::prepareLoop() {
  for (;;) {
    std::shared_ptr<Job> j;
    {
      std::unique_lock<std::mutex> lk(m_Mu);
      m_Cv.wait(lk, [&] { return m_Stop || !m_Prepare.empty(); });
      if (m_Stop) return;
      j = m_Prepare.front();
      m_Prepare.pop_front();
    }
    try {
      j->req.spec.topology =
          std::make_shared<const Topology>(build_topology(*j->req.spec.psf, *j->req.spec.prm));
    } catch (const std::exception &e) {
      ServeResult r;
      r.kind = j->req.kind;
      r.status = 2;
      r.error = std::string("Server: topology: ") + e.what();
      finish(j, std::move(r));
      continue;
    }
    std::lock_guard<std::mutex> lk(m_Mu);
    m_Queue.push_back(j);
    m_Cv.notify_all();
  }
}

bool Server::poll(int id, ServeResult *out) {
  std::lock_guard<std::mutex> lk(m_Mu);
  auto it = m_Results.find(id);
  if (it == m_Results.end()) throw std::invalid_argument("Server: unknown request id");
  if (it->second.status == 0) return false;
  if (out) *out = it->second;
  return true;
}

bool Server::wait(int id, double timeout_s, ServeResult *out) {
  std::unique_lock<std::mutex> lk(m_Mu);
  auto ready = [&] {
    auto it = m_Results.find(id);
    return it == m_Results.end() || it->second.status != 0;
  };
  if (timeout_s < 0) m_Cv.wait(lk, ready);
  else m_Cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
  auto it = m_Results.find(id);
  if (it == m_Results.end()) throw std::invalid_argument("Server: unknown request id");
  if (it->second.status == 0) return false;
  if (out) *out = it->second;
  return true;
}

void Server::release(int id) {
  std::lock_guard<std::mutex> lk(m_Mu);
  m_Results.erase(id);
}

ServerStats Server::stats() {
  std::lock_guard<std::mutex> lk(m_Mu);
  return m_Stats;
}

void Server::finish(const std::shared_ptr<Job> &j, ServeResult &&r) {
  r.latency_s = seconds_since(j->t0);
  std::lock_guard<std::mutex> lk(m_Mu);
  auto it = m_Results.find(j->id);
  if (it != m_Results.end()) it->second = std::move(r);
  m_Cv.notify_all();
}

// answers the energy/force requests of the current batch: one force call
// of the whole batch (every member at its current coordinates; the MD
// members' trajectories are untouched, their forces are recomputed by the
// next step), then they leave at the next re-formation
void Server::evaluateEnergies() {
  bool any = false;
  for (auto &j : m_BatchJobs) any |= j->req.kind == 1 && !j->evaluated;
  if (!any) return;
  m_Batch->calculateForces(true, false);
  for (size_t k = 0; k < m_BatchJobs.size(); ++k) {
    auto &j = m_BatchJobs[k];
    if (j->req.kind != 1 || j->evaluated) continue;
    ServeResult r;
    r.kind = 1;
    r.status = 1;
    r.forces.resize((size_t)3 * j->natom);
    m_Batch->getForces((int)k, r.forces.data());
    auto e = m_Batch->energyComponents((int)k);
    for (int t = 0; t < kNumEnergyTerms; ++t) r.energy[t] = e[kEnergyNames[t]];
    r.xyz = j->req.xyz;
    j->evaluated = true;
    finish(j, std::move(r));
  }
  std::vector<std::shared_ptr<Job>> keep;
  for (auto &j : m_Active)
    if (!(j->req.kind == 1 && j->evaluated)) keep.push_back(j);
  m_Active.swap(keep);
  markIdle();
  std::lock_guard<std::mutex> lk(m_Mu);
  ++m_Stats.energy_evals;
}

// Members that are done (finished MD requests, answered energy requests)
// stay in the batch, held still, until they hold more than kIdleShare of
// its atoms or the batch is re-formed for a new member anyway: a
// re-formation costs more than carrying a few idle systems for a while.
void Server::markIdle() {
  double idle = 0.0, all = 0.0;
  std::map<int, bool> active;
  for (auto &j : m_Active) active[j->id] = true;
  for (auto &j : m_BatchJobs) {
    all += j->natom;
    if (!active.count(j->id)) idle += j->natom;
  }
  if (all > 0.0 && idle > kIdleShare * all) m_Dirty = true;
}

// re-form the batch around m_Active; every continuing system's state moves
// device to device through m_Carry and comes back bit for bit
void Server::reform() {
  const auto t0 = std::chrono::steady_clock::now();
  std::map<int, size_t> carried;  // job id -> offset in m_Carry (double4)
  if (m_Batch) {
    std::map<int, int> in_old;
    for (size_t k = 0; k < m_BatchJobs.size(); ++k) in_old[m_BatchJobs[k]->id] = (int)k;
    size_t total = 0;
    for (auto &j : m_Active)
      if (j->started && j->req.kind == 0 && in_old.count(j->id)) {
        carried[j->id] = total;
        total += 3 * (size_t)j->natom;
      }
    if (m_Carry.n < total) m_Carry.alloc(total);
    for (auto &kv : carried) m_Batch->saveState(in_old[kv.first], m_Carry.p + kv.second);
    m_Batch.reset();  // the old batch's memory is free before the new one is built
  }
  // members that have never run: if the new batch cannot be built (a
  // request whose system is invalid or does not fit in memory), they are
  // answered with the error and the batch is built again without them
  std::map<int, bool> fresh;
  for (auto &j : m_Active)
    if (!j->started) fresh[j->id] = true;
  for (;;) {
    try {
      build(carried);
      break;
    } catch (const std::exception &e) {
      m_Batch.reset();
      std::vector<std::shared_ptr<Job>> keep, bad;
      for (auto &j : m_Active) (fresh.count(j->id) ? bad : keep).push_back(j);
      if (bad.empty()) throw;  // not a new request's doing: the server stops
      for (auto &j : bad) {
        ServeResult r;
        r.kind = j->req.kind;
        r.status = 2;
        r.error = std::string("Server: the batch could not take this request: ") + e.what();
        finish(j, std::move(r));
      }
      fresh.clear();
      m_Active.swap(keep);
      cudaGetLastError();  // a failed allocation leaves no sticky error; clear the last one
      if (m_Active.empty()) {
        m_BatchJobs.clear();
        m_Dirty = false;
        return;
      }
    }
  }
  m_Dirty = false;
  std::lock_guard<std::mutex> lk(m_Mu);
  ++m_Stats.rebuilds;
  m_Stats.reform_s += seconds_since(t0);
}

// builds the batch around m_Active, continuing systems from m_Carry
void Server::build(const std::map<int, size_t> &carried) {
  m_BatchJobs = m_Active;
  m_Batch.reset(new Batch(m_Order, 8, m_Precise));
  for (auto &j : m_Active) m_Batch->addSystem(j->req.spec);
  m_Batch->initialize();
  for (size_t k = 0; k < m_Active.size(); ++k) {
    auto &j = m_Active[k];
    auto it = carried.find(j->id);
    if (it != carried.end()) m_Batch->loadState((int)k, m_Carry.p + it->second);
    else m_Batch->setCoordinates((int)k, j->req.xyz.data());
  }
  m_Batch->setLangevin(m_Dt, m_Friction, m_Temp, m_Seed);
  m_Batch->assignVelocities(m_Temp);   // every system from its own seed
  m_Batch->createIntegrator();         // new systems: constraint + delta from velocities
  std::vector<unsigned long long> rng0;
  std::vector<long long> stop;
  for (size_t k = 0; k < m_Active.size(); ++k) {
    auto &j = m_Active[k];
    auto it = carried.find(j->id);
    // continuing systems: coordinates, velocities and delta as they were;
    // energy requests: their own coordinates (the integrator's constraint
    // set-up may have moved them)
    if (it != carried.end()) m_Batch->loadState((int)k, m_Carry.p + it->second);
    else if (j->req.kind == 1) m_Batch->setCoordinates((int)k, j->req.xyz.data());
    j->started = true;
    rng0.push_back(j->rng);
    stop.push_back(j->req.kind == 1 ? 0 : j->req.steps - j->done);
  }
  m_Batch->integrator()->setSystemLimits(rng0, stop);
}

void Server::loop() {
  try {
    APO_CUDA(cudaSetDevice(m_Device));
    for (;;) {
      std::vector<std::shared_ptr<Job>> admit;
      {
        std::unique_lock<std::mutex> lk(m_Mu);
        if (m_Queue.empty() && m_Active.empty())
          m_Cv.wait_for(lk, std::chrono::milliseconds(2),
                        [&] { return m_Stop || !m_Queue.empty(); });
        if (m_Stop) break;
        // admission by the estimated device memory of the running set
        double used = 0.0;
        for (auto &j : m_Active) used += j->natom * bytesPerAtom();
        while (!m_Queue.empty()) {
          auto &j = m_Queue.front();
          const double need = j->natom * bytesPerAtom();
          const bool nothing_running = m_Active.empty() && admit.empty();
          if (used + need > (double)m_Budget && !nothing_running) break;
          admit.push_back(j);
          used += need;
          m_Queue.pop_front();
        }
      }
      const auto t0 = std::chrono::steady_clock::now();
      if (!admit.empty()) {
        m_Active.insert(m_Active.end(), admit.begin(), admit.end());
        m_Dirty = true;
      }
      if (m_Active.empty()) {
        if (m_Batch) {  // nothing left to run: free the device memory
          m_Batch.reset();
          m_BatchJobs.clear();
        }
        std::lock_guard<std::mutex> lk(m_Mu);
        m_Stats.busy_s += seconds_since(t0);
        continue;
      }
      if (m_Dirty) reform();
      evaluateEnergies();
      bool md = false;
      for (auto &j : m_Active) md |= j->req.kind == 0;
      if (!md) {  // only energy requests were waiting
        std::lock_guard<std::mutex> lk(m_Mu);
        m_Stats.busy_s += seconds_since(t0);
        continue;
      }
      m_Batch->propagate(kSegment);
      long long advanced = 0;
      const int nactive = (int)m_BatchJobs.size();
      std::vector<std::shared_ptr<Job>> keep;
      for (size_t k = 0; k < m_BatchJobs.size(); ++k) {
        auto &j = m_BatchJobs[k];
        if (j->req.kind == 1) continue;         // energy request, held still
        if (j->done >= j->req.steps) continue;  // finished earlier, held still
        const long long take = std::min<long long>(kSegment, j->req.steps - j->done);
        j->done += take;
        j->rng += 4ull * (unsigned long long)take;
        advanced += take;
        if (j->done >= j->req.steps) {
          ServeResult r;
          r.kind = 0;
          r.status = 1;
          r.xyz.resize((size_t)3 * j->natom);
          r.vel.resize((size_t)3 * j->natom);
          m_Batch->getCoordinates((int)k, r.xyz.data());
          m_Batch->getVelocities((int)k, r.vel.data());
          finish(j, std::move(r));
        } else {
          keep.push_back(j);
        }
      }
      m_Active.swap(keep);
      markIdle();
      std::lock_guard<std::mutex> lk(m_Mu);
      ++m_Stats.segments;
      m_Stats.md_steps += advanced;
      m_Stats.sim_ps += advanced * m_Dt;
      m_Stats.max_active = std::max(m_Stats.max_active, nactive);
      m_Stats.busy_s += seconds_since(t0);
    }
  } catch (const std::exception &e) {
    std::lock_guard<std::mutex> lk(m_Mu);
    m_Fatal = e.what();
    for (auto &kv : m_Results)
      if (kv.second.status == 0) {
        kv.second.status = 2;
        kv.second.error = m_Fatal;
      }
    m_Cv.notify_all();
  }
  m_Batch.reset();
}

}  // namespace apo
