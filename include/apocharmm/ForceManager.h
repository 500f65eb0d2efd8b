// ForceView and ForceManager: the reference's C++ force-manager surface
// (include/ForceManager.h:37-105 ForceView, :115-694 ForceManager) over the
// C ABI, header-only.
//
//   ForceManager fm(psf, prm);           // ForceManager(psf, prm)
//   fm.setBoxDimensions({L, L, L});
//   fm.initialize();
//   fm.calcForce(d_xyzq, true, true, false);   // (xyzq, reset, calcEnergy, calcVirial)
//   std::shared_ptr<Force<double>> g = fm.getForces();
//
// d_xyzq: device float4 per atom (x, y, z, charge), atom order.  Forces are
// gradients dU/dx as in the reference.  Every call has finished on the
// manager's stream when it returns.
//
// subscribe() takes any object with the ForceView members
//   void initialize(int numAtoms, const std::vector<double> &box);
//   void clear();
//   void calcForce(const float4 *xyzq, bool calcEnergy, bool calcVirial);
//   void setBoxDimensions(const std::vector<double> &box);
//   std::shared_ptr<Force<long long int>> getForce();      // 2^40 fixed point
//   std::shared_ptr<CudaEnergyVirial> getEnergyVirial();
// and evaluates it with every force call on `forceStream`, adding its
// gradient and the sum of its energies (reported under `forceTag`).  Its
// calcForce must only enqueue stream-ordered work (no synchronisation, no
// allocation): the integrators evaluate forces inside captured segments.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "apocharmm/CharmmPSF.h"
#include "apocharmm/Check.h"
#include "apocharmm/CudaEnergyVirial.h"
#include "apocharmm/Force.h"
#include "apocharmm_c/ForceManager.h"
#include "apocharmm_c/ForceView.h"
#include "apocharmm_c/HarmonicRestraintForce.h"

// Type erasure of a force object: one table of functions per force type.
class ForceView {
 public:
  template <typename ForceType>
  ForceView(ForceType *inputForce) : m_Force(inputForce), m_Ops(&table<ForceType>()) {}

  void initialize(const int numAtoms, const std::vector<double> &boxDimensions) {
    m_Ops->initialize(m_Force, numAtoms, boxDimensions);
  }
  void clear(void) { m_Ops->clear(m_Force); }
  void calcForce(const float4 *xyzq, bool calcEnergy, bool calcVirial) {
    m_Ops->calcForce(m_Force, xyzq, calcEnergy, calcVirial);
  }
  void setBoxDimensions(const std::vector<double> &boxDimensions) {
    m_Ops->setBoxDimensions(m_Force, boxDimensions);
  }
  std::shared_ptr<Force<long long int>> getForce(void) { return m_Ops->getForce(m_Force); }
  std::shared_ptr<CudaEnergyVirial> getEnergyVirial(void) const {
    return m_Ops->getEnergyVirial(m_Force);
  }
  const void *object() const { return m_Force; }

 private:
  struct Ops {
    void (*initialize)(void *, int, const std::vector<double> &);
    void (*clear)(void *);
    void (*calcForce)(void *, const float4 *, bool, bool);
    void (*setBoxDimensions)(void *, const std::vector<double> &);
    std::shared_ptr<Force<long long int>> (*getForce)(void *);
    std::shared_ptr<CudaEnergyVirial> (*getEnergyVirial)(void *);
  };
  template <typename F>
  static const Ops &table() {
    static const Ops ops = {
        [](void *f, int n, const std::vector<double> &b) { static_cast<F *>(f)->initialize(n, b); },
        [](void *f) { static_cast<F *>(f)->clear(); },
        [](void *f, const float4 *xyzq, bool e, bool v) {
          static_cast<F *>(f)->calcForce(xyzq, e, v);
        },
        [](void *f, const std::vector<double> &b) { static_cast<F *>(f)->setBoxDimensions(b); },
        [](void *f) -> std::shared_ptr<Force<long long int>> {
          return static_cast<F *>(f)->getForce();
        },
        [](void *f) -> std::shared_ptr<CudaEnergyVirial> {
          return static_cast<F *>(f)->getEnergyVirial();
        }};
    return ops;
  }
  void *m_Force;
  const Ops *m_Ops;
};

class ForceManager {
 public:
  // the 10 built-in energy terms, in the library's order
  static const std::vector<std::string> &energyTermNames() {
    static const std::vector<std::string> names = {"bond", "angle", "ureyb", "dihe", "imdihe",
                                                   "ewks", "ewse",  "ewex",  "elec", "vdw"};
    return names;
  }

  ForceManager(std::shared_ptr<CharmmPSF> psf, std::shared_ptr<CharmmParameters> prm)
      : m_Psf(std::move(psf)), m_Prm(std::move(prm)) {
    if (!m_Psf || !m_Prm) throw std::invalid_argument("ForceManager: null PSF or parameters");
    apocharmm_detail::check(apo_force_manager_create(&m_H, m_Psf->handle(), m_Prm->handle()));
    m_Stream = std::shared_ptr<cudaStream_t>(new cudaStream_t(nullptr), [](cudaStream_t *s) {
      if (*s) cudaStreamDestroy(*s);
      delete s;
    });
    apocharmm_detail::cuda_check(cudaStreamCreateWithFlags(m_Stream.get(), cudaStreamNonBlocking),
                                 "ForceManager stream");
  }
  ~ForceManager() {
    for (auto &e : m_Subs) {  // the library forgets every view before they go
      int removed = 0;
      apo_force_manager_unsubscribe(&removed, m_H, e->tag.c_str());
    }
    if (m_Stream && *m_Stream) cudaStreamSynchronize(*m_Stream);
    apo_force_manager_destroy(m_H);
  }
  ForceManager(const ForceManager &) = delete;
  ForceManager &operator=(const ForceManager &) = delete;

  // ---- settings (include/ForceManager.h:200-225)
  void setBoxDimensions(const std::vector<double> &size) {
    if (size.size() != 3) throw std::invalid_argument("setBoxDimensions: three edges expected");
    apocharmm_detail::check(apo_force_manager_set_box_dimensions(m_H, size[0], size[1], size[2]));
    m_Box = size;
  }
  void setKappa(const float kappa) { apocharmm_detail::check(apo_force_manager_set_kappa(m_H, kappa)); }
  void setCutoff(const float cutoff) { apocharmm_detail::check(apo_force_manager_set_cutoff(m_H, cutoff)); }
  void setCtonnb(const float ctonnb) { apocharmm_detail::check(apo_force_manager_set_ctonnb(m_H, ctonnb)); }
  void setCtofnb(const float ctofnb) { apocharmm_detail::check(apo_force_manager_set_ctofnb(m_H, ctofnb)); }
  void setFFTGrid(const int nfftx, const int nffty, const int nfftz) {
    apocharmm_detail::check(apo_force_manager_set_fft_grid(m_H, nfftx, nffty, nfftz));
  }
  void setPmeSplineOrder(const int order) {
    apocharmm_detail::check(apo_force_manager_set_spline_order(m_H, order));
  }
  // the box in force (the Langevin piston changes it every step)
  std::vector<double> &getBoxDimensions(void) {
    m_Box.resize(3);
    apocharmm_detail::check(apo_force_manager_get_box_dimensions(m_Box.data(), 3, m_H));
    return m_Box;
  }
  std::shared_ptr<CharmmPSF> getPsf(void) { return m_Psf; }
  std::shared_ptr<CharmmParameters> getPrm(void) { return m_Prm; }
  int getNumAtoms() const {
    int n = 0;
    apocharmm_detail::check(apo_force_manager_get_num_atoms(&n, m_H));
    return n;
  }
  std::shared_ptr<cudaStream_t> getForceManagerStream(void) { return m_Stream; }
  apo_force_manager *handle() { return m_H; }

  // ---- evaluation (include/ForceManager.h:397-424)
  void initialize(void) {
    apocharmm_detail::check(apo_force_manager_initialize(m_H));
    m_Initialized = true;
  }
  bool isInitialized() const { return m_Initialized; }
  void resetNeighborList(const float4 *xyzq) { evaluate(xyzq, true, false, false, 0); }
  void calcForce(const float4 *xyzq, bool reset = false, bool calcEnergy = false,
                 bool calcVirial = false) {
    evaluate(xyzq, reset, calcEnergy, calcVirial, 7);
  }
  // one evaluation of the parts in `components` (1 bonded, 2 direct, 4
  // reciprocal, + 8: 1-4 pairs and exclusion corrections with the direct part)
  void evaluate(const float4 *xyzq, bool reset, bool calcEnergy, bool calcVirial, int components) {
    apocharmm_detail::check(apo_force_manager_calc_force(
        m_H, reinterpret_cast<const float *>(xyzq), getNumAtoms(), reset ? 1 : 0,
        calcEnergy ? 1 : 0, calcVirial ? 1 : 0, components, *m_Stream));
    m_Initialized = true;
  }

  // ---- results of the last evaluation (include/ForceManager.h:292-351)
  std::shared_ptr<Force<double>> getForces(void) {
    if (!m_Total) m_Total = std::make_shared<Force<double>>();
    const int n = getNumAtoms();
    if (m_Total->size() != n) m_Total->realloc(n);
    apocharmm_detail::check(
        apo_force_manager_get_forces_device(m_Total->xyz(), m_Total->stride(), m_H, *m_Stream));
    apocharmm_detail::cuda_check(cudaStreamSynchronize(*m_Stream), "ForceManager::getForces");
    return m_Total;
  }
  // the gradient in the 2^40 fixed point it is summed in, into `out`
  void getForceValues(Force<long long int> &out) {
    const int n = getNumAtoms();
    if (out.size() != n) out.realloc(n);
    apocharmm_detail::check(
        apo_force_manager_get_force_fixed_device(out.xyz(), out.stride(), m_H, *m_Stream));
    apocharmm_detail::cuda_check(cudaStreamSynchronize(*m_Stream), "ForceManager::getForceValues");
  }
  std::map<std::string, double> getEnergyComponents(void) {
    const auto &names = energyTermNames();
    std::vector<double> e(names.size());
    apocharmm_detail::check(apo_force_manager_get_energy_components(e.data(), e.size(), m_H, *m_Stream));
    std::map<std::string, double> m;
    for (size_t k = 0; k < names.size(); ++k) m[names[k]] = e[k];
    for (auto &s : m_Subs) {
      double v = 0.0;
      apocharmm_detail::check(apo_force_manager_get_energy_component(&v, m_H, s->tag.c_str(), *m_Stream));
      m[s->tag] = v;
    }
    return m;
  }
  double getPotentialEnergy(void) {
    double t = 0.0;
    for (auto &kv : getEnergyComponents()) t += kv.second;
    return t;
  }
  std::vector<double> getVirial(void) {
    std::vector<double> v(9);
    apocharmm_detail::check(apo_force_manager_get_virial(v.data(), v.size(), m_H, *m_Stream));
    return v;
  }

  // ---- plug-in forces (include/ForceManager.h:429-475)
  template <typename ForceType>
  void subscribe(std::shared_ptr<ForceType> force, const std::string &forceTag,
                 std::shared_ptr<cudaStream_t> forceStream,
                 std::shared_ptr<Force<long long int>> forceValues,
                 std::shared_ptr<CudaEnergyVirial> energyVirial) {
    if (!force) throw std::invalid_argument("ForceManager::subscribe: null force");
    if (!forceStream || !*forceStream)
      throw std::invalid_argument("ForceManager::subscribe: the force needs a stream of its own");
    std::unique_ptr<Subscription> s(new Subscription{std::static_pointer_cast<void>(force),
                                                     ForceView(force.get()), forceTag,
                                                     forceStream, forceValues, energyVirial, ""});
    apo_force_view v;
    v.object = s.get();
    v.initialize = &Subscription::initialize;
    v.clear = &Subscription::clear;
    v.calc_force = &Subscription::calc_force;
    v.get_force = &Subscription::get_force;
    v.get_energies = &Subscription::get_energies;
    v.stream = *forceStream;
    apocharmm_detail::check(apo_force_manager_subscribe_view(m_H, &v, forceTag.c_str()));
    m_Subs.push_back(std::move(s));
  }
  template <typename ForceType>
  void unsubscribe(std::shared_ptr<ForceType> force) {
    for (size_t i = 0; i < m_Subs.size(); ++i)
      if (m_Subs[i]->keep.get() == static_cast<void *>(force.get())) {
        unsubscribe(m_Subs[i]->tag);
        return;
      }
  }
  void unsubscribe(const std::string &forceTag) {
    for (size_t i = 0; i < m_Subs.size(); ++i)
      if (m_Subs[i]->tag == forceTag) {
        int removed = 0;
        apocharmm_detail::check(apo_force_manager_unsubscribe(&removed, m_H, forceTag.c_str()));
        m_Subs.erase(m_Subs.begin() + i);
        return;
      }
  }
  // the first error a subscribed force raised inside an evaluation ("" = none)
  std::string getSubscriptionError(const std::string &forceTag) const {
    for (auto &s : m_Subs)
      if (s->tag == forceTag) return s->error;
    return "";
  }

 private:
  // one subscribed force; the library calls these through the C table.  An
  // exception is kept (the library sees a missing force buffer and fails
  // the evaluation) instead of crossing the C boundary.
  struct Subscription {
    std::shared_ptr<void> keep;
    ForceView view;
    std::string tag;
    std::shared_ptr<cudaStream_t> stream;
    std::shared_ptr<Force<long long int>> values;
    std::shared_ptr<CudaEnergyVirial> energyVirial;
    std::string error;

    static void initialize(void *o, int n, const double *b) {
      auto *s = static_cast<Subscription *>(o);
      try {
        s->view.initialize(n, {b[0], b[1], b[2]});
      } catch (const std::exception &e) {
        s->error = e.what();
      }
    }
    static void clear(void *o) {
      auto *s = static_cast<Subscription *>(o);
      try {
        s->view.clear();
      } catch (const std::exception &e) {
        s->error = e.what();
      }
    }
    static void calc_force(void *o, const float *xyzq, int e, int v) {
      auto *s = static_cast<Subscription *>(o);
      try {
        s->view.calcForce(reinterpret_cast<const float4 *>(xyzq), e != 0, v != 0);
      } catch (const std::exception &ex) {
        s->error = ex.what();
      }
    }
    static const long long *get_force(void *o, int *stride) {
      auto *s = static_cast<Subscription *>(o);
      if (!s->error.empty()) return nullptr;
      try {
        auto f = s->view.getForce();
        if (!f) return nullptr;
        *stride = f->stride();
        return f->xyz();
      } catch (const std::exception &e) {
        s->error = e.what();
        return nullptr;
      }
    }
    static const double *get_energies(void *o, int *count) {
      auto *s = static_cast<Subscription *>(o);
      try {
        auto ev = s->view.getEnergyVirial();
        if (!ev) return nullptr;
        *count = ev->getN();
        return ev->deviceData();
      } catch (const std::exception &e) {
        s->error = e.what();
        return nullptr;
      }
    }
  };

  std::shared_ptr<CharmmPSF> m_Psf;
  std::shared_ptr<CharmmParameters> m_Prm;
  apo_force_manager *m_H = nullptr;
  std::shared_ptr<cudaStream_t> m_Stream;
  std::vector<double> m_Box;
  bool m_Initialized = false;
  std::shared_ptr<Force<double>> m_Total;
  std::vector<std::unique_ptr<Subscription>> m_Subs;
};
