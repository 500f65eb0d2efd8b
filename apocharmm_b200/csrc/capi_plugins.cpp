// C ABI: plug-in forces (same conventions as capi.cpp).
#include <vector>

#include "apocharmm_c/HarmonicRestraintForce.h"
#include "capi_internal.h"
#include "force_plugins.h"

using namespace apocapi;

struct apo_harmonic_restraint_force { std::shared_ptr<apo::HarmonicRestraintForce> object; };

extern "C" apo_status apo_harmonic_restraint_force_create(apo_harmonic_restraint_force **out,
                                                          const int num_atoms) {
  const char *fn = "apo_harmonic_restraint_force_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    if (num_atoms <= 0) return invalid(fn, "num_atoms must be > 0");
    auto h = std::make_unique<apo_harmonic_restraint_force>();
    h->object = std::make_shared<apo::HarmonicRestraintForce>(num_atoms);
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" void apo_harmonic_restraint_force_destroy(apo_harmonic_restraint_force *f) { delete f; }

extern "C" apo_status apo_harmonic_restraint_force_set_selection(apo_harmonic_restraint_force *f,
                                                                 const int *atoms,
                                                                 const size_t count) {
  const char *fn = "apo_harmonic_restraint_force_set_selection";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(f, fn, "HarmonicRestraintForce"));
    if (count > 0 && !atoms) return invalid(fn, "atoms is NULL");
    std::vector<int> v(atoms, atoms + count);
    for (int a : v)
      if (a < 0 || a >= f->object->getNumAtoms()) return invalid(fn, "atom index out of range");
    f->object->setSelection(v);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_harmonic_restraint_force_set_force_constant(apo_harmonic_restraint_force *f,
                                                                      const double k) {
  const char *fn = "apo_harmonic_restraint_force_set_force_constant";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(f, fn, "HarmonicRestraintForce"));
    if (!std::isfinite(k)) return invalid(fn, "force constant must be finite");
    f->object->setForceConstant(k);
    return APO_STATUS_OK;
  }, fn);
}

namespace {
template <typename Setter>
apo_status set_per_atom(apo_harmonic_restraint_force *f, const double *v, size_t len, size_t per,
                        const char *fn, Setter set) {
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(f, fn, "HarmonicRestraintForce"));
    const size_t need = per * (size_t)f->object->getNumAtoms();
    if (!v) return invalid(fn, "input array is NULL");
    if (len != need)
      return invalid(fn, "expected " + std::to_string(need) + " values, got " + std::to_string(len));
    for (size_t i = 0; i < len; ++i)
      if (!std::isfinite(v[i])) return invalid(fn, "non-finite value");
    set(std::vector<double>(v, v + len));
    return APO_STATUS_OK;
  }, fn);
}
}  // namespace

extern "C" apo_status apo_harmonic_restraint_force_set_force_constants(apo_harmonic_restraint_force *f,
                                                                       const double *k, const size_t len) {
  return set_per_atom(f, k, len, 1, "apo_harmonic_restraint_force_set_force_constants",
                      [&](const std::vector<double> &v) { f->object->setForceConstants(v); });
}

extern "C" apo_status apo_harmonic_restraint_force_set_reference_coordinates(
    apo_harmonic_restraint_force *f, const double *xyz, const size_t len) {
  return set_per_atom(f, xyz, len, 3, "apo_harmonic_restraint_force_set_reference_coordinates",
                      [&](const std::vector<double> &v) { f->object->setReferenceCoordinates(v); });
}

extern "C" apo_status apo_harmonic_restraint_force_set_masses(apo_harmonic_restraint_force *f,
                                                              const double *m, const size_t len) {
  return set_per_atom(f, m, len, 1, "apo_harmonic_restraint_force_set_masses",
                      [&](const std::vector<double> &v) { f->object->setMasses(v); });
}

extern "C" apo_status apo_force_manager_subscribe_harmonic_restraint(apo_force_manager *fm,
                                                                     apo_harmonic_restraint_force *f,
                                                                     const char *tag) {
  const char *fn = "apo_force_manager_subscribe_harmonic_restraint";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    APO_RETURN_IF(require_handle(f, fn, "HarmonicRestraintForce"));
    APO_RETURN_IF(require_string(tag, fn, "tag"));
    if (fm->object->getNumAtoms() != f->object->getNumAtoms())
      return invalid(fn, "the restraint and the force manager differ in the number of atoms");
    try {
      fm->object->subscribe(f->object, tag);
    } catch (const std::invalid_argument &e) {
      return invalid(fn, e.what());
    }
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_unsubscribe(int *removed, apo_force_manager *fm,
                                                    const char *tag) {
  const char *fn = "apo_force_manager_unsubscribe";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(removed, fn, "removed"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    APO_RETURN_IF(require_string(tag, fn, "tag"));
    *removed = fm->object->unsubscribe(std::string(tag)) ? 1 : 0;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_energy_component(double *energy, apo_charmm_context *c,
                                                              const char *name) {
  const char *fn = "apo_charmm_context_get_energy_component";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(energy, fn, "energy"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    APO_RETURN_IF(require_string(name, fn, "name"));
    auto m = c->object->getForceManager()->getEnergyComponents(c->object->stream());
    auto it = m.find(name);
    if (it == m.end()) return invalid(fn, std::string("no energy term named '") + name + "'");
    *energy = it->second;
    return APO_STATUS_OK;
  }, fn);
}
