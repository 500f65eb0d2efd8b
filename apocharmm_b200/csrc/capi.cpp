// C ABI over the C++ classes: files, force manager, context.
//
// Same conventions as the reference's capi (capi/src/apocharmm_c/*.cpp):
// opaque handles that own std::shared_ptr objects, `*_create(T **out, ...)`
// sets *out = NULL before anything else, every call returns apo_status,
// C++ exceptions become APO_STATUS_RUNTIME_ERROR with the message in a
// thread-local string read by apo_last_error() (ErrorInternal.h:27-41).
// CUDA failures are reported as APO_STATUS_CUDA_ERROR.
#include "apocharmm_c/ForceView.h"
#include "capi_internal.h"

#include <cstring>
#include <string>
#include <vector>

namespace {
thread_local std::string g_last_error;
}

namespace apocapi {
void clear_error() noexcept { g_last_error.clear(); }
apo_status set_error(apo_status s, const std::string &m) noexcept {
  try {
    g_last_error = m;
  } catch (...) {
  }
  return s;
}
}  // namespace apocapi

using namespace apocapi;

extern "C" const char *apo_last_error(void) { return g_last_error.c_str(); }

// ------------------------------------------------------------------ PSF ----

extern "C" apo_status apo_charmm_psf_create(apo_charmm_psf **out, const char *path) {
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, "apo_charmm_psf_create"));
    APO_RETURN_IF(require_string(path, "apo_charmm_psf_create", "path"));
    auto h = std::make_unique<apo_charmm_psf>();
    h->object = std::make_shared<apo::CharmmPSF>(path);
    *out = h.release();
    return APO_STATUS_OK;
  }, "apo_charmm_psf_create");
}

extern "C" void apo_charmm_psf_destroy(apo_charmm_psf *psf) { delete psf; }

#define PSF_COUNT(fname, getter)                                                   \
  extern "C" apo_status fname(size_t *n, const apo_charmm_psf *psf) {              \
    return guard([&]() -> apo_status {                                             \
      APO_RETURN_IF(require_ptr(n, #fname, "output"));                             \
      *n = 0;                                                                      \
      APO_RETURN_IF(require_handle(psf, #fname, "CharmmPsf"));                     \
      *n = (size_t)psf->object->getter();                                          \
      return APO_STATUS_OK;                                                        \
    }, #fname);                                                                    \
  }
PSF_COUNT(apo_charmm_psf_get_num_atoms, getNumAtoms)
PSF_COUNT(apo_charmm_psf_get_num_bonds, getNumBonds)
PSF_COUNT(apo_charmm_psf_get_num_angles, getNumAngles)
PSF_COUNT(apo_charmm_psf_get_num_dihedrals, getNumDihedrals)
PSF_COUNT(apo_charmm_psf_get_num_impropers, getNumImpropers)
PSF_COUNT(apo_charmm_psf_get_num_cross_terms, getNumCrossTerms)

static apo_status fill_names(char *buf, size_t len, const std::vector<std::string> &names,
                             const char *fn) {
  const size_t need = 8 * names.size();
  APO_RETURN_IF(require_buffer(buf, len, need, fn, "name buffer"));
  for (size_t i = 0; i < names.size(); ++i)
    for (size_t j = 0; j < 8; ++j) buf[i * 8 + j] = j < names[i].size() ? names[i][j] : ' ';
  return APO_STATUS_OK;
}

#define PSF_NAMES(fname, getter)                                                   \
  extern "C" apo_status fname(char *buf, const size_t len, const apo_charmm_psf *psf) { \
    return guard([&]() -> apo_status {                                             \
      APO_RETURN_IF(require_handle(psf, #fname, "CharmmPsf"));                     \
      return fill_names(buf, len, psf->object->getter(), #fname);                  \
    }, #fname);                                                                    \
  }
PSF_NAMES(apo_charmm_psf_get_segment_identifiers, getSegmentIdentifiers)
PSF_NAMES(apo_charmm_psf_get_residue_names, getResidueNames)
PSF_NAMES(apo_charmm_psf_get_atom_names, getAtomNames)
PSF_NAMES(apo_charmm_psf_get_atom_types, getAtomTypes)

extern "C" apo_status apo_charmm_psf_get_residue_identifiers(int *resis, const size_t len,
                                                             const apo_charmm_psf *psf) {
  const char *fn = "apo_charmm_psf_get_residue_identifiers";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(psf, fn, "CharmmPsf"));
    const auto &v = psf->object->getResidueIdentifiers();
    APO_RETURN_IF(require_buffer(resis, len, v.size(), fn, "residue id buffer"));
    std::copy(v.begin(), v.end(), resis);
    return APO_STATUS_OK;
  }, fn);
}

#define PSF_DOUBLES(fname, getter)                                                 \
  extern "C" apo_status fname(double *out, const size_t len, const apo_charmm_psf *psf) { \
    return guard([&]() -> apo_status {                                             \
      APO_RETURN_IF(require_handle(psf, #fname, "CharmmPsf"));                     \
      const auto &v = psf->object->getter();                                       \
      APO_RETURN_IF(require_buffer(out, len, v.size(), #fname, "output buffer"));  \
      std::copy(v.begin(), v.end(), out);                                          \
      return APO_STATUS_OK;                                                        \
    }, #fname);                                                                    \
  }
PSF_DOUBLES(apo_charmm_psf_get_charges, getCharges)
PSF_DOUBLES(apo_charmm_psf_get_masses, getMasses)

#define PSF_SCALAR(fname, getter)                                                  \
  extern "C" apo_status fname(double *out, const apo_charmm_psf *psf) {            \
    return guard([&]() -> apo_status {                                             \
      APO_RETURN_IF(require_ptr(out, #fname, "output"));                           \
      *out = 0.0;                                                                  \
      APO_RETURN_IF(require_handle(psf, #fname, "CharmmPsf"));                     \
      *out = psf->object->getter();                                                \
      return APO_STATUS_OK;                                                        \
    }, #fname);                                                                    \
  }
PSF_SCALAR(apo_charmm_psf_get_net_charge, getNetCharge)
PSF_SCALAR(apo_charmm_psf_get_total_mass, getTotalMass)

extern "C" apo_status apo_charmm_psf_get_file_name(char *name, const size_t len,
                                                   const apo_charmm_psf *psf) {
  const char *fn = "apo_charmm_psf_get_file_name";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(psf, fn, "CharmmPsf"));
    const std::string &f = psf->object->getFileName();
    APO_RETURN_IF(require_buffer(name, len, f.size(), fn, "file name buffer"));
    std::memcpy(name, f.data(), f.size());
    if (len > f.size()) name[f.size()] = '\0';
    return APO_STATUS_OK;
  }, fn);
}

// ------------------------------------------------------------------ CRD ----

extern "C" apo_status apo_charmm_crd_create(apo_charmm_crd **out, const char *path) {
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, "apo_charmm_crd_create"));
    APO_RETURN_IF(require_string(path, "apo_charmm_crd_create", "path"));
    auto h = std::make_unique<apo_charmm_crd>();
    h->object = std::make_shared<apo::CharmmCrd>(path);
    *out = h.release();
    return APO_STATUS_OK;
  }, "apo_charmm_crd_create");
}
extern "C" void apo_charmm_crd_destroy(apo_charmm_crd *crd) { delete crd; }
extern "C" apo_status apo_charmm_crd_get_num_atoms(size_t *n, const apo_charmm_crd *crd) {
  const char *fn = "apo_charmm_crd_get_num_atoms";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(n, fn, "num_atoms"));
    *n = 0;
    APO_RETURN_IF(require_handle(crd, fn, "CharmmCrd"));
    *n = (size_t)crd->object->getNumAtoms();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" apo_status apo_charmm_crd_get_coordinates(double *xyz, const size_t len,
                                                     const apo_charmm_crd *crd) {
  const char *fn = "apo_charmm_crd_get_coordinates";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(crd, fn, "CharmmCrd"));
    const auto &v = crd->object->getCoordinates();
    APO_RETURN_IF(require_buffer(xyz, len, v.size(), fn, "coordinate buffer"));
    std::copy(v.begin(), v.end(), xyz);
    return APO_STATUS_OK;
  }, fn);
}

// ----------------------------------------------------------- parameters ----

extern "C" apo_status apo_charmm_parameters_create(apo_charmm_parameters **out, const char *path) {
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, "apo_charmm_parameters_create"));
    APO_RETURN_IF(require_string(path, "apo_charmm_parameters_create", "path"));
    auto h = std::make_unique<apo_charmm_parameters>();
    h->object = std::make_shared<apo::CharmmParameters>(std::string(path));
    *out = h.release();
    return APO_STATUS_OK;
  }, "apo_charmm_parameters_create");
}
extern "C" apo_status apo_charmm_parameters_create_from_files(apo_charmm_parameters **out,
                                                              const char *const *paths,
                                                              const size_t num_paths) {
  const char *fn = "apo_charmm_parameters_create_from_files";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    if (paths == nullptr || num_paths == 0) return invalid(fn, "paths is NULL or empty");
    std::vector<std::string> v;
    for (size_t i = 0; i < num_paths; ++i) {
      APO_RETURN_IF(require_string(paths[i], fn, "paths[i]"));
      v.emplace_back(paths[i]);
    }
    auto h = std::make_unique<apo_charmm_parameters>();
    h->object = std::make_shared<apo::CharmmParameters>(v);
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" void apo_charmm_parameters_destroy(apo_charmm_parameters *p) { delete p; }

// -------------------------------------------------------- force manager ----

extern "C" apo_status apo_force_manager_create(apo_force_manager **out, const apo_charmm_psf *psf,
                                               const apo_charmm_parameters *prm) {
  const char *fn = "apo_force_manager_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_handle(psf, fn, "CharmmPsf"));
    APO_RETURN_IF(require_handle(prm, fn, "CharmmParameters"));
    auto h = std::make_unique<apo_force_manager>();
    h->object = std::make_shared<apo::ForceManager>(psf->object, prm->object);
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" void apo_force_manager_destroy(apo_force_manager *fm) { delete fm; }

extern "C" apo_status apo_force_manager_set_box_dimensions(apo_force_manager *fm, const double x,
                                                           const double y, const double z) {
  const char *fn = "apo_force_manager_set_box_dimensions";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    if (!(x > 0 && y > 0 && z > 0) || !std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z))
      return invalid(fn, "box dimensions must be positive and finite");
    fm->object->setBoxDimensions({x, y, z});
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_get_box_dimensions(double *box, const size_t len,
                                                           const apo_force_manager *fm) {
  const char *fn = "apo_force_manager_get_box_dimensions";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_buffer(box, len, 3, fn, "box"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    const auto &b = fm->object->getBoxDimensions();
    for (int d = 0; d < 3; ++d) box[d] = b[d];
    return APO_STATUS_OK;
  }, fn);
}

#define FM_SETTER(fname, type, call, check)                                        \
  extern "C" apo_status fname(apo_force_manager *fm, const type v) {               \
    return guard([&]() -> apo_status {                                             \
      APO_RETURN_IF(require_handle(fm, #fname, "ForceManager"));                   \
      if (!(check)) return invalid(#fname, "value out of range");                  \
      fm->object->call;                                                            \
      return APO_STATUS_OK;                                                        \
    }, #fname);                                                                    \
  }
FM_SETTER(apo_force_manager_set_kappa, double, setKappa(v), v > 0 && std::isfinite(v))
FM_SETTER(apo_force_manager_set_cutoff, double, setCutoff(v), v > 0 && std::isfinite(v))
FM_SETTER(apo_force_manager_set_ctonnb, double, setCtonnb(v), v > 0 && std::isfinite(v))
FM_SETTER(apo_force_manager_set_ctofnb, double, setCtofnb(v), v > 0 && std::isfinite(v))
FM_SETTER(apo_force_manager_set_spline_order, int, setPmeSplineOrder(v), v == 4 || v == 6 || v == 8)
FM_SETTER(apo_force_manager_set_precision_mode, int, setPrecisionMode(v != 0), true)
FM_SETTER(apo_force_manager_set_tiles_per_work, int, setTilesPerWork(v), v >= 1 && v <= 1024)
FM_SETTER(apo_force_manager_set_work_items_per_warp, int, setWorkItemsPerWarp(v), v >= 0 && v <= 1 << 20)
FM_SETTER(apo_force_manager_set_component_mask, int, setComponentMask(v), v >= 0 && v <= 15)
FM_SETTER(apo_force_manager_set_direct_kernel, int, setDirectKernel(v), v >= 0 && v <= 2)
FM_SETTER(apo_force_manager_set_list_capacity, int, setListCapacity(v), v >= 1)
FM_SETTER(apo_force_manager_set_pme_tensor_copies, int, setPmeTensorCopies(v != 0), v == 0 || v == 1)

extern "C" apo_status apo_force_manager_get_pme_tensor_copies(int *on, const apo_force_manager *fm) {
  const char *fn = "apo_force_manager_get_pme_tensor_copies";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(on, fn, "on"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    *on = fm->object->getPmeTensorCopies() ? 1 : 0;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_get_list_capacity(int *tiles, const apo_force_manager *fm) {
  const char *fn = "apo_force_manager_get_list_capacity";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(tiles, fn, "tiles"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    *tiles = fm->object->getListCapacity();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_set_fft_grid(apo_force_manager *fm, const int nx,
                                                     const int ny, const int nz) {
  const char *fn = "apo_force_manager_set_fft_grid";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    if (nx <= 0 || ny <= 0 || nz <= 0) return invalid(fn, "grid dimensions must be positive");
    fm->object->setFFTGrid(nx, ny, nz);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_get_fft_grid(int *n3, const apo_force_manager *fm) {
  const char *fn = "apo_force_manager_get_fft_grid";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(n3, fn, "output"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    auto g = fm->object->getFFTGrid();
    n3[0] = g[0];
    n3[1] = g[1];
    n3[2] = g[2];
    return APO_STATUS_OK;
  }, fn);
}

// -------------------------------------------------------------- context ----

extern "C" apo_status apo_charmm_context_create(apo_charmm_context **out,
                                                const apo_force_manager *fm) {
  const char *fn = "apo_charmm_context_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    auto h = std::make_unique<apo_charmm_context>();
    h->force_manager = fm->object;
    h->object = std::make_shared<apo::CharmmContext>(fm->object);
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" void apo_charmm_context_destroy(apo_charmm_context *c) { delete c; }

extern "C" apo_status apo_charmm_context_set_coordinates(apo_charmm_context *c,
                                                         const apo_charmm_crd *crd) {
  const char *fn = "apo_charmm_context_set_coordinates";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    APO_RETURN_IF(require_handle(crd, fn, "CharmmCrd"));
    if (crd->object->getNumAtoms() != c->object->getNumAtoms())
      return invalid(fn, "coordinate count does not match the topology");
    c->object->setCoordinates(*crd->object);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_set_random_seed_for_velocities(apo_charmm_context *c,
                                                                        const uint64_t seed) {
  const char *fn = "apo_charmm_context_set_random_seed_for_velocities";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    c->object->setRandomSeedForVelocities(seed);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_use_holonomic_constraints(apo_charmm_context *c,
                                                                   const bool flag) {
  const char *fn = "apo_charmm_context_use_holonomic_constraints";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    c->object->useHolonomicConstraints(flag);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_assign_velocities_at_temperature(apo_charmm_context *c,
                                                                          const double t) {
  const char *fn = "apo_charmm_context_assign_velocities_at_temperature";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    if (!(t >= 0) || !std::isfinite(t)) return invalid(fn, "temperature must be >= 0");
    c->object->assignVelocitiesAtTemperature(t);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_compute_temperature(double *t, apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_compute_temperature";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(t, fn, "temperature"));
    *t = 0.0;
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    *t = c->object->computeTemperature();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_calculate_forces(apo_charmm_context *c, const bool reset,
                                                          const bool energy, const bool virial) {
  const char *fn = "apo_charmm_context_calculate_forces";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    c->object->calculateForces(reset, energy, virial);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_forces(double *xyz, const size_t len,
                                                    apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_forces";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    const size_t need = 3 * (size_t)c->object->getNumAtoms();
    APO_RETURN_IF(require_buffer(xyz, len, need, fn, "force buffer"));
    std::vector<double> f;
    c->object->getForceManager()->getForces(f, c->object->stream());
    std::copy(f.begin(), f.end(), xyz);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_energy_components(double *e, const size_t len,
                                                               apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_energy_components";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    APO_RETURN_IF(require_buffer(e, len, (size_t)apo::kNumEnergyTerms, fn, "energy buffer"));
    auto m = c->object->getForceManager()->getEnergyComponents(c->object->stream());
    for (int k = 0; k < apo::kNumEnergyTerms; ++k) e[k] = m[apo::kEnergyNames[k]];
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_virial(double *v, const size_t len,
                                                    apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_virial";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    APO_RETURN_IF(require_buffer(v, len, (size_t)9, fn, "virial buffer"));
    auto w = c->object->getForceManager()->getVirial(c->object->stream());
    for (int k = 0; k < 9; ++k) v[k] = w[k];
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_potential_energy(double *e, apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_potential_energy";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(e, fn, "energy"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    *e = c->object->getForceManager()->getPotentialEnergy(c->object->stream());
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_set_coordinates_xyz(apo_charmm_context *c,
                                                             const double *xyz, const size_t len) {
  const char *fn = "apo_charmm_context_set_coordinates_xyz";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    APO_RETURN_IF(require_ptr(xyz, fn, "xyz"));
    if (len != 3 * (size_t)c->object->getNumAtoms()) return invalid(fn, "len must be 3*N");
    // the list is rebuilt before the next force evaluation or MD segment
    c->object->setCoordinatesXyz(xyz, 0, -1, /*rebuild=*/false);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_coordinates(double *xyz, const size_t len,
                                                         apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_coordinates";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    APO_RETURN_IF(require_buffer(xyz, len, 3 * (size_t)c->object->getNumAtoms(), fn, "buffer"));
    c->object->getCoordinatesXyz(xyz);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_set_velocities(apo_charmm_context *c, const double *v,
                                                        const size_t len) {
  const char *fn = "apo_charmm_context_set_velocities";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    APO_RETURN_IF(require_ptr(v, fn, "v"));
    if (len != 3 * (size_t)c->object->getNumAtoms()) return invalid(fn, "len must be 3*N");
    c->object->setVelocitiesXyz(v);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_velocities(double *v, const size_t len,
                                                        apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_velocities";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    APO_RETURN_IF(require_buffer(v, len, 3 * (size_t)c->object->getNumAtoms(), fn, "buffer"));
    c->object->getVelocitiesXyz(v);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_num_atoms(size_t *n, const apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_num_atoms";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(n, fn, "num_atoms"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    *n = (size_t)c->object->getNumAtoms();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_degrees_of_freedom(int *n,
                                                                const apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_degrees_of_freedom";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(n, fn, "ndegf"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    *n = c->object->getDegreesOfFreedom();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_reset_neighbor_list(apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_reset_neighbor_list";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    c->object->resetNeighborList(c->object->stream());
    APO_CUDA(cudaStreamSynchronize(c->object->stream()));
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_stream(void **stream, const apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_stream";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(stream, fn, "stream"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    *stream = (void *)c->object->stream();
    return APO_STATUS_OK;
  }, fn);
}

namespace {

// Walks the pairs of the current tile list whose distance (FP64, from the
// sorted cluster-local coordinates, the cluster origins and the tile's
// image shift) is below `radius`: fn(atom i, atom j, image code, excluded).
// Padding slots and the lower triangle of a cluster's tile with itself are
// not pairs; `excluded` is the tile's topological exclusion bit.
template <typename Fn>
void for_each_list_pair(apo::ForceManager &fmr, cudaStream_t s, double radius, Fn fn) {
  apo::ForceManager *fm = &fmr;
  auto &nl = fm->neighborList();
  APO_CUDA(cudaStreamSynchronize(s));
  int counts[8];
  APO_CUDA(cudaMemcpy(counts, nl.counts, sizeof(counts), cudaMemcpyDeviceToHost));
  const int S = counts[0], T = counts[1], W = counts[2];
  const int M = std::min(counts[5], nl.dims().mask_cap);
  std::vector<int> perm(S);
  std::vector<float4> xs(S), origin((S + 31) / 32);
  std::vector<int2> tiles(T);
  std::vector<unsigned> masks((size_t)M * 32);
  std::vector<int4> work(W);
  if (S) {
    APO_CUDA(cudaMemcpy(perm.data(), nl.perm, S * sizeof(int), cudaMemcpyDeviceToHost));
    APO_CUDA(cudaMemcpy(xs.data(), nl.xyzq_s, S * sizeof(float4), cudaMemcpyDeviceToHost));
    APO_CUDA(cudaMemcpy(origin.data(), nl.cl_origin, origin.size() * sizeof(float4),
                        cudaMemcpyDeviceToHost));
  }
  if (T) APO_CUDA(cudaMemcpy(tiles.data(), nl.tiles, T * sizeof(int2), cudaMemcpyDeviceToHost));
  if (M) APO_CUDA(cudaMemcpy(masks.data(), nl.masks, masks.size() * sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (W) APO_CUDA(cudaMemcpy(work.data(), nl.work, W * sizeof(int4), cudaMemcpyDeviceToHost));
  auto box = fm->getBoxDimensions();
  const double r2max = radius * radius;
  for (auto &w : work) {
    for (int t = w.y; t < w.z; ++t) {
      const int jc = tiles[t].x, sc = apo::tile_image(tiles[t].y), mi = apo::tile_mask(tiles[t].y);
      const bool self = jc == w.x && sc == 13;
      const double sx = (sc % 3 - 1) * box[0], sy = ((sc / 3) % 3 - 1) * box[1],
                   sz = (sc / 9 - 1) * box[2];
      const float4 oi = origin[w.x], oj = origin[jc];
      for (int i = 0; i < 32; ++i) {
        const int si = w.x * 32 + i;
        if (perm[si] < 0) continue;
        const unsigned m = (mi >= 0 && mi < M) ? masks[(size_t)mi * 32 + i] : 0u;
        for (int j = self ? i + 1 : 0; j < 32; ++j) {
          const int sj = jc * 32 + j;
          if (perm[sj] < 0) continue;
          const double dx = ((double)xs[si].x + oi.x) - ((double)xs[sj].x + oj.x + sx),
                       dy = ((double)xs[si].y + oi.y) - ((double)xs[sj].y + oj.y + sy),
                       dz = ((double)xs[si].z + oi.z) - ((double)xs[sj].z + oj.z + sz);
          if (dx * dx + dy * dy + dz * dz >= r2max) continue;
          fn(perm[si], perm[sj], sc, ((m >> j) & 1u) != 0u);
        }
      }
    }
  }
}

}  // namespace

// Every tile-list pair within `radius`, with its exclusion bit:
// (atom i, atom j, excluded); each unordered pair once.
extern "C" apo_status apo_charmm_context_get_list_pairs(int *pairs, const size_t len,
                                                        size_t *num_pairs, const double radius,
                                                        apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_list_pairs";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(num_pairs, fn, "num_pairs"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    if (!(radius > 0.0)) return invalid(fn, "radius must be positive");
    size_t count = 0;
    c->object->ensureNeighborList();  // coordinates set since the last build
    for_each_list_pair(*c->object->getForceManager(), c->object->stream(), radius, [&](int i, int j, int, bool excluded) {
      if (pairs && 3 * (count + 1) <= len) {
        pairs[3 * count] = i;
        pairs[3 * count + 1] = j;
        pairs[3 * count + 2] = excluded ? 1 : 0;
      }
      ++count;
    });
    *num_pairs = count;
    if (pairs && 3 * count > len) return invalid(fn, "pair buffer too small");
    return APO_STATUS_OK;
  }, fn);
}

// Active tile-list pairs within `radius`: (atom i, atom j, image code).
extern "C" apo_status apo_charmm_context_get_neighbor_pairs(int *pairs, const size_t len,
                                                            size_t *num_pairs, const double radius,
                                                            apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_neighbor_pairs";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(num_pairs, fn, "num_pairs"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    size_t count = 0;
    c->object->ensureNeighborList();  // coordinates set since the last build
    for_each_list_pair(*c->object->getForceManager(), c->object->stream(), radius, [&](int i, int j, int sc, bool excluded) {
      if (excluded) return;
      if (pairs && 3 * (count + 1) <= len) {
        pairs[3 * count] = i;
        pairs[3 * count + 1] = j;
        pairs[3 * count + 2] = sc;
      }
      ++count;
    });
    *num_pairs = count;
    if (pairs && 3 * count > len) return invalid(fn, "pair buffer too small");
    return APO_STATUS_OK;
  }, fn);
}

// The same walk over a force manager's own list (the C++ CudaNeighborList
// view): every pair within `radius` as (atom i, atom j, excluded).
extern "C" apo_status apo_force_manager_get_list_pairs(int *pairs, const size_t len,
                                                       size_t *num_pairs, const double radius,
                                                       apo_force_manager *fm, void *stream) {
  const char *fn = "apo_force_manager_get_list_pairs";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(num_pairs, fn, "num_pairs"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    if (fm->object->isMulti()) return invalid(fn, "needs a single-system force manager");
    if (!fm->object->isListBuilt()) return invalid(fn, "no neighbour list has been built");
    if (!(radius > 0.0)) return invalid(fn, "radius must be positive");
    size_t count = 0;
    for_each_list_pair(*fm->object, reinterpret_cast<cudaStream_t>(stream), radius,
                       [&](int i, int j, int, bool excluded) {
      if (pairs && 3 * (count + 1) <= len) {
        pairs[3 * count] = i;
        pairs[3 * count + 1] = j;
        pairs[3 * count + 2] = excluded ? 1 : 0;
      }
      ++count;
    });
    *num_pairs = count;
    if (pairs && 3 * count > len) return invalid(fn, "pair buffer too small");
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_get_list_counts(int *slots, int *tiles, int *work,
                                                        apo_force_manager *fm, void *stream) {
  const char *fn = "apo_force_manager_get_list_counts";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(slots, fn, "slots"));
    APO_RETURN_IF(require_ptr(tiles, fn, "tiles"));
    APO_RETURN_IF(require_ptr(work, fn, "work_items"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    if (!fm->object->isListBuilt()) return invalid(fn, "no neighbour list has been built");
    auto &nl = fm->object->neighborList();
    nl.sync_counts(reinterpret_cast<cudaStream_t>(stream));
    *slots = nl.h_counts[0];
    *tiles = nl.h_counts[1];
    *work = nl.h_counts[2];
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_get_list_arrays(const int **glo2loc, const int **ind_sorted,
                                                        apo_force_manager *fm) {
  const char *fn = "apo_force_manager_get_list_arrays";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(glo2loc, fn, "glo2loc"));
    APO_RETURN_IF(require_ptr(ind_sorted, fn, "ind_sorted"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    if (!fm->object->isInitialized()) return invalid(fn, "the force manager is not initialized");
    *glo2loc = fm->object->neighborList().glo2loc;
    *ind_sorted = fm->object->neighborList().perm;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_set_kernel_timing(apo_charmm_context *c, const int on) {
  const char *fn = "apo_charmm_context_set_kernel_timing";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    c->object->getForceManager()->setKernelTiming(on != 0);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_kernel_time(double *ms, int *launches,
                                                         apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_kernel_time";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(ms, fn, "ms"));
    APO_RETURN_IF(require_ptr(launches, fn, "launches"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    *ms = c->object->getForceManager()->kernelTimeMs(*launches);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_charmm_context_get_list_counts(int *slots, int *tiles, int *work,
                                                         apo_charmm_context *c) {
  const char *fn = "apo_charmm_context_get_list_counts";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(slots, fn, "slots"));
    APO_RETURN_IF(require_ptr(tiles, fn, "tiles"));
    APO_RETURN_IF(require_ptr(work, fn, "work_items"));
    APO_RETURN_IF(require_handle(c, fn, "CharmmContext"));
    c->object->ensureNeighborList();
    auto &nl = c->object->getForceManager()->neighborList();
    nl.sync_counts(c->object->stream());
    *slots = nl.h_counts[0];
    *tiles = nl.h_counts[1];
    *work = nl.h_counts[2];
    return APO_STATUS_OK;
  }, fn);
}
