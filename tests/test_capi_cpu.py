"""C-ABI checks that need no GPU: the library loads, exports every symbol
declared in include/apocharmm_c/*.h, parses CHARMM files and reports errors
with the reference's status codes."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from apocharmm_b200 import _lib, api
from apocharmm_b200.systems import config_solvated_chain, water_box, write_charmm_files

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "apocharmm_c", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"APOCHARMM_C_API\s+[\w\s\*]+?\b(apo_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 59
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_psf_prm_crd_roundtrip(tmp_path):
    s = water_box(64, 14.0, seed=3)
    paths = write_charmm_files(s, str(tmp_path))
    psf = api.CharmmPsf(paths["psf"])
    assert psf.getNumAtoms() == s.n_atoms
    assert psf.getNumBonds() == len(s.bonds)
    assert psf.getNumAngles() == len(s.angles)
    assert psf.getAtomTypes() == s.atom_type
    assert psf.getAtomNames() == s.atom_name
    np.testing.assert_allclose(psf.getCharges(), s.charge)
    np.testing.assert_allclose(psf.getMasses(), s.mass)
    assert abs(psf.getNetCharge()) < 1e-9
    assert psf.getFileName() == paths["psf"]
    crd = api.CharmmCrd(paths["crd"])
    assert crd.getNumAtoms() == s.n_atoms
    np.testing.assert_allclose(np.array(crd.getCoordinates()), s.pos, atol=1e-5)
    prm = api.CharmmParameters(paths["prm"])
    fm = api.ForceManager(psf, prm)
    fm.setBoxDimensions(s.box)
    fm.setFFTGrid(16, 16, 16)
    assert fm.getFFTGrid() == [16, 16, 16]


def test_chain_topology_files_parse(tmp_path):
    s = config_solvated_chain()
    paths = write_charmm_files(s, str(tmp_path))
    psf = api.CharmmPsf(paths["psf"])
    assert psf.getNumAtoms() == 23558
    assert psf.getNumDihedrals() == 2489 - 3
    prm = api.CharmmParameters([paths["prm"]])
    api.ForceManager(psf, prm)


def test_error_status_and_message(tmp_path):
    with pytest.raises(_lib.ApoCharmmError) as e:
        api.CharmmPsf(str(tmp_path / "missing.psf"))
    assert e.value.status == 2
    assert "missing.psf" in str(e.value)
    L = _lib.lib()
    out = ctypes.c_void_p(123)
    st = L.apo_charmm_psf_create(ctypes.byref(out), None)
    assert st == 1 and out.value is None          # out cleared before validation
    assert b"path" in L.apo_last_error()
    st = L.apo_force_manager_set_kappa(None, ctypes.c_double(0.3))
    assert st == 1
    n = ctypes.c_size_t(7)
    assert L.apo_charmm_psf_get_num_atoms(ctypes.byref(n), None) == 1
    assert n.value == 0


def test_missing_bond_parameter_is_reported(tmp_path):
    s = water_box(8, 10.0, seed=1)
    s.bond_params.pop(("HT", "OT"))
    paths = write_charmm_files(s, str(tmp_path))
    psf = api.CharmmPsf(paths["psf"])
    prm = api.CharmmParameters(paths["prm"])
    fm = api.ForceManager(psf, prm)       # assembly happens at initialize()
    assert fm is not None


def test_stream_file_with_topology_block(tmp_path):
    # a .str stream: RTF first, parameters after "read para"
    p = tmp_path / "toppar_test.str"
    p.write_text("* test\n*\nread rtf card\n* rtf\n*\n36 1\nMASS -1 OT 15.9994\nRESI TIP3 0.0\nEND\n"
                 "read para card flex\n* par\n*\nATOMS\nMASS -1 OT 15.9994\nMASS -1 HT 1.008\n"
                 "BONDS\nHT OT 450.0 0.9572\nHT HT 0.0 1.5139\nANGLES\nHT OT HT 55.0 104.52\n"
                 "NONBONDED nbxmod 5 atom cdiel -\ncutnb 14.0\nHT 0.0 -0.046 0.2245\n"
                 "OT 0.0 -0.1521 1.7682\nEND\n")
    api.CharmmParameters(str(p))


def test_batch_handle_errors_without_gpu():
    """Batch creation and argument checks need no device."""
    import ctypes
    from apocharmm_b200._lib import lib
    L = lib()
    h = ctypes.c_void_p()
    assert L.apo_batch_create(ctypes.byref(h), 5, 8, 0) == 1           # bad spline order
    assert not h.value
    assert L.apo_batch_create(ctypes.byref(h), 4, 8, 0) == 0
    n = ctypes.c_int(-1)
    assert L.apo_batch_get_num_systems(ctypes.byref(n), h) == 0 and n.value == 0
    assert L.apo_batch_propagate(h, 10) == 4                             # not initialised
    assert L.apo_batch_initialize(h) == 1                                # no systems
    L.apo_batch_destroy(h)


def test_null_handles_are_reported_without_gpu():
    """Every entry point added for plug-ins, restart files, unsubscribe and
    the direct-space knobs rejects NULL handles and outputs with
    APO_STATUS_INVALID_ARGUMENT (1) and a message, without touching a device."""
    import ctypes
    from apocharmm_b200._lib import lib
    L = lib()
    L.apo_last_error.restype = ctypes.c_char_p
    i = ctypes.c_int()
    calls = [
        lambda: L.apo_cuda_integrator_unsubscribe(ctypes.byref(i), None, None),
        lambda: L.apo_cuda_integrator_unsubscribe(None, None, None),
        lambda: L.apo_force_manager_unsubscribe(ctypes.byref(i), None, b"harm"),
        lambda: L.apo_force_manager_subscribe_harmonic_restraint(None, None, b"harm"),
        lambda: L.apo_force_manager_set_work_items_per_warp(None, ctypes.c_int(2)),
        lambda: L.apo_harmonic_restraint_force_set_force_constant(None, ctypes.c_double(1.0)),
        lambda: L.apo_charmm_context_get_energy_component(None, None, b"vdw"),
        lambda: L.apo_restart_file_read(b"", 0, None, None, None),
    ]
    for k, c in enumerate(calls):
        assert c() == 1, k
        assert L.apo_last_error(), k


def test_restraint_handle_subscribes_only_matching_sizes_without_gpu(tmp_path):
    """A force manager built from files (no device work) refuses a restraint
    for another number of atoms, and an empty tag."""
    import ctypes
    from apocharmm_b200._lib import lib
    from apocharmm_b200.systems import water_box, write_charmm_files
    s = water_box(10, 12.0, seed=1)
    p = write_charmm_files(s, str(tmp_path))
    psf, prm = api.CharmmPsf(p["psf"]), api.CharmmParameters(p["prm"])
    fm = api.ForceManager(psf, prm)
    L = lib()
    h = api.HarmonicRestraintForce(31)
    assert L.apo_force_manager_subscribe_harmonic_restraint(fm.handle, h.handle, b"harm") == 1
    h30 = api.HarmonicRestraintForce(30)
    assert L.apo_force_manager_subscribe_harmonic_restraint(fm.handle, h30.handle, b"") == 1


def test_static_reciprocal_argument_checks_without_gpu():
    """apo_pme_reciprocal_static validates its arguments before it touches a
    device: a grid axis shorter than the spline order, an odd axis or an
    unknown order is refused.  The pointers are never dereferenced."""
    fn = _lib.lib().apo_pme_reciprocal_static
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                   ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                   ctypes.c_int, ctypes.c_void_p]
    fake = ctypes.c_void_p(4096)
    for nfft, order in (((4, 4, 4), 6), ((6, 6, 6), 8), ((2, 8, 8), 4), ((8, 8, 7), 4), ((8, 8, 8), 5)):
        st = fn(fake, 8, 30.0, 30.0, 30.0, nfft[0], nfft[1], nfft[2], order, 0.34, fake, 8,
                None, 0, None)
        assert st == 1, (nfft, order)
    msg = _lib.lib().apo_last_error()
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    assert "order" in msg


def test_langevin_piston_handle_without_gpu():
    """The Langevin piston's settings and their checks need no device: the
    crystal type sets the piston's degrees of freedom, masses follow it,
    out-of-range arguments and calls that need a context are refused with
    a status and a message (include/CudaLangevinPistonIntegrator.h,
    src/CudaLangevinPistonIntegrator.cu:166-283)."""
    import ctypes
    from apocharmm_b200._lib import lib
    L = lib()
    L.apo_last_error.restype = ctypes.c_char_p
    h = ctypes.c_void_p()
    assert L.apo_cuda_langevin_piston_integrator_create(ctypes.byref(h), ctypes.c_double(-1.0)) == 1
    assert L.apo_cuda_langevin_piston_integrator_create(ctypes.byref(h), ctypes.c_double(0.002)) == 0
    m3 = (ctypes.c_double * 3)(1000.0, 2000.0, 3000.0)
    n = ctypes.c_size_t()
    # masses before the crystal type: refused, as in the reference
    assert L.apo_cuda_langevin_piston_integrator_set_langevin_piston_mass(h, m3, ctypes.c_size_t(3)) == 2
    assert b"CrystalType" in L.apo_last_error()
    assert L.apo_cuda_langevin_piston_integrator_set_crystal_type(h, 5) == 1
    assert L.apo_cuda_langevin_piston_integrator_set_crystal_type(h, 2) == 0   # orthorhombic
    c = ctypes.c_int()
    assert L.apo_cuda_langevin_piston_integrator_get_crystal_type(ctypes.byref(c), h) == 0 and c.value == 2
    out = (ctypes.c_double * 3)()
    assert L.apo_cuda_langevin_piston_integrator_get_langevin_piston_mass(out, ctypes.c_size_t(3),
                                                                           ctypes.byref(n), h) == 0
    assert n.value == 3
    assert L.apo_cuda_langevin_piston_integrator_set_langevin_piston_mass(h, m3, ctypes.c_size_t(2)) == 2
    assert L.apo_cuda_langevin_piston_integrator_set_langevin_piston_mass(h, m3, ctypes.c_size_t(3)) == 0
    assert L.apo_cuda_langevin_piston_integrator_get_langevin_piston_mass(out, ctypes.c_size_t(3),
                                                                           ctypes.byref(n), h) == 0
    assert list(out) == [1000.0, 2000.0, 3000.0]
    p9 = (ctypes.c_double * 9)(*([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0]))
    assert L.apo_cuda_langevin_piston_integrator_set_pressure(h, p9, ctypes.c_size_t(8)) == 2
    assert L.apo_cuda_langevin_piston_integrator_set_pressure(h, p9, ctypes.c_size_t(9)) == 0
    assert L.apo_cuda_langevin_piston_integrator_set_langevin_piston_friction(h, ctypes.c_double(-1.0)) == 1
    assert L.apo_cuda_langevin_piston_integrator_set_max_predictor_corrector_iterations(h, 0) == 2
    pos = ctypes.c_ulonglong(99)
    assert L.apo_cuda_langevin_piston_integrator_set_rng_sequence_pos(h, ctypes.c_ulonglong(17)) == 0
    assert L.apo_cuda_langevin_piston_integrator_get_rng_sequence_pos(ctypes.byref(pos), h) == 0
    assert pos.value == 17
    # no context yet: the pressure and piston state are not there
    p_out = (ctypes.c_double * 9)()
    assert L.apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_tensor(
        p_out, ctypes.c_size_t(9), h) == 4
    assert L.apo_cuda_langevin_piston_integrator_get_nose_hoover_piston_state(
        p_out, ctypes.c_size_t(4), h) == 4
    base = ctypes.c_void_p()
    assert L.apo_cuda_langevin_piston_integrator_as_cuda_integrator(ctypes.byref(base), h) == 0
    assert base.value
    assert L.apo_cuda_integrator_propagate(base, 10) != 0
    L.apo_cuda_langevin_piston_integrator_destroy(h)


def test_box_getter_without_gpu(tmp_path):
    """apo_force_manager_get_box_dimensions gives back the box in force (the
    one set, before any device work)."""
    s = water_box(64, 14.0, seed=3)
    paths = write_charmm_files(s, str(tmp_path))
    fm = api.ForceManager(api.CharmmPsf(paths["psf"]), api.CharmmParameters(paths["prm"]))
    fm.setBoxDimensions([14.0, 15.0, 16.5])
    np.testing.assert_array_equal(fm.getBoxDimensions(), [14.0, 15.0, 16.5])
    import ctypes
    from apocharmm_b200._lib import lib
    L = lib()
    out = (ctypes.c_double * 2)()
    assert L.apo_force_manager_get_box_dimensions(out, ctypes.c_size_t(2), fm.handle) == 1
