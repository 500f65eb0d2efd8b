"""Pins the FP64 oracle against the reference's own known answers.

Golden values come from test/unittests/unittest-eneForces.cpp (CHARMM c47b1 /
c43b1 energies and forces); see tests/golden/make_fixtures.py.
"""
import numpy as np
import pytest

import oracle
from golden_systems import golden, load_case, reference_forces


def _oracle(name):
    s = load_case(name)
    st = s.settings
    return s, oracle.Oracle(s, st["kappa"], st["ctofnb"], st["ctonnb"], st["nfft"], st["order"])


def test_waterbox_energies_match_charmm():
    s, o = _oracle("waterbox")
    E, grad = o.evaluate()
    ref = golden()["waterbox"]["energy"]
    for k, v in ref.items():
        # Catch2 Approx default: relative 1.19e-5 (the reference test's tolerance)
        assert E[k] == pytest.approx(v, rel=1.2e-5), k
        # the oracle is much tighter than the reference test requires
        assert abs(E[k] - v) <= max(2e-3, 1e-8 * abs(v)), k


def test_waterbox_forces_match_charmm():
    s, o = _oracle("waterbox")
    E, grad = o.evaluate()
    ref = reference_forces("waterbox")          # gradient convention
    assert np.abs(grad - ref).max() < 0.01      # reference test tolerance
    assert np.abs(grad - ref).max() < 1e-4      # what the FP64 oracle achieves


def test_water_dimer():
    s, o = _oracle("waterDimer")
    E, grad = o.evaluate()
    g = golden()["waterDimer"]
    for k, v in g["energy"].items():
        assert abs(E[k] - v) <= g["energy_margin"], k
    assert np.abs(grad - reference_forces("waterDimer")).max() < g["force_tol"]


def test_argon10():
    s, o = _oracle("argon10")
    E, grad = o.evaluate()
    g = golden()["argon10"]
    assert E["epot"] == pytest.approx(g["energy"]["epot"], abs=1e-5)
    assert np.abs(grad - np.array(g["forces"])).max() < g["force_tol"]


def test_pme_converges_to_exact_ewald():
    """States the mesh error of PME itself against the exact Ewald sum."""
    s, o = _oracle("waterDimer")
    from apocharmm_b200.systems import water_box
    w = water_box(216, 20.0, seed=5)
    o = oracle.Oracle(w, 0.34, 9.0, 8.0, (32, 32, 32), 6)
    E, g_pme = o.evaluate(parts=("recip",))
    e_ex, g_ex = o.ewald_recip_exact()
    assert E["ewks"] == pytest.approx(e_ex, rel=1e-5)
    rel = np.sqrt(((g_pme - g_ex) ** 2).sum() / (g_ex ** 2).sum())
    assert rel < 1e-4


def test_topology_lists_water():
    """1-2/1-3 pairs of TIP3 (three bonds) give three ex14 pairs, no in14."""
    s, o = _oracle("waterDimer")
    assert o.in14.shape[0] == 0
    assert o.ex14.tolist() == [[0, 1], [0, 2], [1, 2], [3, 4], [3, 5], [4, 5]]


@pytest.mark.parametrize("name,abs_tol", [("waterbox", 1e-3), ("waterDimer", 1e-8),
                                          ("argon10", 1e-8)])
def test_virial_matches_charmm(name, abs_tol):
    """Internal virial (CHARMM c47b1 values asserted by the reference's
    unittest-eneForces.cpp) from the oracle's pair, bonded and PME parts."""
    s, o = _oracle(name)
    E, grad, vir = o.evaluate(virial=True)
    ref = np.array(golden()[name]["virial"]).reshape(3, 3)
    # the reference test's own tolerance: 1e-4 relative to vir[0] (waterbox), 1e-4 / 1e-6 abs
    assert np.abs(vir - ref).max() <= max(1e-4 * abs(ref[0, 0]), 1e-6)
    assert np.abs(vir - ref).max() <= abs_tol
