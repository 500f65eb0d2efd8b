"""Plug-in forces on the GPU: the harmonic positional restraint through
ForceManager::subscribe (reference: src/HarmonicRestraintForce.cu:242-290,
test/unittests/unittest-restraintForce.cpp, which drives a restrained Na-Cl
pair and checks that it stays put)."""
import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200._lib import ApoCharmmError
from apocharmm_b200.systems import water_box

pytestmark = pytest.mark.gpu

SMALL = dict(kappa=0.34, nfft=(24, 24, 24), order=4, ctofnb=9.0, ctonnb=7.5, cutnb=11.0)


def _setup(tmp_path, relax=True):
    s = water_box(1000, 31.0, seed=3)
    keep = api.system_context(s, str(tmp_path), settings=SMALL)
    if relax:
        api.relax(keep[3], api.water_indices(s), iterations=100)
    keep[3].setRandomSeedForVelocities(314159)
    keep[3].assignVelocitiesAtTemperature(300.0)
    return s, keep


def _restraint(n, atoms, ref, k, masses=None):
    h = api.HarmonicRestraintForce(n)
    h.setReferenceCoordinates(ref)
    if masses is not None:
        h.setMasses(masses)
    h.setSelection(atoms)
    h.setForceConstant(k)
    return h


def test_restraint_forces_and_energy_are_analytic(tmp_path):
    s, keep = _setup(tmp_path)
    fm, ctx = keep[2], keep[3]
    n = s.n_atoms
    x = ctx.getCoordinates()
    ctx.calculateForces(False, True, False)
    g0 = ctx.getForces()
    e0 = ctx.getPotentialEnergy()
    rng = np.random.default_rng(11)
    ref = x + rng.normal(0.0, 0.3, x.shape)
    # reference positions one box edge away act through their nearest image
    box = np.asarray(s.box, dtype=float)
    ref[::5] += box * rng.integers(-1, 2, (len(ref[::5]), 3))
    atoms = np.arange(0, n, 7)
    masses = rng.uniform(1.0, 16.0, n)
    k = 3.5
    h = _restraint(n, atoms, ref, k, masses)
    fm.subscribe(h, "harm")
    ctx.calculateForces(False, True, False)
    g1 = ctx.getForces()
    d = x[atoms] - ref[atoms]
    d -= box * np.rint(d / box)
    want = np.zeros_like(g0)
    want[atoms] = 2.0 * k * masses[atoms, None] * d
    # gradients are 2^-40 fixed point: the difference is exact to ~1e-11
    np.testing.assert_allclose(g1 - g0, want, rtol=0, atol=1e-9)
    e_harm = k * np.sum(masses[atoms] * np.sum(d * d, axis=1))
    assert ctx.getEnergyComponent("harm") == pytest.approx(e_harm, rel=1e-9)
    assert ctx.getPotentialEnergy() == pytest.approx(e0 + e_harm, rel=1e-9)
    assert ctx.getEnergyComponent("vdw") == pytest.approx(ctx.getEnergyComponents()["vdw"])
    # leaving the manager restores the unrestrained forces exactly
    assert fm.unsubscribe("harm")
    assert not fm.unsubscribe("harm")
    ctx.calculateForces(False, True, False)
    assert np.array_equal(ctx.getForces(), g0)


def _run(tmp_path, plan):
    """plan: list of ("k", value) | ("sub", k) | ("md", steps)."""
    s, keep = _setup(tmp_path)
    fm, ctx = keep[2], keep[3]
    ref = ctx.getCoordinates()
    n = s.n_atoms
    it = api.CudaLangevinThermostatIntegrator(0.002)
    it.setThermostatFriction(1.0)
    it.setThermostatRngSeed(21)
    it.setCharmmContext(ctx)
    h = None
    for op, v in plan:
        if op == "sub":
            h = _restraint(n, np.arange(n), ref, v)
            fm.subscribe(h, "harm")
        elif op == "k":
            h.setForceConstant(v)
        else:
            it.propagate(v)
    return ctx.getCoordinates(), ref


def test_restraint_joins_and_changes_inside_captured_segments(tmp_path):
    # subscribing between propagate() calls re-captures the segment graphs,
    # and a new force constant reaches graphs that are already captured
    xa, _ = _run(tmp_path / "a", [("md", 20), ("sub", 5.0), ("md", 20)])
    xb, _ = _run(tmp_path / "b", [("sub", 0.0), ("md", 20), ("k", 5.0), ("md", 20)])
    xc, _ = _run(tmp_path / "c", [("md", 40)])
    assert np.array_equal(xa, xb)
    assert not np.array_equal(xa, xc)


def test_strong_restraint_holds_atoms(tmp_path):
    x_free, ref = _run(tmp_path / "free", [("md", 200)])
    # k = 200 kcal/mol/A^2: thermal RMS displacement sqrt(3 kT / 2k) = 0.067 A
    x_held, ref2 = _run(tmp_path / "held", [("sub", 200.0), ("md", 200)])
    assert np.array_equal(ref, ref2)
    free = np.sqrt(np.mean(np.sum((x_free - ref) ** 2, axis=1)))
    held = np.sqrt(np.mean(np.sum((x_held - ref) ** 2, axis=1)))
    assert held < 0.12 < free, (held, free)


def test_subscribe_errors(tmp_path):
    s, keep = _setup(tmp_path, relax=False)
    fm = keep[2]
    with pytest.raises(ApoCharmmError, match="number of atoms"):
        fm.subscribe(api.HarmonicRestraintForce(s.n_atoms + 1), "harm")
    h = api.HarmonicRestraintForce(s.n_atoms)
    with pytest.raises(ApoCharmmError, match="built-in"):
        fm.subscribe(h, "vdw")
    fm.subscribe(h, "harm")
    with pytest.raises(ApoCharmmError, match="already in use"):
        fm.subscribe(api.HarmonicRestraintForce(s.n_atoms), "harm")
    with pytest.raises(ApoCharmmError, match="no energy term"):
        keep[3].getEnergyComponent("nothing")
