"""Restart files on the GPU: a run resumed from a restart file follows the
uninterrupted run bit for bit (reference test:
test/unittests/unittest-restartSubscriber.cpp, which checks the Nose-Hoover
and Langevin piston variables after one step within 1e-12)."""
import shutil

import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200._lib import ApoCharmmError
from apocharmm_b200.systems import water_box

pytestmark = pytest.mark.gpu

SMALL = dict(kappa=0.34, nfft=(24, 24, 24), order=4, ctofnb=9.0, ctonnb=7.5, cutnb=11.0)


def _context(tmp_path, relax=True):
    s = water_box(1000, 31.0, seed=3)
    keep = api.system_context(s, str(tmp_path), settings=SMALL)
    ctx = keep[3]
    if relax:
        api.relax(ctx, api.water_indices(s), iterations=100)
    ctx.setRandomSeedForVelocities(314159)
    ctx.assignVelocitiesAtTemperature(300.0)
    return s, keep


def _langevin(seed):
    it = api.CudaLangevinThermostatIntegrator(0.002)
    it.setThermostatFriction(5.0)
    it.setReferenceTemperature(300.0)
    it.setThermostatRngSeed(seed)
    return it


def _nose_hoover():
    it = api.CudaNoseHooverIntegrator(0.002)
    it.setReferenceTemperature(300.0)
    return it


@pytest.mark.parametrize("kind", ["langevin", "nose_hoover"])
def test_resumed_run_matches_uninterrupted_run(tmp_path, kind):
    make = (lambda: _langevin(1234)) if kind == "langevin" else _nose_hoover
    s, keep1 = _context(tmp_path / "a")
    start = keep1[3].getCoordinates()
    it1 = make()
    it1.setCharmmContext(keep1[3])
    rst = tmp_path / "run.rst"
    sub = api.RestartSubscriber(str(rst), 40)
    it1.subscribe(sub)
    it1.propagate(40)
    saved = tmp_path / "at40.rst"
    shutil.copy(rst, saved)
    it1.propagate(60)
    x1, v1 = keep1[3].getCoordinates(), keep1[3].getVelocities()

    # a second context from the same starting coordinates; the integrator
    # takes every piece of state from the file
    s2, keep2 = _context(tmp_path / "b", relax=False)
    keep2[3].setCoordinates(start)
    it2 = _langevin(99) if kind == "langevin" else _nose_hoover()
    it2.setCharmmContext(keep2[3])
    it2.initializeFromRestartFile(str(saved))
    head = api.read_restart_file(saved)
    assert head["npriv"] == 40
    assert it2.getCurrentPropagatedStep() == 40
    if kind == "langevin":
        assert head["seed"] == 1234 and head["rngpos"] == 160
    it2.propagate(60)
    x2, v2 = keep2[3].getCoordinates(), keep2[3].getVelocities()
    assert np.array_equal(x1, x2), np.abs(x1 - x2).max()
    assert np.array_equal(v1, v2), np.abs(v1 - v2).max()
    assert it2.getCurrentPropagatedStep() == 100


def test_restart_brings_its_box(tmp_path):
    """A context set up with another box takes the restart file's box, as
    the reference's initializeFromRestartFile does
    (src/CudaLangevinThermostatIntegrator.cu:394); with the same FFT grid the
    resumed run then follows the uninterrupted one bit for bit."""
    s, keep1 = _context(tmp_path / "a")
    start = keep1[3].getCoordinates()
    it1 = _langevin(1234)
    it1.setCharmmContext(keep1[3])
    rst = tmp_path / "run.rst"
    it1.subscribe(api.RestartSubscriber(str(rst), 40))
    it1.propagate(40)
    saved = tmp_path / "at40.rst"
    shutil.copy(rst, saved)
    it1.propagate(60)
    x1, v1 = keep1[3].getCoordinates(), keep1[3].getVelocities()

    s2 = water_box(1000, 31.0, seed=3)
    s2.box = (32.5, 32.5, 32.5)  # a placeholder box
    keep2 = api.system_context(s2, str(tmp_path / "b"), settings=SMALL)
    keep2[3].setCoordinates(start)
    it2 = _langevin(99)
    it2.setCharmmContext(keep2[3])
    it2.initializeFromRestartFile(str(saved))
    it2.propagate(60)
    x2, v2 = keep2[3].getCoordinates(), keep2[3].getVelocities()
    assert np.array_equal(x1, x2), np.abs(x1 - x2).max()
    assert np.array_equal(v1, v2), np.abs(v1 - v2).max()


def test_restart_holds_the_state_of_the_report_step(tmp_path):
    s, keep = _context(tmp_path)
    it = _langevin(5)
    it.setCharmmContext(keep[3])
    rst = tmp_path / "r.rst"
    it.subscribe(api.RestartSubscriber(str(rst), 20))
    it.propagate(20)
    r = api.read_restart_file(rst)
    assert r["natom"] == s.n_atoms and r["npriv"] == 20 and r["rngpos"] == 80
    np.testing.assert_array_equal(r["xold"], keep[3].getCoordinates())
    np.testing.assert_array_equal(r["vel"], keep[3].getVelocities())
    # the delta of the last step is the displacement of a water's atoms
    assert 0.0 < np.abs(r["delta"]).max() < 0.2
    np.testing.assert_array_equal(r["box"], s.box)


def test_unsubscribed_restart_stops_reporting(tmp_path):
    # the reference test's pattern (unittest-restartSubscriber.cpp:70-83):
    # report, unsubscribe, propagate on
    s, keep = _context(tmp_path)
    it = _langevin(8)
    it.setCharmmContext(keep[3])
    rst = tmp_path / "u.rst"
    sub = api.RestartSubscriber(str(rst), 20)
    it.subscribe(sub)
    it.propagate(20)
    assert it.unsubscribe(sub)
    assert not it.unsubscribe(sub)
    it.propagate(20)
    assert api.read_restart_file(rst)["npriv"] == 20
    assert it.getCurrentPropagatedStep() == 40


def test_restart_errors(tmp_path):
    s, keep = _context(tmp_path, relax=False)
    keep[3].useHolonomicConstraints(False)
    lf = api.CudaLeapFrogIntegrator(0.0005)
    lf.setCharmmContext(keep[3])
    lf.subscribe(api.RestartSubscriber(str(tmp_path / "lf.rst"), 10))
    with pytest.raises(ApoCharmmError, match="unsupported integrator"):
        lf.propagate(10)
    # a file for another number of atoms is refused
    n = 5
    api.write_restart_file(tmp_path / "small.rst", np.zeros((n, 3)), np.zeros((n, 3)),
                           np.zeros((n, 3)), box=s.box)
    s2, keep2 = _context(tmp_path / "b", relax=False)
    it = _langevin(1)
    it.setCharmmContext(keep2[3])
    with pytest.raises(ApoCharmmError, match="NATOM mismatch"):
        it.initializeFromRestartFile(str(tmp_path / "small.rst"))


def test_piston_resumed_run_matches_uninterrupted_run(tmp_path):
    """The Langevin piston's restart file (crystal tag, HDOT, box, thermostat
    piston, seed and noise position, src/RestartSubscriber.cu:124-139) lets a
    fresh context continue the run bit for bit, the box included.  Piston
    friction 0: the reference re-seeds the noise by skipping the count of
    normals drawn, which does not resume the same stream once noise has
    weight, and this engine reads the file the same way."""
    def make():
        it = api.CudaLangevinPistonIntegrator(0.002)
        it.setCrystalType(it.ORTHORHOMBIC)
        it.setReferenceTemperature(300.0)
        it.setLangevinPistonFrictionSeed(5)
        return it

    s, keep1 = _context(tmp_path / "a")
    start = keep1[3].getCoordinates()
    it1 = make()
    it1.setCharmmContext(keep1[3])
    rst = tmp_path / "run.rst"
    it1.subscribe(api.RestartSubscriber(str(rst), 40))
    it1.propagate(40)
    saved = tmp_path / "at40.rst"
    shutil.copy(rst, saved)
    it1.propagate(60)
    x1, v1, b1 = keep1[3].getCoordinates(), keep1[3].getVelocities(), keep1[2].getBoxDimensions()

    s2, keep2 = _context(tmp_path / "b", relax=False)
    keep2[3].setCoordinates(start)
    it2 = make()
    it2.setCharmmContext(keep2[3])
    it2.initializeFromRestartFile(str(saved))
    head = api.read_restart_file(saved)
    assert head["npriv"] == 40 and it2.getCurrentPropagatedStep() == 40
    assert not np.array_equal(head["box"], s.box)
    assert head["crystal"] == "ORTH" and np.all(head["hdot"] != 0.0)
    it2.propagate(60)
    x2, v2, b2 = keep2[3].getCoordinates(), keep2[3].getVelocities(), keep2[2].getBoxDimensions()
    assert np.array_equal(b1, b2), b1 - b2
    assert np.array_equal(x1, x2), np.abs(x1 - x2).max()
    assert np.array_equal(v1, v2), np.abs(v1 - v2).max()
    assert it2.getCurrentPropagatedStep() == 100
