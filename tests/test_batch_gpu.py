"""The batch engine (apo_batch_*): several independent systems advanced
with one launch per stage.  Each system must give what it gives alone: the
same forces as its own single-system context, the same trajectory alone
and among other systems."""
import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200.systems import batch_system, water_box
from parity_util import oracle_for, rel_rms

pytestmark = pytest.mark.gpu


def _systems():
    a = water_box(216, 19.0, seed=7)
    a.settings = dict(kappa=0.34, nfft=(20, 20, 20), order=4, ctofnb=8.0, ctonnb=7.0, cutnb=9.0)
    b = batch_system(11, 3000)
    c = water_box(400, 23.5, seed=3)
    c.settings = dict(kappa=0.30, nfft=(24, 24, 24), order=4, ctofnb=9.0, ctonnb=7.5, cutnb=10.5)
    return [a, b, c]


def test_batch_forces_equal_single_contexts(tmp_path):
    systems = _systems()
    b = api.batch_from_systems(systems, str(tmp_path / "batch"))
    b.calculateForces(True, False)
    for k, s in enumerate(systems):
        keep = api.system_context(s, str(tmp_path / f"single{k}"))
        ctx = keep[3]
        ctx.calculateForces(False, True, False)
        F1, E1 = ctx.getForces(), ctx.getEnergyComponents()
        Fb, Eb = b.getForces(k), b.getEnergyComponents(k)
        # same per-system list and kernels (the batch instantiations can
        # contract float expressions differently: agreement to float rounding)
        assert rel_rms(Fb, F1) < 1e-7, k
        for t in E1:
            assert Eb[t] == pytest.approx(E1[t], rel=1e-9, abs=1e-6), (k, t)
        Eo, Go = oracle_for(s).evaluate(pos=b.getCoordinates(k))
        assert rel_rms(Fb, Go) < 1e-5, k


def test_trajectory_alone_equals_in_mix(tmp_path):
    systems = _systems()
    mix = api.batch_from_systems(systems, str(tmp_path / "mix"), seeds=[5, 6, 7])
    alone = api.batch_from_systems([systems[1]], str(tmp_path / "alone"), seeds=[6])
    api.relax_batch(mix, [api.water_indices(s) for s in systems], iterations=100)
    api.relax_batch(alone, [api.water_indices(systems[1])], iterations=100)
    assert np.array_equal(mix.getCoordinates(1), alone.getCoordinates(0))
    for bt in (mix, alone):
        bt.assignVelocities(300.0)
        bt.setLangevin(0.002, 1.0, 300.0, 42)
        bt.propagate(40)
    x_mix, x_alone = mix.getCoordinates(1), alone.getCoordinates(0)
    v_mix, v_alone = mix.getVelocities(1), alone.getVelocities(0)
    assert np.array_equal(x_mix, x_alone)
    assert np.array_equal(v_mix, v_alone)
    assert np.all(np.isfinite(mix.getCoordinates(-1)))
    t = mix.getTemperatures()
    assert t.shape == (3,) and np.all((t > 150) & (t < 450)), t


def test_autotune_restores_state(tmp_path):
    systems = _systems()
    b = api.batch_from_systems(systems, str(tmp_path / "tune"))
    api.relax_batch(b, [api.water_indices(s) for s in systems], iterations=100)
    b.assignVelocities(300.0)
    b.setLangevin(0.002, 1.0, 300.0, 9)
    x0 = b.getCoordinates(-1)
    best = b.autotune(20, [2, 8])
    assert best in (2, 8)
    assert np.array_equal(b.getCoordinates(-1), x0)
    b.propagate(20)
    assert np.all(np.isfinite(b.getCoordinates(-1)))
