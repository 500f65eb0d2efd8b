"""GPU tests of the integrators through the C ABI."""
import os

import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200.systems import config_ethanol, config_small_water, solvated_chain, water_box

pytestmark = pytest.mark.gpu

SMALL = dict(kappa=0.34, nfft=(24, 24, 24), order=4, ctofnb=9.0, ctonnb=7.5, cutnb=11.0)


def _setup(tmp_path, n=1000, L=31.0, seed=3):
    s = water_box(n, L, seed=seed)
    keep = api.system_context(s, str(tmp_path), settings=SMALL)
    ctx = keep[3]
    api.relax(ctx, api.water_indices(s), iterations=100)
    ctx.setRandomSeedForVelocities(314159)
    ctx.assignVelocitiesAtTemperature(300.0)
    return s, keep


def _water_geometry(xyz):
    o, h1, h2 = xyz[0::3], xyz[1::3], xyz[2::3]
    return (np.linalg.norm(h1 - o, axis=1), np.linalg.norm(h2 - o, axis=1),
            np.linalg.norm(h2 - h1, axis=1))


def test_settle_keeps_tip3_geometry(tmp_path):
    s, keep = _setup(tmp_path)
    integ = api.CudaLangevinThermostatIntegrator(0.002)
    integ.setThermostatFriction(5.0)
    integ.setReferenceTemperature(300.0)
    integ.setThermostatRngSeed(42)
    integ.setCharmmContext(keep[3])
    integ.propagate(100)
    d1, d2, d3 = _water_geometry(keep[3].getCoordinates())
    assert np.abs(d1 - 0.9572).max() < 1e-6
    assert np.abs(d2 - 0.9572).max() < 1e-6
    assert np.abs(d3 - np.sqrt(2.29189321)).max() < 1e-6
    assert integ.getCurrentPropagatedStep() == 100


def test_langevin_runs_are_bit_identical(tmp_path):
    out = []
    for rep in range(2):
        s, keep = _setup(tmp_path / f"r{rep}")
        integ = api.CudaLangevinThermostatIntegrator(0.002)
        integ.setThermostatFriction(1.0)
        integ.setThermostatRngSeed(7)
        integ.setCharmmContext(keep[3])
        integ.propagate(60)
        out.append((keep[3].getCoordinates(), keep[3].getVelocities()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_graph_and_eager_paths_agree(tmp_path):
    res = []
    for graphs in (True, False):
        s, keep = _setup(tmp_path / f"g{int(graphs)}")
        integ = api.CudaLangevinThermostatIntegrator(0.002)
        integ.setThermostatFriction(1.0)
        integ.setThermostatRngSeed(11)
        integ.setUseGraphs(graphs)
        integ.setCharmmContext(keep[3])
        integ.propagate(45)
        res.append(keep[3].getCoordinates())
    assert np.array_equal(res[0], res[1])


def test_nve_energy_is_conserved(tmp_path):
    s, keep = _setup(tmp_path)
    ctx = keep[3]
    integ = api.CudaLangevinThermostatIntegrator(0.001)
    integ.setThermostatFriction(0.0)
    integ.setCharmmContext(ctx)
    kb = 1.987191e-3 * 0.5 * ctx.getDegreesOfFreedom()

    def total():
        # on-step kinetic energy of step n is known after step n+1, when the
        # context holds x(n+1): pair it with the potential energy at x(n)
        pe = ctx.calculatePotentialEnergy(False)
        integ.propagate(1)
        return pe + kb * integ.getInstantaneousTemperature()

    integ.propagate(40)
    series = []
    for _ in range(40):
        series.append(total())
        integ.propagate(9)
    series = np.array(series)
    ke = kb * 300.0
    drift = abs(series[-10:].mean() - series[:10].mean())
    assert drift < 0.01 * ke, (drift, series)
    assert series.std() < 0.01 * ke, series


def test_leapfrog_conserves_energy(tmp_path):
    """NVE with the leapfrog integrator (SETTLE on): total energy, with the
    on-step kinetic energy taken as the mean of the two half-step values
    around x(n), stays within 1 % of the kinetic energy over 400 steps."""
    s = water_box(1000, 31.0, seed=3)
    st = dict(kappa=0.34, nfft=(32, 32, 32), order=4, ctofnb=10.0, ctonnb=8.0, cutnb=12.0)
    keep = api.system_context(s, str(tmp_path), settings=st)
    ctx = keep[3]
    api.relax(ctx, api.water_indices(s), iterations=100)
    ctx.setRandomSeedForVelocities(27)
    ctx.assignVelocitiesAtTemperature(300.0)
    lf = api.CudaLeapFrogIntegrator(0.001)
    lf.setCharmmContext(ctx)
    m = s.mass[:, None]

    def total():
        pe = ctx.calculatePotentialEnergy(False)
        k1 = 0.5 * (m * ctx.getVelocities() ** 2).sum()
        lf.propagate(1)
        k2 = 0.5 * (m * ctx.getVelocities() ** 2).sum()
        return pe + 0.5 * (k1 + k2)

    lf.propagate(40)
    series = []
    for _ in range(40):
        series.append(total())
        lf.propagate(9)
    series = np.array(series)
    ke = 0.5 * ctx.getDegreesOfFreedom() * 1.987191e-3 * 300.0
    drift = abs(series[-10:].mean() - series[:10].mean())
    print(f"leapfrog NVE: drift {drift:.3f} kcal/mol, std {series.std():.3f}, KE {ke:.1f}")
    assert drift < 0.01 * ke, (drift, series)
    assert series.std() < 0.01 * ke, series


def test_shake_holds_x_h_bonds(tmp_path):
    """SHAKE clusters of 2 (O-H), 3 (CH2) and 4 (CH3) atoms keep their bond
    lengths through 200 Langevin steps; SETTLE keeps the waters rigid."""
    s = config_ethanol()
    keep = api.system_context(s, str(tmp_path))
    ctx = keep[3]
    api.relax(ctx, api.water_indices(s), iterations=150, max_step=0.02)
    ctx.setRandomSeedForVelocities(8)
    ctx.assignVelocitiesAtTemperature(300.0)
    it = api.CudaLangevinThermostatIntegrator(0.002)
    it.setThermostatFriction(5.0)
    it.setThermostatRngSeed(9)
    it.setCharmmContext(ctx)
    it.propagate(200)
    x = ctx.getCoordinates()
    box = np.asarray(s.box)

    def dist(i, j):
        d = x[i] - x[j]
        return np.linalg.norm(d - box * np.round(d / box), axis=-1)
    b0 = {("CT3", "HA"): 1.111, ("CT2", "HA"): 1.111, ("H", "OH1"): 0.96}
    worst, count = 0.0, 0
    for i, j in s.bonds:
        key = tuple(sorted((s.atom_type[i], s.atom_type[j])))
        if key in b0:
            worst = max(worst, abs(dist(i, j) - b0[key]))
            count += 1
    print(f"{count} X-H bonds, largest deviation {worst:.2e} A")
    assert count == 40 * 6
    assert worst < 1e-5
    w = api.water_indices(s)
    assert np.abs(dist(w[:, 1], w[:, 0]) - 0.9572).max() < 1e-6


def test_list_overflow_during_propagate_is_grown_and_replayed(tmp_path):
    """A neighbour list that outgrows its buffers during propagate() freezes
    the state at the start of that segment; the list is grown and the
    segment run again, so the trajectory is bit for bit the one of a run
    that never overflowed (the reference checks at report frequency,
    src/CudaIntegrator.cu:357-369)."""
    runs = []
    for small in (False, True):
        s, keep = _setup(tmp_path / f"o{int(small)}")
        fm, ctx = keep[2], keep[3]
        it = api.CudaLangevinThermostatIntegrator(0.002)
        it.setThermostatFriction(1.0)
        it.setThermostatRngSeed(5)
        it.setCharmmContext(ctx)
        it.propagate(20)
        before = fm.getListCapacity()
        if small:
            fm.setListCapacity(64)      # far below the ~1e4 tiles this box needs
        it.propagate(45)
        assert it.getCurrentPropagatedStep() == 65
        if small:
            assert fm.getListCapacity() > 64
        runs.append((ctx.getCoordinates(), ctx.getVelocities(), before))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


def test_non_finite_coordinates_are_refused(tmp_path):
    """Non-finite coordinates never reach the device: setCoordinates refuses
    them and the state is unchanged (inside propagate the list build flags
    them and every step kernel then leaves the state alone)."""
    s, keep = _setup(tmp_path)
    ctx = keep[3]
    x = ctx.getCoordinates()
    bad = x.copy()
    bad[7, 1] = np.nan
    with pytest.raises(RuntimeError, match="non-finite"):
        ctx.setCoordinates(bad)
    assert np.array_equal(ctx.getCoordinates(), x)


def test_langevin_thermostat_reaches_target(tmp_path):
    s, keep = _setup(tmp_path)
    integ = api.CudaLangevinThermostatIntegrator(0.002)
    integ.setThermostatFriction(10.0)
    integ.setReferenceTemperature(300.0)
    integ.setThermostatRngSeed(3)
    integ.setCharmmContext(keep[3])
    integ.propagate(300)
    t = integ.getAverageTemperature()
    assert 240.0 < t < 360.0


def test_nose_hoover_and_leapfrog_run(tmp_path):
    s, keep = _setup(tmp_path)
    nh = api.CudaNoseHooverIntegrator(0.002)
    nh.setReferenceTemperature(300.0)
    nh.setCharmmContext(keep[3])
    nh.propagate(100)
    t = nh.getInstantaneousTemperature()
    assert 150.0 < t < 600.0
    d1, _, _ = _water_geometry(keep[3].getCoordinates())
    assert np.abs(d1 - 0.9572).max() < 1e-6
    s2, keep2 = _setup(tmp_path / "lf")
    keep2[3].useHolonomicConstraints(False)
    lf = api.CudaLeapFrogIntegrator(0.0005)
    lf.setCharmmContext(keep2[3])
    lf.propagate(40)
    assert np.isfinite(keep2[3].getCoordinates()).all()


def test_dcd_subscriber_writes_frames(tmp_path):
    s, keep = _setup(tmp_path)
    integ = api.CudaLangevinThermostatIntegrator(0.002)
    integ.setThermostatFriction(1.0)
    integ.setCharmmContext(keep[3])
    path = tmp_path / "traj.dcd"
    dcd = api.DcdSubscriber(str(path), 25)
    integ.subscribe(dcd)
    integ.propagate(100)
    dcd.close()
    raw = path.read_bytes()
    n = s.n_atoms
    frame = 4 + 48 + 4 + 3 * (4 + 4 * n + 4)
    header = (4 + 84 + 4) + (4 + 84 + 4) + (4 + 4 + 4)
    assert len(raw) == header + 4 * frame
    assert raw[4:8] == b"CORD"
    assert int.from_bytes(raw[8:12], "little") == 4


def test_langevin_piston_orthorhombic_box_and_pressure(tmp_path):
    """The orthorhombic Langevin piston (src/CudaLangevinPistonIntegrator.cu)
    on a relaxed water box: every edge moves on its own, SETTLE holds the
    waters at every new box, the pressure is finite, a DCD subscriber sees
    the steps, a second run from the same state and seeds repeats the first
    bit for bit, and a restart subscriber records the piston's box, seed and
    noise position."""
    runs = []
    for rep in range(2):
        s, keep = _setup(tmp_path / f"r{rep}")
        fm, ctx = keep[2], keep[3]
        it = api.CudaLangevinPistonIntegrator(0.002)
        it.setCrystalType(it.ORTHORHOMBIC)
        it.setReferenceTemperature(300.0)
        it.setLangevinPistonFriction(10.0)
        it.setLangevinPistonFrictionSeed(11)
        it.setCharmmContext(ctx)
        assert len(it.getLangevinPistonMass()) == 3
        dcd = api.DcdSubscriber(str(tmp_path / f"r{rep}.dcd"), 10)
        it.subscribe(dcd)
        it.propagate(30)
        box = fm.getBoxDimensions()
        x = ctx.getCoordinates()
        runs.append((box, x, ctx.getVelocities(), it.getInstantaneousPressureScalar()))
        assert it.getCurrentPropagatedStep() == 30
        assert it.getRngSequencePos() == 90
        assert np.all(np.abs(box - s.box) > 1e-7) and len(set(box.tolist())) == 3
        np.testing.assert_allclose(it.getLangevinPistonOnStepPosition(), box, rtol=0, atol=1e-12)
        # half-step edge = on-step edge - half the last displacement
        np.testing.assert_allclose(it.getLangevinPistonHalfStepPosition(),
                                   box - 0.5 * it.getLangevinPistonDeltaPosition(), rtol=0, atol=1e-12)
        assert len(it.getLangevinPistonOnStepVelocity()) == 3
        assert len(it.getLangevinPistonDeltaPressure()) == 3
        assert it.getCrystalType() == it.ORTHORHOMBIC
        assert np.isfinite(it.getInstantaneousSurfaceTension())
        nh = it.getNoseHooverPistonState()
        assert np.isfinite(nh).all() and nh[0] != 0.0
        d1, d2, d3 = _water_geometry(x)
        assert np.abs(d1 - 0.9572).max() < 1e-6 and np.abs(d3 - np.sqrt(2.29189321)).max() < 1e-6
        p = it.getInstantaneousPressureTensor()
        assert np.isfinite(p).all() and np.isfinite(it.getAveragePressureScalar())
        assert os.path.getsize(tmp_path / f"r{rep}.dcd") > 0
        if rep == 1:
            it.setNoseHooverPistonState(*nh)   # a round trip leaves the state as it was
            np.testing.assert_array_equal(it.getNoseHooverPistonState(), nh)
            rst = api.RestartSubscriber(str(tmp_path / "p.rst"), 5)
            it.subscribe(rst)
            it.propagate(5)
            head = api.read_restart_file(tmp_path / "p.rst")
            assert head["npriv"] == 35 and head["seed"] == 11 and head["rngpos"] == 105
            np.testing.assert_array_equal(head["box"], fm.getBoxDimensions())
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][2], runs[1][2])


def test_settings_changed_between_calls_take_effect(tmp_path):
    """Captured segments hold the thermostat's settings as launch arguments:
    a setter called between propagate calls must reach the next call (the
    segments are captured again).  Langevin at 50/ps driven from 300 K to
    a 600 K bath heats the water box; the same run with the graphs of the
    first call would stay near 300 K."""
    s, keep = _setup(tmp_path)
    ctx = keep[3]
    it = api.CudaLangevinThermostatIntegrator(0.002)
    it.setThermostatFriction(50.0)
    it.setReferenceTemperature(300.0)
    it.setThermostatRngSeed(3)
    it.setCharmmContext(ctx)
    it.propagate(40)
    t300 = ctx.computeTemperature()
    it.setReferenceTemperature(600.0)
    it.propagate(300)
    t600 = ctx.computeTemperature()
    assert 200.0 < t300 < 450.0
    assert t600 > 480.0, (t300, t600)
