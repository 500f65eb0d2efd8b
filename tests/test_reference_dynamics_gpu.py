"""Dynamics and neighbour list of this engine against the reference's own
CUDA build on identical inputs (same CRD file, same velocities, same seed).

The reference's integrators: Langevin src/CudaLangevinThermostatIntegrator.cu
(position update :576-640, noise curand_init(seed, atom, 0) + skipahead +
curand_normal4 :805-814), Nose-Hoover src/CudaNoseHooverIntegrator.cu:838,
leapfrog src/CudaLeapFrogIntegrator.cu:22-79 (no constraints, advances the
single-precision coordinates only), Langevin piston
src/CudaLangevinPistonIntegrator.cu:1705-2060, SHAKE src/CudaHolonomicConstraint.cu:
324-468.  The solute is ethylene glycol, whose X-H clusters have 2 and 3
atoms: the reference's 4-atom SHAKE kernel (src/CudaHolonomicConstraint.cu:
468-600) computes its multipliers but never moves the atoms, so a CH3 group
stays unconstrained there; this engine constrains it (tested on its own in
tests/test_integrators_gpu.py).  The neighbour list: src/CudaNeighborListBuild.cu (ientry,
tile_indj, tile_excl with bit t of j-lane l excluding i-lane (l+t) mod 32).

Skipped where oracle/_ref (built by `make -f oracle/Makefile.ref`) is absent.
"""
import numpy as np
import pytest

import reference_build as rb
from apocharmm_b200 import api
from apocharmm_b200.systems import config_ethanol, config_glycol, config_small_water, write_charmm_files

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not rb.available(), reason="reference build not present")]

KB = 1.987191e-3


def _prepared(tmp_path, sys, seed=5):
    """Relaxes `sys` on this engine, writes it as CHARMM files and returns
    (paths, CRD coordinates, Maxwell-Boltzmann velocities at 300 K)."""
    keep = api.system_context(sys, str(tmp_path / "relax"))
    sys.pos = api.relax(keep[3], api.water_indices(sys), iterations=150, max_step=0.02)
    del keep
    paths = write_charmm_files(sys, str(tmp_path))
    pos = np.array(api.CharmmCrd(paths["crd"]).getCoordinates())
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(sys.n_atoms, 3)) * np.sqrt(KB * 300.0 / sys.mass)[:, None]
    v -= (sys.mass[:, None] * v).sum(0) / sys.mass.sum()
    return paths, pos, v


def _engine(tmp_path, sys, pos, v, kind, steps, seed=0, friction=0.0, holonomic=True):
    keep = api.system_context(sys, str(tmp_path / f"b200_{kind}"))
    ctx = keep[3]
    ctx.setCoordinates(pos)
    ctx.useHolonomicConstraints(holonomic)
    ctx.setVelocities(v)
    if kind == "langevin":
        it = api.CudaLangevinThermostatIntegrator(0.002)
        it.setThermostatFriction(friction)
        it.setReferenceTemperature(300.0)
        it.setThermostatRngSeed(seed)
    elif kind == "nosehoover":
        it = api.CudaNoseHooverIntegrator(0.002)
        it.setReferenceTemperature(300.0)
    else:
        it = api.CudaLeapFrogIntegrator(0.002)
    it.setCharmmContext(ctx)
    it.propagate(steps)
    return ctx.getCoordinates(), ctx.getVelocities(), keep, it


def _wrapped_diff(a, b, box):
    d = np.asarray(a) - np.asarray(b)
    return d - np.asarray(box) * np.round(d / np.asarray(box))


@pytest.fixture(scope="module")
def glycol(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("glycol")
    s = config_glycol()
    paths, pos, v = _prepared(tmp, s)
    return tmp, s, paths, pos, v


@pytest.mark.parametrize("friction", [1.0, 20.0])
def test_langevin_trajectory_matches_reference_build(glycol, friction):
    """Same coordinates, velocities and noise seed: after 10 steps (one list
    build, SETTLE and SHAKE every step) the coordinates agree to FP32 force
    rounding.  At 20/ps the noise moves every atom by ~1e-3 A per step, so
    agreement to 1e-5 A shows that the two noise streams are equal."""
    tmp, s, paths, pos, v = glycol
    xr, _, vr = rb.traj(paths, s.box, s.settings, "langevin", 10, 2024, friction, v, str(tmp))
    x, vb, *_ = _engine(tmp, s, pos, v, "langevin", 10, seed=2024, friction=friction)
    dx = _wrapped_diff(x, xr, s.box)
    moved = np.abs(_wrapped_diff(x, pos, s.box)).max()
    print(f"Langevin {friction}/ps: max |dx| {np.abs(dx).max():.2e} A, rms {np.sqrt((dx**2).mean()):.2e} A; "
          f"largest move {moved:.3f} A; velocity rel-RMS {np.linalg.norm(vb - vr) / np.linalg.norm(vr):.2e}")
    assert moved > 0.05
    assert np.abs(dx).max() < 1e-5
    assert np.linalg.norm(vb - vr) / np.linalg.norm(vr) < 1e-5


def test_nose_hoover_trajectory_matches_reference_build(glycol):
    tmp, s, paths, pos, v = glycol
    xr, _, vr = rb.traj(paths, s.box, s.settings, "nosehoover", 10, 1, 0.0, v, str(tmp))
    x, vb, *_ = _engine(tmp, s, pos, v, "nosehoover", 10)
    dx = _wrapped_diff(x, xr, s.box)
    print(f"Nose-Hoover: max |dx| {np.abs(dx).max():.2e} A; velocity rel-RMS "
          f"{np.linalg.norm(vb - vr) / np.linalg.norm(vr):.2e}")
    assert np.abs(dx).max() < 1e-5
    assert np.linalg.norm(vb - vr) / np.linalg.norm(vr) < 1e-5


def test_leapfrog_trajectory_matches_reference_build(glycol):
    """The reference's leapfrog has no constraints and advances only the
    single-precision coordinates with single-precision forces; this engine
    advances the FP64 state (constraints off), so positions agree to the
    rounding of those FP32 updates."""
    tmp, s, paths, pos, v = glycol
    _, xr32, vr = rb.traj(paths, s.box, s.settings, "leapfrog", 10, 1, 0.0, v, str(tmp))
    x, vb, *_ = _engine(tmp, s, pos, v, "leapfrog", 10, holonomic=False)
    dx = _wrapped_diff(x, xr32, s.box)
    print(f"leapfrog: max |dx| {np.abs(dx).max():.2e} A; velocity rel-RMS "
          f"{np.linalg.norm(vb - vr) / np.linalg.norm(vr):.2e}")
    assert np.abs(dx).max() < 5e-5
    # the reference's forces come from its FP32 positions: a rounding of
    # ~2e-6 A on a bond of 545 kcal/mol/A^2 moves a hydrogen's velocity by
    # ~1e-4 of its size over 10 steps
    assert np.linalg.norm(vb - vr) / np.linalg.norm(vr) < 1e-4


@pytest.mark.parametrize("friction", [0.0, 20.0])
def test_langevin_piston_trajectory_matches_reference_build(glycol, friction):
    """Constant pressure: the reference's cubic Langevin piston at 1 atm with
    its Nose-Hoover thermostat at 300 K (src/CudaLangevinPistonIntegrator.cu:
    1705-2060), same coordinates, velocities and piston seed.  After 10 steps
    (SETTLE and SHAKE, three predictor-corrector passes a step, a new box
    every step) the box edge and the coordinates agree; at 20/ps the piston
    noise dominates the box motion, so agreement shows equal noise streams."""
    tmp, s, paths, pos, v = glycol
    xr, _, vr, boxr = rb.piston(paths, s.box, s.settings, 10, 77, friction, v, str(tmp))
    keep = api.system_context(s, str(tmp / f"b200_piston_{friction}"))
    fm, ctx = keep[2], keep[3]
    ctx.setCoordinates(pos)
    ctx.setVelocities(v)
    it = api.CudaLangevinPistonIntegrator(0.002)
    it.setCrystalType(it.CUBIC)
    it.setReferenceTemperature(300.0)
    it.setLangevinPistonFriction(friction)
    it.setLangevinPistonFrictionSeed(77)
    it.setCharmmContext(ctx)
    it.propagate(10)
    box = fm.getBoxDimensions()
    x, vb = ctx.getCoordinates(), ctx.getVelocities()
    dx = _wrapped_diff(x, xr, box)
    dbox = np.abs(box - boxr).max()
    print(f"piston {friction}/ps: box {box[0]:.9f} (reference {boxr[0]:.9f}, start {s.box[0]}), "
          f"|dbox| {dbox:.2e} A, max |dx| {np.abs(dx).max():.2e} A, velocity rel-RMS "
          f"{np.linalg.norm(vb - vr) / np.linalg.norm(vr):.2e}; P {it.getInstantaneousPressureScalar():.1f} atm")
    assert box[0] == box[1] == box[2]
    assert abs(box[0] - s.box[0]) > 1e-7          # the piston moved
    assert dbox < 1e-6
    assert np.abs(dx).max() < 1e-5
    assert np.linalg.norm(vb - vr) / np.linalg.norm(vr) < 1e-5
    assert it.getRngSequencePos() == 30


@pytest.mark.parametrize("kind", ["piston_tetra", "piston_ortho", "piston_nonh"])
def test_langevin_piston_crystal_types_match_reference_build(glycol, kind):
    """The tetragonal and orthorhombic pistons (x and y edges together, z on
    its own; three edges on their own) and the cubic piston without its
    Nose-Hoover thermostat, against the reference build over 10 steps at
    piston friction 10/ps."""
    tmp, s, paths, pos, v = glycol
    xr, _, vr, boxr = rb.piston(paths, s.box, s.settings, 10, 91, 10.0, v, str(tmp), kind=kind)
    keep = api.system_context(s, str(tmp / f"b200_{kind}"))
    fm, ctx = keep[2], keep[3]
    ctx.setCoordinates(pos)
    ctx.setVelocities(v)
    it = api.CudaLangevinPistonIntegrator(0.002)
    it.setCrystalType({"piston_tetra": it.TETRAGONAL, "piston_ortho": it.ORTHORHOMBIC,
                       "piston_nonh": it.CUBIC}[kind])
    it.setReferenceTemperature(300.0)
    it.setLangevinPistonFriction(10.0)
    it.setLangevinPistonFrictionSeed(91)
    if kind == "piston_nonh":
        it.useNoseHooverThermostat(False)
    it.setCharmmContext(ctx)
    it.propagate(10)
    box = fm.getBoxDimensions()
    x, vb = ctx.getCoordinates(), ctx.getVelocities()
    dx = _wrapped_diff(x, xr, box)
    dbox = np.abs(box - boxr).max()
    print(f"{kind}: box {box} (reference {boxr}), |dbox| {dbox:.2e} A, max |dx| "
          f"{np.abs(dx).max():.2e} A, velocity rel-RMS {np.linalg.norm(vb - vr) / np.linalg.norm(vr):.2e}")
    assert np.abs(box - s.box).min() > 1e-7
    if kind == "piston_tetra":
        assert box[0] == box[1] != box[2]
    if kind == "piston_ortho":
        assert len(set(box.tolist())) == 3
    assert dbox < 1e-6
    assert np.abs(dx).max() < 1e-5
    assert np.linalg.norm(vb - vr) / np.linalg.norm(vr) < 1e-5


def _canonical(pairs, pos, box, radius):
    """{(min g, max g): excluded} for the pairs within `radius` (FP64,
    minimum image, from the coordinates both engines read); a pair that
    appears more than once is excluded only if every copy is; an atom with
    itself (the diagonal of the reference's self tile) is no pair."""
    i, j, e = pairs[:, 0].astype(np.int64), pairs[:, 1].astype(np.int64), pairs[:, 2]
    d = pos[i] - pos[j]
    d -= box * np.round(d / box)
    keep = ((d * d).sum(1) < radius * radius) & (i != j)
    a, b, e = np.minimum(i, j)[keep], np.maximum(i, j)[keep], e[keep]
    out = {}
    for k, flag in zip(zip(a.tolist(), b.tolist()), e.tolist()):
        out[k] = out.get(k, 1) & int(flag)
    return out


@pytest.mark.parametrize("case", ["ethanol", "water"])
def test_neighbor_list_pairs_and_masks_match_reference_build(tmp_path, case):
    """Both lists hold every pair within the cutoff (2 A inside the list
    radius) exactly once as an active or a masked pair: the canonical pair
    sets and their exclusion flags are equal, with no slack."""
    s = config_ethanol() if case == "ethanol" else config_small_water()
    paths = write_charmm_files(s, str(tmp_path))
    pos = np.array(api.CharmmCrd(paths["crd"]).getCoordinates())
    st = s.settings
    keep = api.system_context(s, str(tmp_path / "b200"))
    ctx = keep[3]
    ctx.setCoordinates(pos)
    ctx.calculateForces(True, False, False)
    r = st["ctofnb"]
    export = r + 0.5
    mine = _canonical(ctx.getListPairs(export), pos, np.asarray(s.box), r)
    ref = _canonical(rb.nblist(paths, s.box, st, export, str(tmp_path)), pos, np.asarray(s.box), r)
    only_mine = set(mine) - set(ref)
    only_ref = set(ref) - set(mine)
    flag_diff = [k for k in mine.keys() & ref.keys() if mine[k] != ref[k]]
    nexcl = sum(mine.values())
    print(f"{case}: {len(mine)} pairs within {r} A ({nexcl} excluded); only here {len(only_mine)}, "
          f"only in the reference {len(only_ref)}, exclusion flags differing {len(flag_diff)}")
    assert not only_mine and not only_ref
    assert not flag_diff
    assert nexcl > 0
