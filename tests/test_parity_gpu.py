"""GPU parity: the sm_100a path through the C ABI against the FP64 oracle
and the reference's CHARMM golden values.

Tolerances (north star): forces within 1e-5 relative RMS, energies within
1e-6 relative (total potential), each against the FP64 oracle.
"""
import os

import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200.systems import config_solvated_chain, config_small_water, water_box
from golden_systems import golden, load_case, reference_forces
from parity_util import brute_force_pairs, oracle_for, rel_rms

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-5
ENERGY_RTOL = 1e-6


def _run(sys, tmp_path, precise=False, settings=None):
    psf, prm, fm, ctx = api.system_context(sys, str(tmp_path), precise=precise, settings=settings)
    ctx.calculateForces(False, True, False)
    return (psf, prm, fm, ctx), ctx.getEnergyComponents(), ctx.getForces()


@pytest.mark.parametrize("precise", [False, True])
def test_waterbox_matches_charmm_and_oracle(tmp_path, precise):
    s = load_case("waterbox")
    keep, E, F = _run(s, tmp_path, precise)
    g = golden()["waterbox"]
    for k, v in g["energy"].items():
        val = sum(E.values()) if k == "epot" else E[k]
        assert val == pytest.approx(v, rel=1.2e-5), k     # the reference test's tolerance
    assert np.abs(F - reference_forces("waterbox")).max() < g["force_tol"]
    Eo, Go = oracle_for(s).evaluate()
    # this fixture is an energy-minimised box: net forces are ~1e-2 while the
    # stiff O-H bond and exclusion terms are ~1e2, so single-precision
    # coordinates (the reference's own float path) set an absolute error
    # floor; the relative-RMS bar is applied to the non-minimised systems
    assert np.abs(F - Go).max() < 5e-3
    assert sum(E.values()) == pytest.approx(Eo["epot"], rel=ENERGY_RTOL)


def test_solvated_chain_forces_and_energies(tmp_path):
    s = config_solvated_chain()
    keep, E, F = _run(s, tmp_path)
    Eo, Go = oracle_for(s).evaluate()
    assert rel_rms(F, Go) < FORCE_RTOL
    assert sum(E.values()) == pytest.approx(Eo["epot"], rel=ENERGY_RTOL)
    for k in ("bond", "angle", "dihe", "vdw", "elec", "ewks", "ewse", "ewex"):
        assert E[k] == pytest.approx(Eo[k], rel=1e-5, abs=1e-3), k


def test_components_separately(tmp_path):
    s = water_box(512, 25.0, seed=11)
    settings = dict(kappa=0.34, nfft=(24, 24, 24), order=4, ctofnb=10.0, ctonnb=8.0, cutnb=12.0)
    psf, prm, fm, ctx = api.system_context(s, str(tmp_path), settings=settings)
    o = oracle_for(s, settings)
    for mask, parts in ((1, ("bonded", "14")), (2, ("direct",)), (4, ("recip", "self"))):
        fm.setComponentMask(mask)
        ctx.calculateForces(False, True, False)
        F = ctx.getForces()
        Eo, Go = o.evaluate(parts=parts)
        assert rel_rms(F, Go) < FORCE_RTOL, parts
        E = ctx.getEnergyComponents()
        assert sum(E.values()) == pytest.approx(Eo["epot"], rel=ENERGY_RTOL), parts


def test_neighbor_pairs_match_brute_force(tmp_path):
    s = water_box(1200, 23.0, seed=5)
    settings = dict(kappa=0.34, nfft=(24, 24, 24), order=4, ctofnb=9.0, ctonnb=7.0, cutnb=11.0)
    psf, prm, fm, ctx = api.system_context(s, str(tmp_path), settings=settings)
    o = oracle_for(s, settings)
    # every pair within the list radius must be covered exactly once, and no
    # topologically excluded pair may be active
    got = ctx.getNeighborPairs(11.0)
    canon = {(min(i, j), max(i, j)) for i, j, _ in got.tolist()}
    assert len(canon) == len(got), "a pair appears in more than one tile"
    ref = brute_force_pairs(s.pos, s.box, 11.0, o.eptr, o.eidx)
    # pairs within single-precision rounding of the radius may fall on either
    # side; every other pair must agree exactly
    box = np.asarray(s.box)

    def dist(p):
        d = s.pos[p[0]] - s.pos[p[1]]
        d -= box * np.round(d / box)
        return float(np.sqrt((d * d).sum()))

    diff = [p for p in canon ^ ref if abs(dist(p) - 11.0) > 1e-4]
    assert not diff, [(p, dist(p)) for p in diff[:10]]
    assert len(canon ^ ref) < 10


def test_forces_are_deterministic(tmp_path):
    s = config_small_water()
    psf, prm, fm, ctx = api.system_context(s, str(tmp_path))
    ctx.calculateForces(False, True, False)
    f1, e1 = ctx.getForces(), ctx.getEnergyComponents()
    ctx.calculateForces(True, True, False)
    f2, e2 = ctx.getForces(), ctx.getEnergyComponents()
    assert np.array_equal(f1, f2)
    assert e1 == e2


@pytest.mark.parametrize("form", [0, 2])
def test_direct_space_schedule_does_not_change_results(tmp_path, form):
    """Work items are handed out dynamically; with a persistent grid or with
    1, 2 or 4 items per warp, forces, energies and the virial are the same
    bit for bit (every item's forces and energies are rounded to fixed
    point on their own), for the tile-batch and the octet-list forms."""
    s = config_solvated_chain()
    out = {}
    for k in (0, 1, 2, 4):
        psf, prm, fm, ctx = api.system_context(s, str(tmp_path / f"k{k}"), items_per_warp=k)
        fm.setDirectKernel(form)
        ctx.calculateForces(False, True, True)
        out[k] = (ctx.getForces(), ctx.getEnergyComponents(), ctx.getVirial())
        # a second evaluation on the same context: the counters were reset
        ctx.calculateForces(False, True, True)
        assert np.array_equal(ctx.getForces(), out[k][0])
    for k in (1, 2, 4):
        assert np.array_equal(out[0][0], out[k][0])
        assert out[0][1] == out[k][1]
        assert np.array_equal(out[0][2], out[k][2])


@pytest.mark.parametrize("name", ["waterDimer", "argon10"])
def test_small_golden_cases(tmp_path, name):
    """The reference's waterDimer (unittest-eneForces.cpp:110-206) and argon10
    (:208-286) known answers through the GPU path."""
    s = load_case(name)
    keep, E, F = _run(s, tmp_path)
    g = golden()[name]
    if name == "waterDimer":
        for k, v in g["energy"].items():
            val = sum(E.values()) if k == "epot" else E[k]
            assert abs(val - v) <= g["energy_margin"], k
        ref = reference_forces(name)
    else:
        assert sum(E.values()) == pytest.approx(g["energy"]["epot"], abs=1e-5)
        ref = np.array(g["forces"])
    assert np.abs(F - ref).max() < g["force_tol"]


@pytest.mark.parametrize("precise", [False, True])
def test_direct_kernel_forms_agree(tmp_path, precise):
    """The three direct-space kernel forms (tile batches, grouped queues,
    octet lists) against the FP64 oracle and against each other on the
    solvated chain."""
    s = config_solvated_chain()
    psf, prm, fm, ctx = api.system_context(s, str(tmp_path), precise=precise)
    fm.setComponentMask(2)
    Eo, Go = oracle_for(s).evaluate(pos=ctx.getCoordinates(), parts=("direct",))
    out = {}
    for form in (0, 1, 2):
        fm.setDirectKernel(form)
        ctx.calculateForces(False, True, False)
        F, E = ctx.getForces(), ctx.getEnergyComponents()
        assert rel_rms(F, Go) < FORCE_RTOL, form
        assert E["elec"] + E["vdw"] == pytest.approx(Eo["elec"] + Eo["vdw"], rel=ENERGY_RTOL)
        out[form] = (F, E)
    for form in (1, 2):
        assert rel_rms(out[0][0], out[form][0]) < 2e-6, form
        if precise:   # per-pair fixed point: the same pairs give the same sums in any order
            assert np.array_equal(out[0][0], out[form][0]), form


@pytest.mark.parametrize("nfft", [(48, 48, 48), (64, 60, 50), (40, 48, 56)])
def test_pme_tensor_copies_give_the_same_results(tmp_path, nfft):
    """The z-pencil slabs moved by tiled tensor copies (TMA) or by plain
    loads and stores: the same arithmetic on the same values, so forces,
    energies and the virial are bit for bit the same (grids whose
    half-spectrum rows are odd (48: 25) and even (40: 21 -> padded, 64: 33))."""
    s = water_box(1500, 36.0, seed=4)
    settings = dict(kappa=0.34, nfft=nfft, order=4, ctofnb=10.0, ctonnb=8.0, cutnb=12.0)
    out = []
    for on in (True, False):
        psf, prm, fm, ctx = api.system_context(s, str(tmp_path / f"t{int(on)}"), settings=settings)
        fm.setPmeTensorCopies(on)
        ctx.calculateForces(False, True, True)
        assert fm.getPmeTensorCopies() == on
        out.append((ctx.getForces(), ctx.getEnergyComponents(), ctx.getVirial()))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
    Eo, Go = oracle_for(s, settings).evaluate(parts=("recip",))
    assert out[0][1]["ewks"] == pytest.approx(Eo["ewks"], rel=1e-5)
