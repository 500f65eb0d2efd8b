"""Internal virial (ForceManager::getVirial, src/ForceManager.cu:393) on the
GPU against CHARMM's values asserted by the reference's
unittest-eneForces.cpp and against the FP64 oracle (itself pinned to those
values in test_oracle_golden.py)."""
import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200.systems import config_solvated_chain, water_box
from golden_systems import golden, load_case
from parity_util import oracle_for

pytestmark = pytest.mark.gpu

VIRIAL_RTOL = 1e-5      # Frobenius norm of the difference over that of the FP64 virial


def _virial(sys, tmp_path, precise=False, settings=None):
    psf, prm, fm, ctx = api.system_context(sys, str(tmp_path), precise=precise, settings=settings)
    ctx.calculateForces(False, True, True)
    return ctx.getVirial(), ctx.getForces(), (psf, prm, fm, ctx)


@pytest.mark.parametrize("precise", [False, True])
def test_waterbox_virial_matches_charmm(tmp_path, precise):
    s = load_case("waterbox")
    W, F, keep = _virial(s, tmp_path, precise)
    ref = np.array(golden()["waterbox"]["virial"]).reshape(3, 3)
    # the reference test's tolerance (unittest-eneForces.cpp:346): 1e-4 |vir[0]|
    assert np.abs(W - ref).max() < 1e-4 * abs(ref[0, 0])
    Eo, Go, Wo = oracle_for(s).evaluate(virial=True)
    assert np.linalg.norm(W - Wo) / np.linalg.norm(Wo) < VIRIAL_RTOL


@pytest.mark.parametrize("name,tol", [("waterDimer", 1e-4), ("argon10", 1e-6)])
def test_small_cases_virial_match_charmm(tmp_path, name, tol):
    s = load_case(name)
    W, F, keep = _virial(s, tmp_path)
    ref = np.array(golden()[name]["virial"]).reshape(3, 3)
    assert np.abs(W - ref).max() < tol


@pytest.mark.parametrize("precise", [False, True])
def test_chain_virial_against_oracle(tmp_path, precise):
    s = config_solvated_chain()
    W, F, keep = _virial(s, tmp_path, precise)
    Eo, Go, Wo = oracle_for(s).evaluate(virial=True)
    err = np.linalg.norm(W - Wo) / np.linalg.norm(Wo)
    print(f"virial rel. error vs FP64: {err:.2e}")
    assert err < VIRIAL_RTOL


def test_virial_components_add_up(tmp_path):
    """Per-part virials (bonded+1-4, direct, reciprocal) sum to the total,
    and each matches the oracle's part."""
    s = water_box(512, 25.0, seed=11)
    settings = dict(kappa=0.34, nfft=(24, 24, 24), order=4, ctofnb=10.0, ctonnb=8.0, cutnb=12.0)
    psf, prm, fm, ctx = api.system_context(s, str(tmp_path), settings=settings)
    o = oracle_for(s, settings)
    total = np.zeros((3, 3))
    for mask, parts in ((1, ("bonded", "14")), (2, ("direct",)), (4, ("recip",))):
        fm.setComponentMask(mask)
        ctx.calculateForces(False, True, True)
        W = ctx.getVirial()
        Eo, Go, Wo = o.evaluate(parts=parts, virial=True)
        assert np.linalg.norm(W - Wo) <= VIRIAL_RTOL * np.linalg.norm(Wo) + 1e-6, parts
        total += W
    fm.setComponentMask(7)
    ctx.calculateForces(False, True, True)
    assert np.allclose(ctx.getVirial(), total, rtol=0, atol=1e-6)


def test_virial_requires_a_virial_evaluation(tmp_path):
    s = water_box(64, 13.0, seed=3)
    settings = dict(kappa=0.34, nfft=(16, 16, 16), order=4, ctofnb=6.0, ctonnb=5.0, cutnb=6.5)
    psf, prm, fm, ctx = api.system_context(s, str(tmp_path), settings=settings)
    ctx.calculateForces(False, True, False)
    with pytest.raises(Exception):
        ctx.getVirial()
