"""Parity against the reference engine's own CUDA build on the same inputs.

Skipped where oracle/_ref (built by `make -f oracle/Makefile.ref`) is absent.
Forces within 1e-5 relative RMS of the reference build and of the FP64
oracle on non-minimised systems; energies within 1e-6 relative.
"""
import numpy as np
import pytest

import reference_build as rb
from apocharmm_b200 import api
from apocharmm_b200.systems import config_solvated_chain, water_box, write_charmm_files, write_crd
from golden_systems import golden, load_case
from parity_util import oracle_for, rel_rms

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not rb.available(), reason="reference build not present")]


def _both(sys, tmp_path, settings=None):
    st = dict(sys.settings)
    st.update(settings or {})
    paths = write_charmm_files(sys, str(tmp_path))
    # identical coordinates for both engines: the CRD file the reference reads
    crd = api.CharmmCrd(paths["crd"])
    pos = np.array(crd.getCoordinates())
    keep = api.system_context(sys, str(tmp_path / "b200"), settings=st)
    ctx = keep[3]
    ctx.setCoordinates(pos)
    ctx.calculateForces(False, True, False)
    E, F = ctx.getEnergyComponents(), ctx.getForces()
    Er, Fr = rb.forces(paths, sys.box, st, str(tmp_path / "ref.txt"))
    return pos, E, F, Er, Fr, st


def test_waterbox_against_reference_build(tmp_path):
    s = load_case("waterbox")
    pos, E, F, Er, Fr, st = _both(s, tmp_path)
    g = golden()["waterbox"]["energy"]
    for k in ("bond", "angle", "vdw", "elec", "ewks", "ewse", "ewex"):
        assert Er[k] == pytest.approx(g[k], rel=1.2e-5), k        # the build reproduces CHARMM
        # the reference sums angle energies in FP32 (3e-6 relative off CHARMM);
        # this engine must be at least as close to CHARMM as the reference build
        assert abs(E[k] - g[k]) <= max(abs(Er[k] - g[k]), 2e-6 * abs(g[k])) + 2e-3, k
        assert E[k] == pytest.approx(Er[k], rel=5e-6, abs=2e-3), k
    assert sum(E.values()) == pytest.approx(sum(Er.values()), rel=1e-6)
    assert np.abs(F - Fr).max() < 5e-3


def test_chain_against_reference_build(tmp_path):
    s = config_solvated_chain()
    pos, E, F, Er, Fr, st = _both(s, tmp_path)
    s.pos = pos
    Eo, Go = oracle_for(s).evaluate()
    err_b200, err_ref = rel_rms(F, Go), rel_rms(Fr, Go)
    print(f"force rel-RMS vs FP64: b200 {err_b200:.2e}, reference build {err_ref:.2e}; "
          f"b200 vs reference {rel_rms(F, Fr):.2e}")
    assert err_b200 < 1e-5
    assert rel_rms(F, Fr) < 1e-5 + 2 * err_ref
    assert sum(E.values()) == pytest.approx(sum(Er.values()), rel=1e-6)
    assert sum(E.values()) == pytest.approx(Eo["epot"], rel=1e-6)


def test_water1m_force_error_matches_reference_build(tmp_path):
    """At a million atoms (PME grid 216^3) the force stays within 1e-5
    relative RMS of FP64.  The B-spline anchoring of spread and gather is
    taken in FP64 from the exact global position: in FP32 its rounding,
    multiplied by the grid size, made the reciprocal force the largest error
    (1.37e-5 before).  The reference's own build, on the same relaxed
    coordinates, is further from FP64 (1.16e-4 measured on a B200)."""
    from apocharmm_b200.systems import config_large_water
    s = config_large_water()
    keep = api.system_context(s, str(tmp_path / "relax"))
    s.pos = api.relax(keep[3], api.water_indices(s), iterations=150, max_step=0.03)
    del keep
    pos, E, F, Er, Fr, st = _both(s, tmp_path)
    s.pos = pos
    Eo, Go = oracle_for(s).evaluate()
    err_b200, err_ref = rel_rms(F, Go), rel_rms(Fr, Go)
    print(f"1M atoms, force rel-RMS vs FP64: b200 {err_b200:.2e}, reference build {err_ref:.2e}; "
          f"b200 vs reference {rel_rms(F, Fr):.2e}")
    assert err_b200 < 1e-5
    assert err_b200 < err_ref
    assert rel_rms(F, Fr) < 2 * (err_b200 + err_ref)
    assert sum(E.values()) == pytest.approx(Eo["epot"], rel=1e-6)
