"""The reference's own, unmodified Python package (python/apocharmm of the
reference sources, installed into baseline/_ref by
oracle/install_reference_package.sh) driving this library on the GPU the
way its own scripts do: ForceManager, CharmmContext, CharmmCrd,
CudaNoseHooverIntegrator.propagate (python/apocharmm/cuda_integrator.py:129)
and a restart subscriber.  The same calls made through apocharmm_b200.api
must end in the same state bit for bit (one library underneath).  Skipped
where baseline/_ref holds no package."""
import os
import subprocess
import sys

import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200.systems import water_box, write_charmm_files, write_crd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "baseline", "_ref")
LIB = os.path.join(ROOT, "apocharmm_b200", "libapocharmm_c.so")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.isdir(os.path.join(PKG, "apocharmm")),
                                 reason="reference package not installed in baseline/_ref")]

CHILD = r"""
import sys
import apocharmm                      # the reference's package
psf_path, prm_path, crd_path, L, out = sys.argv[1], sys.argv[2], sys.argv[3], float(sys.argv[4]), sys.argv[5]
assert apocharmm.__file__.startswith(sys.argv[6]), apocharmm.__file__
psf = apocharmm.CharmmPsf(psf_path)
prm = apocharmm.CharmmParameters([prm_path])
fm = apocharmm.ForceManager(psf, prm)
fm.setBoxDimensions([L, L, L])
ctx = apocharmm.CharmmContext(fm)
ctx.setCoordinates(apocharmm.CharmmCrd(crd_path))
ctx.setRandomSeedForVelocities(2024)
ctx.assignVelocitiesAtTemperature(300.0)
t0 = ctx.computeTemperature()
it = apocharmm.CudaNoseHooverIntegrator(0.002)
it.setReferenceTemperature(300.0)
it.setCharmmContext(ctx)
rst = apocharmm.RestartSubscriber(out, 40)
it.subscribe(rst)
it.propagate(40)
print("RESULT", t0, ctx.computeTemperature(), it.getAverageTemperature())
"""


def test_reference_package_propagates_on_this_library(tmp_path):
    s = water_box(1000, 31.0, seed=3)
    keep = api.system_context(s, str(tmp_path / "relax"), settings=dict(
        kappa=0.34, nfft=(32, 32, 32), order=4, ctofnb=12.0, ctonnb=10.0, cutnb=14.0))
    relaxed = api.relax(keep[3], api.water_indices(s), iterations=100)
    del keep
    paths = write_charmm_files(s, str(tmp_path / "files"))
    write_crd(s, paths["crd"], pos=relaxed)
    L = float(s.box[0])

    env = dict(os.environ, APOCHARMM_LIBRARY_PATH=LIB,
               PYTHONPATH=os.pathsep.join([PKG, ROOT, os.environ.get("PYTHONPATH", "")]))
    out_ref = str(tmp_path / "refpkg.rst")
    r = subprocess.run([sys.executable, "-c", CHILD, paths["psf"], paths["prm"], paths["crd"],
                        repr(L), out_ref, PKG], env=env, stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]
    t0, t1, tavg = [float(x) for x in r.stdout.split("RESULT")[-1].split()[:3]]
    print(f"reference package: T {t0:.2f} K -> {t1:.2f} K (average {tavg:.2f} K)")

    # the same calls through this repository's own binding
    psf = api.CharmmPsf(paths["psf"])
    prm = api.CharmmParameters(paths["prm"])
    fm = api.ForceManager(psf, prm)
    fm.setBoxDimensions([L, L, L])
    ctx = api.CharmmContext(fm)
    ctx.setCoordinates(api.CharmmCrd(paths["crd"]))
    ctx.setRandomSeedForVelocities(2024)
    ctx.assignVelocitiesAtTemperature(300.0)
    assert ctx.computeTemperature() == t0
    it = api.CudaNoseHooverIntegrator(0.002)
    it.setReferenceTemperature(300.0)
    it.setCharmmContext(ctx)
    out_own = str(tmp_path / "own.rst")
    rst = api.RestartSubscriber(out_own, 40)
    it.subscribe(rst)
    it.propagate(40)
    assert ctx.computeTemperature() == t1
    assert it.getAverageTemperature() == tavg
    a, b = api.read_restart_file(out_ref), api.read_restart_file(out_own)
    assert a["npriv"] == b["npriv"] == 40
    for key in ("xold", "vel", "delta", "box"):
        np.testing.assert_array_equal(a[key], b[key])
    assert a["pnhv"] == b["pnhv"] and a["pnhf"] == b["pnhf"]
    assert 150.0 < t1 < 600.0
