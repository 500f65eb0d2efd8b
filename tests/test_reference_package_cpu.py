"""The reference's own, unmodified Python package (python/apocharmm in the
reference sources) driving this library through APOCHARMM_LIBRARY_PATH, on
the host-side objects that need no GPU: PSF, parameters, coordinates, the
force manager, both subscribers and the error path.  Skipped where the
reference sources are not present."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_PY = os.path.join(os.environ.get("APOCHARMM_REFERENCE_SOURCES", "/root/reference"), "python")
LIB = os.path.join(ROOT, "apocharmm_b200", "libapocharmm_c.so")

CHILD = r"""
import sys
import numpy as np
import apocharmm                      # the reference's package
from apocharmm_b200.systems import water_box, write_charmm_files
work = sys.argv[1]
s = water_box(10, 12.0, seed=1)
p = write_charmm_files(s, work)
psf = apocharmm.CharmmPsf(p["psf"])
assert psf.getNumAtoms() == 30
assert psf.getAtomNames()[:3] == ["OH2", "H1", "H2"]
assert abs(psf.getNetCharge()) < 1e-9
assert abs(psf.getTotalMass() - 10 * (15.9994 + 2 * 1.008)) < 1e-6
prm = apocharmm.CharmmParameters([p["prm"]])
crd = apocharmm.CharmmCrd(p["crd"])
assert crd.getNumAtoms() == 30
np.testing.assert_allclose(np.array(crd.getCoordinates()), s.pos, atol=1e-5)
fm = apocharmm.ForceManager(psf, prm)
fm.setBoxDimensions([12.0, 12.0, 12.0])
r = apocharmm.RestartSubscriber(work + "/run.rst", 10)
assert r.getReportFrequency() == 10
d = apocharmm.DcdSubscriber(work + "/run.dcd")
assert d.getReportFrequency() == 1000
d.setReportFrequency(50)
assert d.getReportFrequency() == 50
try:
    apocharmm.CharmmPsf(work + "/missing.psf")
    raise SystemExit("no error for a missing file")
except apocharmm.ApoCharmmError as e:
    assert "missing.psf" in str(e)
print("ok")
"""


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_PY, "apocharmm")),
                    reason="reference sources not present")
def test_reference_python_package_drives_this_library(tmp_path):
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1", APOCHARMM_LIBRARY_PATH=LIB,
               PYTHONPATH=os.pathsep.join([REF_PY, ROOT]))
    r = subprocess.run([sys.executable, "-c", CHILD, str(tmp_path)], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
