"""Restart files on the host: layout, exact round trip, the reference's
column rules and its 16-digit form (src/RestartSubscriber.cu:39-445,
src/CudaLangevinThermostatIntegrator.cu:264-545)."""
import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200._lib import ApoCharmmError as ApoError


def _state(n, seed=5):
    rng = np.random.default_rng(seed)
    xold = rng.uniform(-40.0, 40.0, (n, 3))
    vel = rng.normal(0.0, 0.2, (n, 3))
    delta = rng.normal(0.0, 0.01, (n, 3))
    # values that exercise every exponent form of the 22 columns
    special = np.array([0.0, -0.0, 1.0, -1.0, 123.456, -987.654321, 1e-5, -1e-5, 3e-9, -3e-9,
                        1e-12, 7.5e11, -7.5e11, 1e-300, -1e-300, 2.5e300, -2.5e300,
                        np.nextafter(1.0, 2.0), -np.nextafter(1.0, 2.0), 1.0 / 3.0, -2.0 / 3.0])
    m = min(special.size, delta.size)
    delta.reshape(-1)[:m] = special[:m]
    return xold, vel, delta


def _reference_parse(field: str) -> float:
    # the reference reader: 22 columns, D -> e, std::stod
    assert len(field) == 22
    return float(field.replace("D", "e"))


def test_round_trip_is_exact(tmp_path):
    n = 500
    xold, vel, delta = _state(n)
    p = tmp_path / "run.rst"
    api.write_restart_file(p, xold, vel, delta, box=[50.0, 50.0, 51.5], npriv=12340, ndegf=1497,
                           seed=2**63 + 12345, rngpos=4 * 12340)
    r = api.read_restart_file(p)
    assert r["natom"] == n and r["npriv"] == 12340 and r["ndegf"] == 1497
    assert r["seed"] == 2**63 + 12345 and r["rngpos"] == 4 * 12340
    np.testing.assert_array_equal(r["box"], [50.0, 50.0, 51.5])
    np.testing.assert_array_equal(r["xold"], xold)
    np.testing.assert_array_equal(r["vel"], vel)
    # every value is exact except a negative one below 1e-9 in magnitude,
    # which keeps 16 significant digits
    tiny_neg = (delta < 0) & (np.abs(delta) < 1e-9)
    np.testing.assert_array_equal(r["delta"][~tiny_neg], delta[~tiny_neg])
    np.testing.assert_allclose(r["delta"][tiny_neg], delta[tiny_neg], rtol=1e-15, atol=0)


def test_layout_follows_the_reference(tmp_path):
    n = 7
    xold, vel, delta = _state(n, seed=9)
    p = tmp_path / "lay.rst"
    api.write_restart_file(p, xold, vel, delta, box=[30.0, 31.0, 32.0], npriv=100, ndegf=18,
                           seed=42, rngpos=400)
    lines = p.read_text().split("\n")
    assert lines[0].startswith("REST    50     1  ORTH")
    assert api.read_restart_file(p)["crystal"] == "ORTH"
    assert lines[0][30:33] == "APO"
    assert lines[2] == "       2 !NTITLE followed by title"
    cry = lines.index(" !CRYSTAL PARAMETERS")
    xtl0, xtl1 = lines[cry + 1], lines[cry + 2]
    assert _reference_parse(xtl0[0:22]) == 30.0 and _reference_parse(xtl0[44:66]) == 31.0
    assert _reference_parse(xtl1[44:66]) == 32.0
    k = lines.index(" !NATOM,NPRIV,NSTEP,NSAVC,NSAVV,JHSTRT,NDEGF,SEED,NSAVL")
    ln = lines[k + 1]
    assert int(ln[0:12]) == n and int(ln[12:24]) == 100 and int(ln[24:36]) == 100
    assert int(ln[72:84]) == 18 and int(ln[84:106]) == 42 and int(ln[106:]) == 400
    stats = lines.index(" !ENERGIES and STATISTICS")
    assert lines[stats + 1] == "T" * 60 and lines[stats + 2] == "T" * 128
    for title, arr in ((" !XOLD, YOLD, ZOLD", xold), (" !VX, VY, VZ", vel), (" !X, Y, Z", delta)):
        s = lines.index(title)
        for i in range(n):
            row = lines[s + 1 + i]
            assert len(row) == 66
            got = [_reference_parse(row[22 * d: 22 * d + 22]) for d in range(3)]
            assert got == list(arr[i])  # the reference's reader gets the same doubles


def test_reads_the_reference_sixteen_digit_form(tmp_path):
    # a file in the reference writer's own number form: %.15E with D, width 22
    n = 5
    xold, vel, delta = _state(n, seed=3)
    delta = np.round(delta, 6)

    def f(v):
        return ("%.15E" % v).replace("E", "D").rjust(22)

    def tri(a):
        return "".join(f(v) for v in a) + "\n"

    head = ("REST    50     1  TETR          APO\n\n       2 !NTITLE followed by title\n"
            "* APOCHARMM RESTART FILE\n* USED FOR CONTINUING MOLECULAR DYNAMICS TRAJECTORY\n\n"
            " !CRYSTAL PARAMETERS\n")
    body = tri([40.0, 0.0, 40.0]) + tri([0.0, 0.0, 40.0]) + tri([1.5e-4, -2.25e-4, 0]) + tri([0, 0, 0])
    body += tri([0.0, 0.25, -0.5]) + tri([0, 0, 0]) * 8 + tri([0, 0, 0]) + f(0.0) + "\n\n"
    body += " !NATOM,NPRIV,NSTEP,NSAVC,NSAVV,JHSTRT,NDEGF,SEED,NSAVL\n"
    body += "".join(str(v).rjust(12) for v in (n, 2000, 2000, 1000, 0, 0, 9)) + "7".rjust(22)
    body += "  8000\n\n !ENERGIES and STATISTICS\n" + "T" * 60 + "\n" + "T" * 128 + "\n"
    body += "0".rjust(8) + f(0.0) + f(0.0) + f(301.5) + "\n"
    body += tri([0, 0, 0]) * 60 + (f(0) * 2 + "\n") * 60 + tri([0, 0, 0]) * 128
    body += (f(0) * 2 + "\n") * 128 + tri([0, 0, 0]) * 50 + (f(0) * 2 + "\n") * 50 + "\n"
    for title, arr in ((" !XOLD, YOLD, ZOLD", xold), (" !VX, VY, VZ", vel), (" !X, Y, Z", delta)):
        body += title + "\n" + "".join(tri(r) for r in arr) + "\n"
    p = tmp_path / "ref16.rst"
    p.write_text(head + body)
    r = api.read_restart_file(p)
    assert r["natom"] == n and r["npriv"] == 2000 and r["ndegf"] == 9
    assert r["seed"] == 7 and r["rngpos"] == 8000
    assert r["pnhv"] == 0.25 and r["pnhf"] == -0.5
    # the Langevin piston's part (src/CudaLangevinPistonIntegrator.cu:706-830)
    assert r["crystal"] == "TETR"
    np.testing.assert_array_equal(r["hdot"], [1.5e-4, -2.25e-4, 0.0])
    for key, arr in (("xold", xold), ("vel", vel), ("delta", delta)):
        want = np.array([[float(f(v).replace("D", "e")) for v in row] for row in arr])
        np.testing.assert_array_equal(r[key], want)


def test_errors(tmp_path):
    with pytest.raises(ApoError):
        api.read_restart_file(tmp_path / "missing.rst")
    bad = tmp_path / "bad.rst"
    bad.write_text("not a restart file\n")
    with pytest.raises(ApoError):
        api.read_restart_file(bad)
    xold, vel, delta = _state(4)
    p = tmp_path / "cut.rst"
    api.write_restart_file(p, xold, vel, delta, box=[20.0, 20.0, 20.0])
    text = p.read_text()
    (tmp_path / "cut2.rst").write_text(text[: text.index(" !X, Y, Z") + 12])
    with pytest.raises(ApoError):
        api.read_restart_file(tmp_path / "cut2.rst")
    with pytest.raises(ApoError):
        api.write_restart_file(p, xold, vel, np.full((4, 3), np.nan), box=[20.0, 20.0, 20.0])
    with pytest.raises(ApoError):
        api.RestartSubscriber(tmp_path / "no" / "such" / "dir.rst", 10)
