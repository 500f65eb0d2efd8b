"""The C++ class surface (include/apocharmm/: ForceManager with
calcForce(xyzq, reset, calcEnergy, calcVirial) / getForces, ForceView
subscriptions, CudaBondedForce, CudaPMEDirectForce, CudaPMEReciprocalForce,
CudaNeighborList<32>, CharmmCrd, CharmmContext, the integrators and the
subscribers) compiled into user programs (tests/cpp/force_classes.cu,
tests/cpp/md_classes.cu) and linked against the library.

CPU: every header compiles on its own and the programs link.  GPU: the
force program runs on the ethylene-glycol box; the whole field and each part
match the FP64 oracle at the program's single-precision coordinates, the
parts add up to the whole in fixed point, a user force subscribed through
ForceView adds exactly its gradient and energy, and the list's index arrays
and pairs are consistent.  The MD program's Langevin run ends in the same
state, bit for bit, as the same run made through the Python API."""
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

from apocharmm_b200.systems import config_glycol, write_charmm_files
from parity_util import brute_force_pairs, oracle_for, rel_rms

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "apocharmm_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "force_classes.cu")
MD_SRC = os.path.join(ROOT, "tests", "cpp", "md_classes.cu")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CUDA_INC = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(NVCC))), "include")

FORCE_RTOL = 1e-5
ENERGY_RTOL = 1e-6


def build_program(out_dir, src=SRC):
    exe = os.path.join(out_dir, os.path.splitext(os.path.basename(src))[0])
    cmd = [NVCC, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-I", INC,
           src, "-L", LIBDIR, "-lapocharmm_c", "-Xlinker", "-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-4000:]
    return exe


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not found")
def test_headers_compile_alone(tmp_path):
    for h in sorted(glob.glob(os.path.join(INC, "apocharmm", "*.h"))):
        src = tmp_path / "one.cpp"
        src.write_text(f'#include "apocharmm/{os.path.basename(h)}"\nint main() {{ return 0; }}\n')
        r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", "-I", INC,
                            "-I", CUDA_INC, str(src)], stdout=subprocess.PIPE,
                           stderr=subprocess.STDOUT, text=True, timeout=120)
        assert r.returncode == 0, (h, r.stdout[-3000:])


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not found")
def test_program_links(tmp_path):
    assert os.path.exists(os.path.join(LIBDIR, "libapocharmm_c.so"))
    build_program(str(tmp_path))
    build_program(str(tmp_path), MD_SRC)


def _results(path):
    out = {"total": {}, "part": {}}
    for line in open(path):
        f = line.split()
        if not f:
            continue
        if f[0] == "total":
            out["total"][f[1]] = float(f[2])
        elif f[0] == "part":
            out["part"][(int(f[1]), f[2])] = float(f[3])
        else:
            out[f[0]] = [float(x) for x in f[1:]]
    return out


@pytest.mark.gpu
def test_force_classes_against_oracle(tmp_path):
    exe = build_program(str(tmp_path))
    s = config_glycol()
    st = s.settings
    paths = write_charmm_files(s, str(tmp_path))
    xyzq = np.zeros((s.n_atoms, 4), np.float32)
    xyzq[:, :3] = s.pos
    xyzq[:, 3] = s.charge
    xyzq.tofile(str(tmp_path / "xyzq.bin"))
    out = tmp_path / "out"
    out.mkdir()
    args = [exe, paths["psf"], paths["prm"], str(tmp_path / "xyzq.bin"), repr(s.box[0]),
            repr(st["kappa"]), repr(st["cutnb"]), repr(st["ctonnb"]), repr(st["ctofnb"]),
            str(st["nfft"][0]), str(st["nfft"][1]), str(st["nfft"][2]), str(st["order"]), str(out)]
    r = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-4000:]
    res = _results(out / "results.txt")
    assert res["done"] == []

    def grad(name):
        return np.fromfile(out / f"{name}.bin", np.float64).reshape(-1, 3)

    pos32 = xyzq[:, :3].astype(np.float64)
    o = oracle_for(s)
    Eo, Go = o.evaluate(pos=pos32)
    G = grad("total")
    assert rel_rms(G, Go) < FORCE_RTOL
    assert sum(res["total"].values()) == pytest.approx(Eo["epot"], rel=ENERGY_RTOL)
    assert len(res["virial"]) == 9 and np.isfinite(res["virial"]).all()

    # parts: bonded terms / direct space with 1-4 and exclusions / reciprocal with self
    parts = {1 | 8: ("bonded.bin", ("bonded",), ("bond", "angle", "ureyb", "dihe", "imdihe")),
             2 | 8: ("direct.bin", ("direct", "14"), ("elec", "vdw", "ewex")),
             4: ("recip.bin", ("recip", "self"), ("ewks", "ewse"))}
    # each part's error measured against the whole field's norm: the
    # bonded part alone is small (bond forces near equilibrium) and carries
    # the single-precision rounding of its bond lengths, ~1e-5 kcal/mol/A
    # absolute, which is what the whole-field bar allows
    norm = np.sqrt((Go ** 2).sum())
    total = np.zeros_like(G)
    for comp, (fname, oparts, terms) in parts.items():
        Gp = grad(fname[:-4])
        Ep, Gop = o.evaluate(pos=pos32, parts=oparts)
        assert np.sqrt(((Gp - Gop) ** 2).sum()) < FORCE_RTOL * norm, oparts
        esum = sum(res["part"][(comp, t)] for t in terms)
        assert esum == pytest.approx(Ep["epot"], abs=ENERGY_RTOL * abs(Eo["epot"])), oparts
        for t in terms:
            assert res["part"][(comp, t)] == pytest.approx(res["total"][t], rel=1e-12, abs=1e-9), t
        total += Gp
    # the parts add up to the whole (fixed-point sums of the same terms)
    np.testing.assert_allclose(total, G, rtol=0, atol=1e-9)

    # the tile list: index arrays invert each other; list pairs within the
    # cut-off agree with a brute-force search up to rounding at the radius
    assert res["list"][0] == 1 and res["glo2loc_roundtrip"] == [1.0]
    nslots, ntiles, nwork = res["list"][1:]
    assert nslots >= s.n_atoms and nslots % 32 == 0 and ntiles > 0 and nwork > 0
    ref = brute_force_pairs(pos32, s.box, st["ctofnb"], o.eptr, o.eidx)
    npairs, nexcl = res["pairs"]
    assert abs((npairs - nexcl) - len(ref)) <= 10

    # ForceView: E = k sum |r|^2 with k = 0.05 on the single-precision coordinates
    k = 0.05
    Gw = grad("with_well")
    np.testing.assert_allclose(Gw - G, 2 * k * pos32, rtol=0, atol=2e-9)
    assert res["well_energy"][0] == pytest.approx(k * float((pos32 ** 2).sum()), rel=1e-9)
    assert res["well_calls"] == [1.0, 1.0]  # initialised on subscription, evaluated once
    np.testing.assert_array_equal(grad("after_unsubscribe"), G)
    assert res["after_unsubscribe_has_well"] == [0.0]
    assert res["bad_cutoff_exception"] == [1.0]


MD_SETTINGS = dict(kappa=0.34, nfft=(24, 24, 24), order=4, ctofnb=9.0, ctonnb=7.5, cutnb=11.0)


@pytest.mark.gpu
def test_md_classes_match_python_api(tmp_path):
    """CharmmContext + CudaLangevinThermostatIntegrator + Dcd/Restart
    subscribers in C++ against the same calls through the Python API: the
    same library underneath, so positions, velocities, forces, energies and
    the restart file agree exactly."""
    from apocharmm_b200 import api
    from apocharmm_b200.systems import water_box, write_crd

    exe = build_program(str(tmp_path), MD_SRC)
    s = water_box(1000, 31.0, seed=3)
    keep = api.system_context(s, str(tmp_path / "relax"), settings=MD_SETTINGS)
    api.relax(keep[3], api.water_indices(s), iterations=100)
    relaxed = keep[3].getCoordinates()
    del keep
    paths = write_charmm_files(s, str(tmp_path / "files"))
    write_crd(s, paths["crd"], pos=relaxed)
    st = MD_SETTINGS
    nsteps = 40
    out = tmp_path / "cpp"
    out.mkdir()
    args = [exe, paths["psf"], paths["prm"], paths["crd"], repr(s.box[0]), repr(st["kappa"]),
            repr(st["cutnb"]), repr(st["ctonnb"]), repr(st["ctofnb"]), str(st["nfft"][0]),
            str(st["nfft"][1]), str(st["nfft"][2]), str(st["order"]), str(nsteps), str(out)]
    r = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-4000:]
    res = {}
    energies = {}
    for line in open(out / "results.txt"):
        f = line.split()
        if f and f[0] == "energy":
            energies[f[1]] = float(f[2])
        elif f:
            res[f[0]] = f[1:]
    assert "done" in res

    # the same sequence through the Python API; the C++ setters take float,
    # as the reference's do, so the Python side is given the same float values
    f32 = lambda x: float(np.float32(x))  # noqa: E731
    psf = api.CharmmPsf(paths["psf"])
    prm = api.CharmmParameters(paths["prm"])
    fm = api.ForceManager(psf, prm)
    fm.setBoxDimensions(s.box)
    fm.setKappa(f32(st["kappa"]))
    fm.setCutoff(f32(st["cutnb"]))
    fm.setCtonnb(f32(st["ctonnb"]))
    fm.setCtofnb(f32(st["ctofnb"]))
    fm.setFFTGrid(*st["nfft"])
    fm.setPmeSplineOrder(st["order"])
    ctx = api.CharmmContext(fm)
    ctx.setCoordinates(api.CharmmCrd(paths["crd"]))
    ctx.setRandomSeedForVelocities(314159)
    ctx.assignVelocitiesAtTemperature(300.0)
    it = api.CudaLangevinThermostatIntegrator(0.002)
    it.setThermostatFriction(5.0)
    it.setReferenceTemperature(300.0)
    it.setThermostatRngSeed(1234)
    it.setCharmmContext(ctx)
    py = tmp_path / "py"
    py.mkdir()
    dcd = api.DcdSubscriber(str(py / "traj.dcd"), 10)
    rst = api.RestartSubscriber(str(py / "run.rst"), nsteps)
    it.subscribe(dcd)
    it.subscribe(rst)
    it.propagate(nsteps)

    n = s.n_atoms
    assert res["crd_atoms"] == [str(n), str(n)]
    assert int(res["ndegf"][0]) == ctx.getDegreesOfFreedom()
    assert res["report_frequency"] == ["10", str(nsteps), "5"]
    assert res["subscribers"] == ["2"]
    assert int(res["step"][0]) == nsteps == it.getCurrentPropagatedStep()
    assert int(res["rngpos"][0]) == it.getRngSequencePos()
    x_cpp = np.fromfile(out / "coords.bin", np.float64).reshape(-1, 3)
    v_cpp = np.fromfile(out / "velocities.bin", np.float64).reshape(-1, 3)
    np.testing.assert_array_equal(x_cpp, ctx.getCoordinates())
    np.testing.assert_array_equal(v_cpp, np.asarray(ctx.getVelocities()).reshape(-1, 3))
    assert float(res["temperature"][0]) == pytest.approx(ctx.computeTemperature(), rel=1e-6)

    ctx.calculateForces(True, True, True)
    e_py = ctx.getEnergyComponents()
    for k, v in energies.items():
        assert v == e_py[k], k
    np.testing.assert_array_equal(np.fromfile(out / "forces.bin", np.float64).reshape(-1, 3),
                                  ctx.getForces())
    a, b = api.read_restart_file(out / "run.rst"), api.read_restart_file(py / "run.rst")
    assert a["npriv"] == b["npriv"] == nsteps and a["rngpos"] == b["rngpos"]
    for key in ("xold", "vel", "delta", "box"):
        np.testing.assert_array_equal(a[key], b[key])
    assert os.path.getsize(out / "traj.dcd") == os.path.getsize(py / "traj.dcd") > 0
    assert res["leapfrog_step"] == ["5"]
    pb = [float(x) for x in res["piston_box"]]
    assert pb[0] == pb[1] == pb[2] and pb[0] != s.box[0]
    assert np.isfinite(float(res["piston_pressure"][0])) and res["piston_pressure"][1:] == ["1", "15"]
