"""Runs the reference engine's own sm_100a build (oracle/_ref/ref_harness,
built by oracle/Makefile.ref from the reference sources) on CHARMM files."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
TERMS = ("bond", "angle", "ureyb", "dihe", "imdihe", "ewks", "ewse", "ewex", "elec", "vdw")


def available() -> bool:
    return os.path.exists(HARNESS)


def settings_args(box, st):
    return [str(box[0]), str(st["kappa"]), str(st["cutnb"]), str(st["ctonnb"]), str(st["ctofnb"]),
            str(st["nfft"][0]), str(st["nfft"][1]), str(st["nfft"][2]), str(st["order"])]


def forces(paths, box, st, out_path, timeout=600):
    cmd = [HARNESS, "forces", paths["psf"], paths["prm"], paths["crd"]] + settings_args(box, st) + [out_path]
    subprocess.run(cmd, check=True, timeout=timeout, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    with open(out_path) as f:
        e = [float(v) for v in f.readline().split()]
        g = np.loadtxt(f)
    return dict(zip(TERMS, e)), g


def md(paths, box, st, warmup, steps, seed=1, friction=1.0, timeout=1800):
    import json
    cmd = [HARNESS, "md", paths["psf"], paths["prm"], paths["crd"]] + settings_args(box, st) + \
        [str(warmup), str(steps), str(seed), str(friction)]
    r = subprocess.run(cmd, check=True, timeout=timeout, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True)
    for line in r.stdout.splitlines()[::-1]:
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError("reference harness printed no result: " + r.stdout[-2000:])


def traj(paths, box, st, kind, steps, seed, friction, velocities, workdir, timeout=900):
    """Runs `steps` steps of the reference's integrator `kind` from the CRD
    coordinates and the given (N,3) velocities; returns (x FP64, x FP32, v)."""
    vpath = os.path.join(workdir, f"v_{kind}.txt")
    np.savetxt(vpath, np.asarray(velocities, np.float64).reshape(-1), fmt="%.17g")
    out = os.path.join(workdir, f"traj_{kind}.txt")
    cmd = [HARNESS, "traj", paths["psf"], paths["prm"], paths["crd"]] + settings_args(box, st) + \
        [kind, str(steps), str(seed), str(friction), vpath, out]
    subprocess.run(cmd, check=True, timeout=timeout, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    a = np.loadtxt(out)
    return a[:, 0:3], a[:, 3:6], a[:, 6:9]


def piston(paths, box, st, steps, seed, friction, velocities, workdir, timeout=900, kind="piston"):
    """The reference's Langevin piston (1 atm, Nose-Hoover at 300 K, piston
    friction and seed as given; kind "piston" cubic, "piston_tetra",
    "piston_ortho", "piston_nonh" cubic without the thermostat):
    (x FP64, x FP32, v, final box)."""
    x, x32, v = traj(paths, box, st, kind, steps, seed, friction, velocities, workdir, timeout)
    b = np.loadtxt(os.path.join(workdir, f"traj_{kind}.txt.box"))
    return x, x32, v, b


def nblist(paths, box, st, radius, workdir, timeout=900):
    """The reference's tile-list pairs within `radius`: (i, j, excluded) rows."""
    out = os.path.join(workdir, "ref_pairs.bin")
    cmd = [HARNESS, "nblist", paths["psf"], paths["prm"], paths["crd"]] + settings_args(box, st) + \
        [str(radius), out]
    subprocess.run(cmd, check=True, timeout=timeout, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return np.fromfile(out, dtype=np.int32).reshape(-1, 3)
