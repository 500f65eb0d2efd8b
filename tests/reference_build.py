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
