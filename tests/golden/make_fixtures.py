"""Regenerates the golden fixtures in this directory from the reference's tests.

Run once in a checkout that has the reference project next to it:

    python tests/golden/make_fixtures.py /path/to/reference

It reads the reference's own test inputs (test/data/*.psf, *.crd, the CHARMM
c47b1 force dumps) and stores them as compact arrays, and it records the known
answers that test/unittests/unittest-eneForces.cpp asserts:
  * waterDimer  :110-206 (energies +-1e-5, forces +-1e-4, virial 1e-4)
  * argon10     :208-286 (ePot -0.17984, forces +-1e-5, virial 1e-6)
  * waterbox    :288-365 (energies, virial 1e-4 rel, forces +-0.01)
Nothing here is needed at test time except the generated .npz/.json files.
"""
import json
import os
import sys

import numpy as np


def read_psf(path):
    with open(path) as f:
        lines = f.read().splitlines()
    out = {}
    i = 0
    while i < len(lines):
        tok = lines[i].split()
        if len(tok) == 2 and tok[1] == "!NATOM":
            n = int(tok[0])
            recs = [lines[i + 1 + k].split() for k in range(n)]
            out["seg"] = [r[1] for r in recs]
            out["resid"] = [int(r[2]) for r in recs]
            out["resn"] = [r[3] for r in recs]
            out["name"] = [r[4] for r in recs]
            out["type"] = [r[5] for r in recs]
            out["charge"] = np.array([float(r[6]) for r in recs])
            out["mass"] = np.array([float(r[7]) for r in recs])
            i += n + 1
            continue
        for key, width in (("!NBOND:", 2), ("!NTHETA:", 3), ("!NPHI:", 4), ("!NIMPHI:", 4)):
            if len(tok) >= 2 and tok[1] == key:
                cnt = int(tok[0])
                vals = []
                j = i + 1
                while len(vals) < cnt * width:
                    vals += [int(v) - 1 for v in lines[j].split()]
                    j += 1
                out[key] = np.array(vals, np.int32).reshape(-1, width)
                i = j - 1
        i += 1
    return out


def read_crd(path):
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    while lines[k].startswith("*"):
        k += 1
    tok = lines[k].split()
    n = int(tok[0])
    ext = len(tok) > 1 and tok[1] == "EXT"
    xyz = []
    for line in lines[k + 1:k + 1 + n]:
        if ext:
            xyz.append([float(line[40:60]), float(line[60:80]), float(line[80:100])])
        else:
            xyz.append([float(line[20:30]), float(line[30:40]), float(line[40:50])])
    return np.array(xyz)


def read_forces(path):
    out = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if len(t) == 3:
                out.append([float(v) for v in t])
    return np.array(out)


def main(ref):
    data = os.path.join(ref, "test", "data")
    here = os.path.dirname(os.path.abspath(__file__))
    cases = {
        "waterbox": ("waterbox.psf", "waterbox.crd", "waterbox.forces.c47b1.dat"),
        "waterDimer": ("waterDimer.psf", "waterDimer.crd", "waterDimer.forces.c47b1.dat"),
        "argon10": ("argon_10.psf", "argon_10.crd", None),
    }
    for name, (psf, crd, frc) in cases.items():
        p = read_psf(os.path.join(data, psf))
        arrays = dict(
            pos=read_crd(os.path.join(data, crd)),
            charge=p["charge"], mass=p["mass"],
            type_names=np.array(sorted(set(p["type"]))),
            type_index=np.array([sorted(set(p["type"])).index(t) for t in p["type"]], np.int16),
            atom_name=np.array(p["name"]), res_name=np.array(p["resn"]),
            res_id=np.array(p["resid"], np.int32), seg_id=np.array(p["seg"]),
            bonds=p["!NBOND:"], angles=p["!NTHETA:"],
        )
        if frc:
            arrays["forces_c47b1"] = read_forces(os.path.join(data, frc)).astype(np.float32)
        np.savez_compressed(os.path.join(here, f"{name}.npz"), **arrays)

    # known answers asserted by test/unittests/unittest-eneForces.cpp
    golden = {
        "waterbox": {
            "source": "test/unittests/unittest-eneForces.cpp:288-365",
            "box": 50.0, "nfft": [48, 48, 48], "kappa": 0.34, "cutoff": 10.0,
            "ctonnb": 7.0, "ctofnb": 8.0, "order": 4,
            "energy": {"epot": -49755.02125, "bond": 1915.85339, "angle": 1071.29551,
                       "vdw": 8697.43632, "elec": -56211.95319, "ewks": 156.45211,
                       "ewse": -260256.60420, "ewex": 254872.49980},
            "virial": [-7071.0775896888, -315.6040942237, -605.0510971046,
                       -315.6040942237, -6636.9115981748, -255.8901308852,
                       -605.0510971047, -255.8901308853, -6935.7815227056],
            "force_tol": 0.01,
        },
        "waterDimer": {
            "source": "test/unittests/unittest-eneForces.cpp:110-206",
            "box": 520.0, "nfft": [48, 48, 48], "kappa": 1e-8, "cutoff": 255.0,
            "ctonnb": 250.0, "ctofnb": 254.0, "order": 4,
            "energy": {"bond": 0.00003, "angle": 0.00002, "vdw": -0.00132,
                       "elec": 0.12185, "epot": 0.12057},
            "energy_margin": 1e-5,
            "virial": [0.4435916880, 0.0, 0.1160047166, 0.0, -0.0071274780, 0.0,
                       0.1160047166, 0.0, 0.0512243359],
            "force_tol": 1e-4,
        },
        "argon10": {
            "source": "test/unittests/unittest-eneForces.cpp:208-286",
            "box": 50.0, "nfft": [48, 48, 48], "kappa": 0.34, "cutoff": 9.0,
            "ctonnb": 7.0, "ctofnb": 8.0, "order": 4,
            "lj": {"AR": [-0.0240273, 2.285639]},
            "energy": {"epot": -0.17984},
            "forces": [[0.00567, -0.00087, -0.01986], [-0.00791, 0.00989, 0.00778],
                       [0.00513, -0.00134, 0.00932], [-0.00427, -0.00227, -0.00540],
                       [-0.00334, 0.00684, 0.01087], [-0.00301, -0.01385, -0.02313],
                       [0.01136, 0.00056, -0.00589], [-0.00778, 0.00468, 0.00800],
                       [0.00337, 0.00260, 0.00934], [0.00078, -0.00625, 0.00898]],
            "force_tol": 1e-5,
            "virial": [-0.0095837290, 0.0066020280, 0.0224834946, 0.0066020280,
                       -0.0307467278, -0.0684782285, 0.0224834946, -0.0684782285,
                       -0.0510912119],
        },
    }
    with open(os.path.join(here, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
