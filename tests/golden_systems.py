"""Builds System objects from the golden fixtures of the reference's tests."""
import json
import os

import numpy as np

from apocharmm_b200.systems import System, _water_params

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden():
    with open(os.path.join(HERE, "golden.json")) as f:
        return json.load(f)


def load_case(name: str) -> System:
    """Fixture arrays + the parameters the reference test reads from
    test/data/toppar_water_ions.str (water) or test/data/argon.prm (argon)."""
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    g = golden()[name]
    types = [str(t) for t in z["type_names"]]
    atom_type = [types[i] for i in z["type_index"]]
    L = float(g["box"])
    if name == "argon10":
        params = dict(masses_by_type={"AR": 39.948}, bond_params={}, angle_params={},
                      lj={"AR": tuple(g["lj"]["AR"])})
    else:
        params = _water_params()
    return System(
        name=name, box=(L, L, L), pos=np.array(z["pos"], np.float64),
        charge=np.array(z["charge"], np.float64), mass=np.array(z["mass"], np.float64),
        atom_type=atom_type, atom_name=[str(s) for s in z["atom_name"]],
        res_name=[str(s) for s in z["res_name"]], res_id=[int(v) for v in z["res_id"]],
        seg_id=[str(s) for s in z["seg_id"]],
        bonds=np.array(z["bonds"], np.int64).reshape(-1, 2),
        angles=np.array(z["angles"], np.int64).reshape(-1, 3),
        dihedrals=np.zeros((0, 4), np.int64), impropers=np.zeros((0, 4), np.int64),
        masses_by_type=params["masses_by_type"], bond_params=params["bond_params"],
        angle_params=params["angle_params"], dihedral_params={}, improper_params={},
        lj_params=params["lj"], lj14_params={},
        settings=dict(kappa=g["kappa"], nfft=tuple(g["nfft"]), order=g["order"],
                      ctofnb=g["ctofnb"], ctonnb=g["ctonnb"], cutnb=g["cutoff"]),
    )


def reference_forces(name: str):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    return np.array(z["forces_c47b1"], np.float64) if "forces_c47b1" in z else None
