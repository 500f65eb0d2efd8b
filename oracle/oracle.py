"""FP64 CPU oracle: topology assembly + ctypes front-end to apo_oracle.c.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``, always as the checker or the
timed CPU reference, never by the product package.

The topology functions restate the reference's host-side assembly:
  * exclusions, 1-4 inclusions, 1-2/1-3 exclusion corrections:
    CharmmPSF::buildTopologicalExclusions (src/CharmmPSF.cu:331-385) and
    CharmmPSF::getInclusionExclusionLists (src/CharmmPSF.cu:235-279);
  * LJ pair tables (sorted type set, eps = sqrt(ei ej), rmin = sum of rmin/2,
    NBFIX override, 1-4 variants): CharmmParameters::getVdwParamsAndTypes
    (src/CharmmParameters.cu:718-844);
  * bonded parameter lookup by atom types (bond/UB/angle/dihedral with the
    X-b-c-X wildcard): CharmmParameters::getBondedParamsAndLists
    (src/CharmmParameters.cu:357-700).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import Dict, List, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

CCELEC = 332.0716
KBOLTZ = 1.987191e-3


def build() -> str:
    """Compile the C oracle (gcc -O2 -fopenmp) next to this file."""
    src = os.path.join(_HERE, "apo_oracle.c")
    if (not os.path.exists(_LIB_PATH)
            or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared",
                               "-o", _LIB_PATH, src, "-lm"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        d = ctypes.c_double
        _lib.or_self_energy.restype = d
        _lib.or_bonds.restype = d
        _lib.or_angles.restype = d
        _lib.or_dihedrals.restype = d
        _lib.or_max_threads.restype = ctypes.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------
# topology (restated reference host assembly)
# ---------------------------------------------------------------------------

def connectivity(n: int, bonds: np.ndarray):
    c12 = [set() for _ in range(n)]
    for i, j in bonds:
        c12[i].add(int(j))
        c12[j].add(int(i))
    c13 = [set() for _ in range(n)]
    for i, j in bonds:
        for k in c12[j]:
            if k != i:
                c13[i].add(k)
        for k in c12[i]:
            if k != j:
                c13[j].add(k)
    c14 = [set() for _ in range(n)]
    for i in range(n):
        for j in c13[i]:
            for k in c12[j]:
                if k not in c12[i]:
                    c14[i].add(k)
    return c12, c13, c14


def exclusion_lists(n: int, bonds: np.ndarray):
    """Returns (excl CSR ptr, idx) symmetric over 1-2/1-3/1-4, in14, ex14."""
    c12, c13, c14 = connectivity(n, bonds)
    in14, ex14 = [], []
    pairs = []
    for i in range(n):
        for j in sorted(c14[i]):
            if j > i and j not in c12[i] and j not in c13[i]:
                in14.append((i, j))
        for j in sorted(c12[i] | c13[i]):
            if j > i:
                ex14.append((i, j))
        for j in sorted(c12[i] | c13[i] | c14[i]):
            if j > i:
                pairs.append((i, j))
    nbr = [[] for _ in range(n)]
    for i, j in pairs:
        nbr[i].append(j)
        nbr[j].append(i)
    ptr = np.zeros(n + 1, np.int32)
    for i in range(n):
        ptr[i + 1] = ptr[i] + len(nbr[i])
    idx = np.zeros(int(ptr[-1]), np.int32)
    for i in range(n):
        idx[ptr[i]:ptr[i + 1]] = sorted(nbr[i])
    return (ptr, idx, np.array(in14, np.int32).reshape(-1, 2),
            np.array(ex14, np.int32).reshape(-1, 2), pairs)


def lj_tables(atom_type: List[str], lj: Dict[str, Tuple[float, float]],
              lj14: Dict[str, Tuple[float, float]],
              nbfix: Dict[Tuple[str, str], Tuple[float, float]] | None = None):
    """Full (T,T,2) raw c6/c12 tables for main and 1-4 LJ plus per-atom type."""
    nbfix = nbfix or {}
    types = sorted(set(atom_type))
    T = len(types)
    tab = np.zeros((T, T, 2))
    tab14 = np.zeros((T, T, 2))
    for a in range(T):
        for b in range(a + 1):
            ti, tj = types[a], types[b]
            key = (tj, ti) if tj <= ti else (ti, tj)
            for which, target in ((0, tab), (1, tab14)):
                if key in nbfix:
                    eps, rmin = abs(nbfix[key][0]), nbfix[key][1]
                else:
                    ei, ri = lj[ti]
                    ej, rj = lj[tj]
                    if which == 1:
                        if ti in lj14:
                            ei, ri = lj14[ti]
                        if tj in lj14:
                            ej, rj = lj14[tj]
                    eps = math.sqrt(ei * ej)
                    rmin = ri + rj
                c12 = eps * rmin ** 12
                c6 = 2.0 * eps * rmin ** 6
                target[a, b] = target[b, a] = (c6, c12)
    tidx = np.array([types.index(t) for t in atom_type], np.int32)
    return types, tidx, tab, tab14


def bonded_terms(sys):
    """Per-term parameter arrays resolved from atom types (oracle layout)."""
    at = sys.atom_type
    kb, b0 = [], []
    for i, j in sys.bonds:
        a, b = sorted((at[i], at[j]))
        k, r0 = sys.bond_params[(a, b)]
        kb.append(k)
        b0.append(r0)
    kt, t0 = [], []
    for i, j, k in sys.angles:
        a, c = sorted((at[i], at[k]))
        kk, th = sys.angle_params[(a, at[j], c)]
        kt.append(kk)
        t0.append(math.radians(th))
    ub = getattr(sys, "ub_params", {}) or {}
    ub_list, ub_k, ub_s0 = [], [], []
    for i, j, k in sys.angles:
        a, c = sorted((at[i], at[k]))
        key = (a, at[j], c)
        if key in ub and abs(ub[key][0]) > 0.01:
            ub_list.append((i, k))
            ub_k.append(ub[key][0])
            ub_s0.append(ub[key][1])
    dptr, dk, dn, dd = [0], [], [], []
    for i, j, k, l in sys.dihedrals:
        a, b, c, d = at[i], at[j], at[k], at[l]
        if a > d or (a == d and b > c):
            a, b, c, d = d, c, b, a
        key = (a, b, c, d)
        if key not in sys.dihedral_params:
            b2, c2 = sorted((b, c))
            key = ("X", b2, c2, "X")
        for (kk, nn, dl) in sys.dihedral_params[key]:
            dk.append(kk)
            dn.append(nn)
            dd.append(math.radians(dl))
        dptr.append(len(dk))
    iptr, ik, idl = [0], [], []
    for i, j, k, l in sys.impropers:
        a, b, c, d = at[i], at[j], at[k], at[l]
        if a > d or (a == d and b > c):
            a, b, c, d = d, c, b, a
        kk, p0 = sys.improper_params[(a, b, c, d)]
        ik.append(kk)
        idl.append(math.radians(p0))
        iptr.append(len(ik))
    return dict(
        kb=np.array(kb), b0=np.array(b0), kt=np.array(kt), t0=np.array(t0),
        ub=np.array(ub_list, np.int32).reshape(-1, 2), ub_k=np.array(ub_k),
        ub_s0=np.array(ub_s0),
        dptr=np.array(dptr, np.int32), dk=np.array(dk), dn=np.array(dn, np.int32),
        dd=np.array(dd), iptr=np.array(iptr, np.int32), ik=np.array(ik),
        idl=np.array(idl), in_n=np.zeros(len(ik), np.int32))


# ---------------------------------------------------------------------------
# energy / gradient evaluation
# ---------------------------------------------------------------------------

class Oracle:
    """FP64 evaluation of one system (topology assembled once)."""

    def __init__(self, sys, kappa: float, roff: float, ron: float,
                 nfft: Tuple[int, int, int], order: int, nbfix=None):
        self.sys = sys
        self.n = sys.n_atoms
        self.kappa, self.roff, self.ron = float(kappa), float(roff), float(ron)
        self.nfft = tuple(int(v) for v in nfft)
        self.order = int(order)
        (self.eptr, self.eidx, self.in14, self.ex14, self.excl_pairs) = \
            exclusion_lists(self.n, np.asarray(sys.bonds))
        (self.types, self.tidx, self.tab, self.tab14) = lj_tables(
            sys.atom_type, sys.lj_params, sys.lj14_params, nbfix)
        self.bt = bonded_terms(sys)
        self.q = np.ascontiguousarray(sys.charge, np.float64)
        self.box = np.array(sys.box, np.float64)

    def evaluate(self, pos=None, nthreads: int = 0, parts=("bonded", "direct", "14", "recip", "self"),
                 virial: bool = False):
        """Energies (dict) and gradient (n, 3); with virial=True also the
        3x3 internal virial W = -sum over interactions of r (x) dU/dr, in
        the reference's convention (src/CudaEnergyVirial.cu:91-200 for the
        direct part, src/CudaPMERecip.cu:674-929 for the reciprocal part).
        Bonded and 1-4 terms use raw coordinate differences (whole
        molecules), so their virial is -sum_i x_i (x) g_i of their own
        gradient; the direct part sums -d (x) g over minimum-image pairs."""
        L = lib()
        xyz = np.ascontiguousarray(self.sys.pos if pos is None else pos, np.float64).reshape(-1)
        n = self.n
        grad_all = np.zeros(3 * n)
        vir = np.zeros(9)
        grad = np.zeros(3 * n) if virial else grad_all
        E = dict(bond=0.0, angle=0.0, ureyb=0.0, dihe=0.0, imdihe=0.0,
                 ewks=0.0, ewse=0.0, ewex=0.0, elec=0.0, vdw=0.0)
        bt = self.bt
        if "bonded" in parts:
            bonds = np.ascontiguousarray(self.sys.bonds, np.int32)
            E["bond"] = L.or_bonds(ctypes.c_int(len(bonds)), _p(bonds), _p(bt["kb"]),
                                   _p(bt["b0"]), _p(xyz), _p(grad))
            ub = np.ascontiguousarray(bt["ub"], np.int32)
            E["ureyb"] = L.or_bonds(ctypes.c_int(len(ub)), _p(ub), _p(bt["ub_k"]),
                                    _p(bt["ub_s0"]), _p(xyz), _p(grad))
            ang = np.ascontiguousarray(self.sys.angles, np.int32)
            E["angle"] = L.or_angles(ctypes.c_int(len(ang)), _p(ang), _p(bt["kt"]),
                                     _p(bt["t0"]), _p(xyz), _p(grad))
            dih = np.ascontiguousarray(self.sys.dihedrals, np.int32)
            E["dihe"] = L.or_dihedrals(ctypes.c_int(len(dih)), _p(dih), _p(bt["dptr"]),
                                       _p(bt["dk"]), _p(bt["dn"]), _p(bt["dd"]),
                                       ctypes.c_int(0), _p(xyz), _p(grad))
            imp = np.ascontiguousarray(self.sys.impropers, np.int32)
            E["imdihe"] = L.or_dihedrals(ctypes.c_int(len(imp)), _p(imp), _p(bt["iptr"]),
                                         _p(bt["ik"]), _p(bt["in_n"]), _p(bt["idl"]),
                                         ctypes.c_int(1), _p(xyz), _p(grad))
        if virial:
            x3 = xyz.reshape(n, 3)
            vir -= np.einsum("ia,ib->ab", x3, grad.reshape(n, 3)).reshape(-1)
            grad_all += grad
            grad = np.zeros(3 * n)
        ee, ev, ex = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        if "direct" in parts:
            tab = np.ascontiguousarray(self.tab)
            L.or_direct(ctypes.c_int(n), _p(xyz), _p(self.q), _p(self.tidx),
                        ctypes.c_int(len(self.types)), _p(tab), _p(self.eptr), _p(self.eidx),
                        _p(self.box), ctypes.c_double(self.kappa), ctypes.c_double(self.roff),
                        ctypes.c_double(self.ron), _p(grad), ctypes.byref(ee), ctypes.byref(ev),
                        _p(vir) if virial else None, ctypes.c_int(nthreads))
            E["elec"] += ee.value
            E["vdw"] += ev.value
            if virial:
                grad_all += grad
                grad = np.zeros(3 * n)
        if "14" in parts:
            in14 = np.ascontiguousarray(self.in14, np.int32)
            ex14 = np.ascontiguousarray(self.ex14, np.int32)
            tab14 = np.ascontiguousarray(self.tab14)
            L.or_14(ctypes.c_int(len(in14)), _p(in14), ctypes.c_int(len(ex14)), _p(ex14),
                    _p(xyz), _p(self.q), _p(self.tidx), ctypes.c_int(len(self.types)),
                    _p(tab14), ctypes.c_double(self.kappa), ctypes.c_double(self.roff),
                    ctypes.c_double(self.ron), _p(grad), ctypes.byref(ee), ctypes.byref(ev),
                    ctypes.byref(ex))
            E["elec"] += ee.value
            E["vdw"] += ev.value
            E["ewex"] += ex.value
            if virial:
                vir -= np.einsum("ia,ib->ab", xyz.reshape(n, 3), grad.reshape(n, 3)).reshape(-1)
                grad_all += grad
                grad = np.zeros(3 * n)
        if "recip" in parts:
            ek = ctypes.c_double()
            v6 = np.zeros(6)
            nx, ny, nz = self.nfft
            L.or_pme(ctypes.c_int(n), _p(xyz), _p(self.q), _p(self.box),
                     ctypes.c_double(self.kappa), ctypes.c_int(nx), ctypes.c_int(ny),
                     ctypes.c_int(nz), ctypes.c_int(self.order), _p(grad), ctypes.byref(ek),
                     _p(v6), ctypes.c_int(nthreads))
            E["ewks"] = ek.value
            if virial:
                vir += v6[[0, 1, 2, 1, 3, 4, 2, 4, 5]]
                grad_all += grad
                grad = np.zeros(3 * n)
        if "self" in parts:
            E["ewse"] = L.or_self_energy(ctypes.c_int(n), _p(self.q), ctypes.c_double(self.kappa))
        E["epot"] = sum(v for k, v in E.items())
        if virial:
            return E, grad_all.reshape(n, 3), vir.reshape(3, 3)
        return E, grad_all.reshape(n, 3)

    def ewald_recip_exact(self, pos=None, kmax=None, nthreads: int = 0):
        """Exact Ewald k-space sum (no mesh), for the PME error statement."""
        xyz = np.ascontiguousarray(self.sys.pos if pos is None else pos, np.float64).reshape(-1)
        if kmax is None:
            mmax = math.sqrt(40.0) * self.kappa / math.pi
            kmax = [int(math.ceil(mmax * b)) for b in self.box]
        grad = np.zeros(3 * self.n)
        e = ctypes.c_double()
        lib().or_ewald_recip(ctypes.c_int(self.n), _p(xyz), _p(self.q), _p(self.box),
                             ctypes.c_double(self.kappa), ctypes.c_int(kmax[0]),
                             ctypes.c_int(kmax[1]), ctypes.c_int(kmax[2]), _p(grad),
                             ctypes.byref(e), ctypes.c_int(nthreads))
        return e.value, grad.reshape(self.n, 3)


def degrees_of_freedom(n_atoms: int, n_water: int, n_shake_constraints: int,
                       holonomic: bool = True) -> int:
    """CharmmContext::useHolonomicConstraints (src/CharmmContext.cu:919-946)."""
    ndegf = 3 * n_atoms - 3
    if holonomic:
        ndegf -= 3 * n_water + n_shake_constraints
    return ndegf
