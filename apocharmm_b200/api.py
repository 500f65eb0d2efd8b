"""Python front-end over the C ABI, mirroring the reference's python/apocharmm
package (same class and method names: CharmmPsf, CharmmCrd, CharmmParameters,
ForceManager, CharmmContext, CudaNoseHooverIntegrator, ...), plus accessors
for forces, energies, coordinates and velocities that the reference exposes
only in C++.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Iterable, List, Sequence

import numpy as np

from ._lib import call, lib

ENERGY_TERMS = ("bond", "angle", "ureyb", "dihe", "imdihe", "ewks", "ewse", "ewex", "elec", "vdw")

_vp = ctypes.c_void_p
_d = ctypes.c_double
_i = ctypes.c_int
_sz = ctypes.c_size_t


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _enc(path) -> bytes:
    return os.fsencode(str(path))


class _Handle:
    _destroy = ""

    def __init__(self):
        self._h = _vp()

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h and self._h.value:
            getattr(lib(), self._destroy)(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class CharmmPsf(_Handle):
    _destroy = "apo_charmm_psf_destroy"

    def __init__(self, path):
        super().__init__()
        call("apo_charmm_psf_create", ctypes.byref(self._h), _enc(path))

    def _count(self, what):
        n = _sz()
        call(f"apo_charmm_psf_get_num_{what}", ctypes.byref(n), self._h)
        return n.value

    def getNumAtoms(self): return self._count("atoms")
    def getNumBonds(self): return self._count("bonds")
    def getNumAngles(self): return self._count("angles")
    def getNumDihedrals(self): return self._count("dihedrals")
    def getNumImpropers(self): return self._count("impropers")
    def getNumCrossTerms(self): return self._count("cross_terms")

    def _names(self, fn):
        n = self.getNumAtoms()
        buf = ctypes.create_string_buffer(8 * n)
        call(fn, buf, _sz(8 * n), self._h)
        raw = buf.raw.decode()
        return [raw[8 * i:8 * i + 8].strip() for i in range(n)]

    def getSegmentIdentifiers(self): return self._names("apo_charmm_psf_get_segment_identifiers")
    def getResidueNames(self): return self._names("apo_charmm_psf_get_residue_names")
    def getAtomNames(self): return self._names("apo_charmm_psf_get_atom_names")
    def getAtomTypes(self): return self._names("apo_charmm_psf_get_atom_types")

    def getResidueIdentifiers(self):
        n = self.getNumAtoms()
        a = np.zeros(n, np.int32)
        call("apo_charmm_psf_get_residue_identifiers", _ptr(a), _sz(n), self._h)
        return a.tolist()

    def getCharges(self):
        n = self.getNumAtoms()
        a = np.zeros(n)
        call("apo_charmm_psf_get_charges", _ptr(a), _sz(n), self._h)
        return a.tolist()

    def getMasses(self):
        n = self.getNumAtoms()
        a = np.zeros(n)
        call("apo_charmm_psf_get_masses", _ptr(a), _sz(n), self._h)
        return a.tolist()

    def getNetCharge(self):
        v = _d()
        call("apo_charmm_psf_get_net_charge", ctypes.byref(v), self._h)
        return v.value

    def getTotalMass(self):
        v = _d()
        call("apo_charmm_psf_get_total_mass", ctypes.byref(v), self._h)
        return v.value

    def getFileName(self):
        buf = ctypes.create_string_buffer(4096)
        call("apo_charmm_psf_get_file_name", buf, _sz(4096), self._h)
        return buf.value.decode()


class CharmmCrd(_Handle):
    _destroy = "apo_charmm_crd_destroy"

    def __init__(self, path):
        super().__init__()
        call("apo_charmm_crd_create", ctypes.byref(self._h), _enc(path))

    def getNumAtoms(self):
        n = _sz()
        call("apo_charmm_crd_get_num_atoms", ctypes.byref(n), self._h)
        return n.value

    def getCoordinates(self):
        n = self.getNumAtoms()
        a = np.zeros(3 * n)
        call("apo_charmm_crd_get_coordinates", _ptr(a), _sz(3 * n), self._h)
        return a.reshape(n, 3).tolist()


class CharmmParameters(_Handle):
    _destroy = "apo_charmm_parameters_destroy"

    def __init__(self, paths):
        super().__init__()
        if isinstance(paths, (str, bytes, os.PathLike)):
            call("apo_charmm_parameters_create", ctypes.byref(self._h), _enc(paths))
        else:
            enc = [_enc(p) for p in paths]
            arr = (ctypes.c_char_p * len(enc))(*enc)
            call("apo_charmm_parameters_create_from_files", ctypes.byref(self._h), arr,
                 _sz(len(enc)))


class ForceManager(_Handle):
    _destroy = "apo_force_manager_destroy"

    def __init__(self, psf: CharmmPsf, parameters: CharmmParameters):
        super().__init__()
        self._psf, self._prm = psf, parameters  # keep the inputs alive
        call("apo_force_manager_create", ctypes.byref(self._h), psf.handle, parameters.handle)

    def setBoxDimensions(self, box: Sequence[float]):
        call("apo_force_manager_set_box_dimensions", self._h, _d(box[0]), _d(box[1]), _d(box[2]))

    def getBoxDimensions(self) -> np.ndarray:
        """The box in force (A); the Langevin piston changes it every step."""
        a = np.zeros(3)
        call("apo_force_manager_get_box_dimensions", _ptr(a), _sz(3), self._h)
        return a

    def setKappa(self, v): call("apo_force_manager_set_kappa", self._h, _d(v))
    def setCutoff(self, v): call("apo_force_manager_set_cutoff", self._h, _d(v))
    def setCtonnb(self, v): call("apo_force_manager_set_ctonnb", self._h, _d(v))
    def setCtofnb(self, v): call("apo_force_manager_set_ctofnb", self._h, _d(v))
    def setPmeSplineOrder(self, v): call("apo_force_manager_set_spline_order", self._h, _i(v))
    def setFFTGrid(self, nx, ny, nz): call("apo_force_manager_set_fft_grid", self._h, _i(nx), _i(ny), _i(nz))
    def setPrecisionMode(self, on: bool): call("apo_force_manager_set_precision_mode", self._h, _i(int(on)))
    def setTilesPerWork(self, t: int): call("apo_force_manager_set_tiles_per_work", self._h, _i(t))
    def setWorkItemsPerWarp(self, k: int): call("apo_force_manager_set_work_items_per_warp", self._h, _i(k))
    def setComponentMask(self, m: int): call("apo_force_manager_set_component_mask", self._h, _i(m))
    def setDirectKernel(self, form: int): call("apo_force_manager_set_direct_kernel", self._h, _i(form))
    def setListCapacity(self, tiles: int): call("apo_force_manager_set_list_capacity", self._h, _i(tiles))
    def setPmeTensorCopies(self, on: bool): call("apo_force_manager_set_pme_tensor_copies", self._h, _i(int(on)))

    def getPmeTensorCopies(self) -> bool:
        v = _i()
        call("apo_force_manager_get_pme_tensor_copies", ctypes.byref(v), self._h)
        return bool(v.value)

    def getListCapacity(self) -> int:
        v = _i()
        call("apo_force_manager_get_list_capacity", ctypes.byref(v), self._h)
        return v.value

    def getFFTGrid(self):
        a = (ctypes.c_int * 3)()
        call("apo_force_manager_get_fft_grid", a, self._h)
        return list(a)

    def subscribe(self, force: "HarmonicRestraintForce", tag: str):
        """Adds a plug-in force to every evaluation; its energy is reported as `tag`."""
        self._plugins = getattr(self, "_plugins", {})
        call("apo_force_manager_subscribe_harmonic_restraint", self._h, force.handle, _enc(tag))
        self._plugins[tag] = force

    def unsubscribe(self, tag: str) -> bool:
        removed = _i()
        call("apo_force_manager_unsubscribe", ctypes.byref(removed), self._h, _enc(tag))
        getattr(self, "_plugins", {}).pop(tag, None)
        return bool(removed.value)


class HarmonicRestraintForce(_Handle):
    """E = sum k_i m_i |r_i - r0_i|^2 over the selected atoms (masses 1 unless set)."""

    _destroy = "apo_harmonic_restraint_force_destroy"

    def __init__(self, num_atoms: int):
        super().__init__()
        self._n = int(num_atoms)
        call("apo_harmonic_restraint_force_create", ctypes.byref(self._h), _i(self._n))

    def setSelection(self, atoms):
        a = np.ascontiguousarray(atoms, dtype=np.int32).reshape(-1)
        call("apo_harmonic_restraint_force_set_selection", self._h, _ptr(a), _sz(a.size))

    def setForceConstant(self, k: float):
        call("apo_harmonic_restraint_force_set_force_constant", self._h, _d(k))

    def _per_atom(self, fn, v, per):
        a = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        call(fn, self._h, _ptr(a), _sz(a.size))

    def setForceConstants(self, k):
        self._per_atom("apo_harmonic_restraint_force_set_force_constants", k, 1)

    def setReferenceCoordinates(self, xyz):
        self._per_atom("apo_harmonic_restraint_force_set_reference_coordinates", xyz, 3)

    def setMasses(self, m):
        self._per_atom("apo_harmonic_restraint_force_set_masses", m, 1)


class CharmmContext(_Handle):
    _destroy = "apo_charmm_context_destroy"

    def __init__(self, force_manager: ForceManager):
        super().__init__()
        self._fm = force_manager
        call("apo_charmm_context_create", ctypes.byref(self._h), force_manager.handle)

    def setCoordinates(self, crd):
        if isinstance(crd, CharmmCrd):
            call("apo_charmm_context_set_coordinates", self._h, crd.handle)
        else:
            a = np.ascontiguousarray(crd, np.float64).reshape(-1)
            call("apo_charmm_context_set_coordinates_xyz", self._h, _ptr(a), _sz(a.size))

    def setRandomSeedForVelocities(self, seed: int):
        call("apo_charmm_context_set_random_seed_for_velocities", self._h, ctypes.c_uint64(seed))

    def useHolonomicConstraints(self, flag: bool):
        call("apo_charmm_context_use_holonomic_constraints", self._h, ctypes.c_bool(flag))

    def assignVelocitiesAtTemperature(self, t: float):
        call("apo_charmm_context_assign_velocities_at_temperature", self._h, _d(t))

    def computeTemperature(self) -> float:
        v = _d()
        call("apo_charmm_context_compute_temperature", ctypes.byref(v), self._h)
        return v.value

    def getNumAtoms(self) -> int:
        n = _sz()
        call("apo_charmm_context_get_num_atoms", ctypes.byref(n), self._h)
        return n.value

    def getDegreesOfFreedom(self) -> int:
        n = _i()
        call("apo_charmm_context_get_degrees_of_freedom", ctypes.byref(n), self._h)
        return n.value

    def calculateForces(self, reset: bool = False, calcEnergy: bool = True, calcVirial: bool = False):
        call("apo_charmm_context_calculate_forces", self._h, ctypes.c_bool(reset),
             ctypes.c_bool(calcEnergy), ctypes.c_bool(calcVirial))

    def calculatePotentialEnergy(self, reset: bool = False) -> float:
        self.calculateForces(reset, True, False)
        return self.getPotentialEnergy()

    def getForces(self) -> np.ndarray:
        """Total gradient dU/dx, (N,3), the reference's force-buffer sign."""
        n = self.getNumAtoms()
        a = np.zeros(3 * n)
        call("apo_charmm_context_get_forces", _ptr(a), _sz(3 * n), self._h)
        return a.reshape(n, 3)

    def getEnergyComponents(self) -> Dict[str, float]:
        a = np.zeros(len(ENERGY_TERMS))
        call("apo_charmm_context_get_energy_components", _ptr(a), _sz(a.size), self._h)
        return dict(zip(ENERGY_TERMS, a.tolist()))

    def getPotentialEnergy(self) -> float:
        v = _d()
        call("apo_charmm_context_get_potential_energy", ctypes.byref(v), self._h)
        return v.value

    def getEnergyComponent(self, name: str) -> float:
        """A built-in energy term or a plug-in force's energy, by name."""
        v = _d()
        call("apo_charmm_context_get_energy_component", ctypes.byref(v), self._h, _enc(name))
        return v.value

    def getVirial(self) -> np.ndarray:
        """3x3 internal virial of the last evaluation made with calc_virial."""
        a = np.zeros(9)
        call("apo_charmm_context_get_virial", _ptr(a), _sz(9), self._h)
        return a.reshape(3, 3)

    def getCoordinates(self) -> np.ndarray:
        n = self.getNumAtoms()
        a = np.zeros(3 * n)
        call("apo_charmm_context_get_coordinates", _ptr(a), _sz(3 * n), self._h)
        return a.reshape(n, 3)

    def setVelocities(self, v):
        a = np.ascontiguousarray(v, np.float64).reshape(-1)
        call("apo_charmm_context_set_velocities", self._h, _ptr(a), _sz(a.size))

    def getVelocities(self) -> np.ndarray:
        n = self.getNumAtoms()
        a = np.zeros(3 * n)
        call("apo_charmm_context_get_velocities", _ptr(a), _sz(3 * n), self._h)
        return a.reshape(n, 3)

    def resetNeighborList(self):
        call("apo_charmm_context_reset_neighbor_list", self._h)

    def getNeighborPairs(self, radius: float) -> np.ndarray:
        n = _sz()
        call("apo_charmm_context_get_neighbor_pairs", None, _sz(0), ctypes.byref(n), _d(radius), self._h)
        a = np.zeros(3 * max(1, n.value), np.int32)
        call("apo_charmm_context_get_neighbor_pairs", _ptr(a), _sz(a.size), ctypes.byref(n),
             _d(radius), self._h)
        return a[:3 * n.value].reshape(-1, 3)

    def getListPairs(self, radius: float) -> np.ndarray:
        """Every pair of the tile list within `radius`: (i, j, excluded) rows."""
        n = _sz()
        call("apo_charmm_context_get_list_pairs", None, _sz(0), ctypes.byref(n), _d(radius), self._h)
        a = np.zeros(3 * max(1, n.value), np.int32)
        call("apo_charmm_context_get_list_pairs", _ptr(a), _sz(a.size), ctypes.byref(n),
             _d(radius), self._h)
        return a[:3 * n.value].reshape(-1, 3)

    def getStream(self) -> int:
        p = _vp()
        call("apo_charmm_context_get_stream", ctypes.byref(p), self._h)
        return p.value or 0


def system_context(sys, workdir: str, precise: bool = False, settings=None,
                   tiles_per_work: int = None, items_per_warp: int = None):
    """Writes `sys` (apocharmm_b200.systems.System) as CHARMM files, loads it
    through the C ABI and returns (psf, prm, fm, ctx).  `settings` overrides
    sys.settings (kappa, nfft, order, ctofnb, ctonnb, cutnb)."""
    from .systems import write_charmm_files
    st = dict(sys.settings)
    st.update(settings or {})
    paths = write_charmm_files(sys, workdir)
    psf = CharmmPsf(paths["psf"])
    prm = CharmmParameters(paths["prm"])
    fm = ForceManager(psf, prm)
    fm.setBoxDimensions(sys.box)
    fm.setKappa(st["kappa"])
    fm.setCutoff(st["cutnb"])
    fm.setCtonnb(st["ctonnb"])
    fm.setCtofnb(st["ctofnb"])
    fm.setFFTGrid(*st["nfft"])
    fm.setPmeSplineOrder(st["order"])
    fm.setPrecisionMode(precise)
    if tiles_per_work is not None:
        fm.setTilesPerWork(tiles_per_work)
    if items_per_warp is not None:
        fm.setWorkItemsPerWarp(items_per_warp)
    ctx = CharmmContext(fm)
    ctx.setCoordinates(sys.pos)
    return psf, prm, fm, ctx


class Subscriber(_Handle):
    """Borrowed base view of a concrete subscriber (owned by the subclass)."""

    def __init__(self):
        super().__init__()
        self._view = _vp()

    def setReportFrequency(self, f: int):
        call("apo_subscriber_set_report_frequency", self._view, _i(f))

    def getReportFrequency(self) -> int:
        v = _i()
        call("apo_subscriber_get_report_frequency", ctypes.byref(v), self._view)
        return v.value


class DcdSubscriber(Subscriber):
    _destroy = "apo_dcd_subscriber_destroy"

    def __init__(self, path, report_frequency: int | None = None):
        super().__init__()
        if report_frequency is None:
            call("apo_dcd_subscriber_create", ctypes.byref(self._h), _enc(path))
        else:
            call("apo_dcd_subscriber_create_with_report_frequency", ctypes.byref(self._h),
                 _enc(path), _i(report_frequency))
        call("apo_dcd_subscriber_as_subscriber", ctypes.byref(self._view), self._h)


class RestartSubscriber(Subscriber):
    """Rewrites a CHARMM-layout restart file every `report_frequency` steps
    (Langevin thermostat and Nose-Hoover integrators)."""

    _destroy = "apo_restart_subscriber_destroy"

    def __init__(self, path, report_frequency: int | None = None):
        super().__init__()
        if report_frequency is None:
            call("apo_restart_subscriber_create", ctypes.byref(self._h), _enc(path))
        else:
            call("apo_restart_subscriber_create_with_report_frequency", ctypes.byref(self._h),
                 _enc(path), _i(report_frequency))
        call("apo_restart_subscriber_as_subscriber", ctypes.byref(self._view), self._h)


def read_restart_file(path) -> dict:
    """Scalars and per-atom sections of a restart file (no device needed)."""
    natom, ndegf, has_rng = _i(), _i(), _i()
    npriv = ctypes.c_longlong()
    seed, rngpos = ctypes.c_ulonglong(), ctypes.c_ulonglong()
    box = np.zeros(3)
    pnhv, pnhf = _d(), _d()
    call("apo_restart_file_read_header", _enc(path), ctypes.byref(natom), ctypes.byref(npriv),
         ctypes.byref(ndegf), ctypes.byref(seed), ctypes.byref(rngpos), ctypes.byref(has_rng),
         _ptr(box), ctypes.byref(pnhv), ctypes.byref(pnhf))
    n = natom.value
    xold, vel, delta = (np.zeros((max(n, 1), 3)) for _ in range(3))
    call("apo_restart_file_read", _enc(path), _i(n), _ptr(xold), _ptr(vel), _ptr(delta))
    crystal = ctypes.create_string_buffer(5)
    hdot = np.zeros(3)
    call("apo_restart_file_read_crystal", _enc(path), crystal, _ptr(hdot))
    return {"natom": n, "npriv": npriv.value, "ndegf": ndegf.value, "seed": seed.value,
            "rngpos": rngpos.value if has_rng.value else None, "box": box,
            "pnhv": pnhv.value, "pnhf": pnhf.value, "crystal": crystal.value.decode(),
            "hdot": hdot, "xold": xold[:n], "vel": vel[:n], "delta": delta[:n]}


def write_restart_file(path, xold, vel, delta, box, npriv: int = 0, ndegf: int = 0,
                       seed: int = 0, rngpos: int | None = None, pnhv: float = 0.0,
                       pnhf: float = 0.0):
    """Writes a restart file from host arrays (natom x 3 each)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 3) for a in (xold, vel, delta)]
    n = arrs[0].shape[0]
    if any(a.shape[0] != n for a in arrs):
        raise ValueError("xold, vel and delta must have the same number of atoms")
    b = np.ascontiguousarray(box, dtype=np.float64).reshape(3)
    call("apo_restart_file_write", _enc(path), _i(n), ctypes.c_longlong(npriv), _i(ndegf),
         ctypes.c_ulonglong(seed), ctypes.c_ulonglong(rngpos or 0), _i(rngpos is not None),
         _ptr(b), _d(pnhv), _d(pnhf), _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]))


class CudaIntegrator(_Handle):
    """Base of the integrators; `_view` is the borrowed apo_cuda_integrator."""

    _as_base = ""

    def __init__(self):
        super().__init__()
        self._view = _vp()
        self._keep = []

    def _bind_view(self):
        call(self._as_base, ctypes.byref(self._view), self._h)

    def setTimeStep(self, dt_ps: float):
        call("apo_cuda_integrator_set_time_step", self._view, _d(dt_ps))

    def setCharmmContext(self, context: CharmmContext):
        self._keep.append(context)
        call("apo_cuda_integrator_set_charmm_context", self._view, context.handle)

    def subscribe(self, subscriber: Subscriber):
        self._keep.append(subscriber)
        call("apo_cuda_integrator_subscribe", self._view, subscriber._view)

    def unsubscribe(self, subscriber: Subscriber) -> bool:
        removed = _i()
        call("apo_cuda_integrator_unsubscribe", ctypes.byref(removed), self._view, subscriber._view)
        return bool(removed.value)

    def propagate(self, num_steps: int):
        call("apo_cuda_integrator_propagate", self._view, _i(num_steps))

    def initializeFromRestartFile(self, path):
        call("apo_cuda_integrator_initialize_from_restart_file", self._view, _enc(path))

    def setNonbondedListUpdateFrequency(self, f: int):
        call("apo_cuda_integrator_set_nonbonded_list_update_frequency", self._view, _i(f))

    def setUseGraphs(self, on: bool):
        call("apo_cuda_integrator_set_use_graphs", self._view, _i(int(on)))

    def getCurrentPropagatedStep(self) -> int:
        v = ctypes.c_longlong()
        call("apo_cuda_integrator_get_current_step", ctypes.byref(v), self._view)
        return v.value

    def getAverageTemperature(self) -> float:
        v = _d()
        call("apo_cuda_integrator_get_average_temperature", ctypes.byref(v), self._view)
        return v.value

    def getInstantaneousTemperature(self) -> float:
        v = _d()
        call("apo_cuda_integrator_get_instantaneous_temperature", ctypes.byref(v), self._view)
        return v.value

    def getKernelsPerStep(self) -> int:
        v = _i()
        call("apo_cuda_integrator_get_kernels_per_step", ctypes.byref(v), self._view)
        return v.value


class CudaNoseHooverIntegrator(CudaIntegrator):
    _destroy = "apo_cuda_nose_hoover_integrator_destroy"
    _as_base = "apo_cuda_nose_hoover_integrator_as_cuda_integrator"

    def __init__(self, time_step: float):
        super().__init__()
        call("apo_cuda_nose_hoover_integrator_create", ctypes.byref(self._h), _d(time_step))
        self._bind_view()

    def setReferenceTemperature(self, t: float):
        call("apo_cuda_nose_hoover_integrator_set_reference_temperature", self._h, _d(t))

    def setNoseHooverPistonMass(self, m: float):
        call("apo_cuda_nose_hoover_integrator_set_nose_hoover_piston_mass", self._h, _d(m))

    def useOldTemperature(self, flag: bool = True):
        call("apo_cuda_nose_hoover_integrator_use_old_temperature", self._h, ctypes.c_bool(flag))

    def resetAverageTemperature(self):
        call("apo_cuda_nose_hoover_integrator_reset_average_temperature", self._h)

    def getReferenceTemperature(self) -> float:
        v = _d()
        call("apo_cuda_nose_hoover_integrator_get_reference_temperature", ctypes.byref(v), self._h)
        return v.value


class CudaLangevinThermostatIntegrator(CudaIntegrator):
    _destroy = "apo_cuda_langevin_thermostat_integrator_destroy"
    _as_base = "apo_cuda_langevin_thermostat_integrator_as_cuda_integrator"

    def __init__(self, time_step: float):
        super().__init__()
        call("apo_cuda_langevin_thermostat_integrator_create", ctypes.byref(self._h), _d(time_step))
        self._bind_view()

    def setThermostatFriction(self, f: float):
        call("apo_cuda_langevin_thermostat_integrator_set_thermostat_friction", self._h, _d(f))

    def setReferenceTemperature(self, t: float):
        call("apo_cuda_langevin_thermostat_integrator_set_reference_temperature", self._h, _d(t))

    def setThermostatRngSeed(self, seed: int):
        call("apo_cuda_langevin_thermostat_integrator_set_thermostat_rng_seed", self._h,
             ctypes.c_uint64(seed))

    def getRngSequencePos(self) -> int:
        v = ctypes.c_ulonglong()
        call("apo_cuda_langevin_thermostat_integrator_get_rng_sequence_pos", ctypes.byref(v), self._h)
        return v.value


class CudaLeapFrogIntegrator(CudaIntegrator):
    _destroy = "apo_cuda_leap_frog_integrator_destroy"
    _as_base = "apo_cuda_leap_frog_integrator_as_cuda_integrator"

    def __init__(self, time_step: float):
        super().__init__()
        call("apo_cuda_leap_frog_integrator_create", ctypes.byref(self._h), _d(time_step))
        self._bind_view()


class CudaLangevinPistonIntegrator(CudaIntegrator):
    """Constant pressure (Langevin piston on the box edges, optional
    Nose-Hoover thermostat): include/CudaLangevinPistonIntegrator.h.
    Crystal types 1 cubic, 2 orthorhombic, 3 tetragonal (enum CRYSTAL);
    pressures in atm, 3x3 row major."""

    _destroy = "apo_cuda_langevin_piston_integrator_destroy"
    _as_base = "apo_cuda_langevin_piston_integrator_as_cuda_integrator"
    CUBIC, ORTHORHOMBIC, TETRAGONAL = 1, 2, 3

    def __init__(self, time_step: float):
        super().__init__()
        call("apo_cuda_langevin_piston_integrator_create", ctypes.byref(self._h), _d(time_step))
        self._bind_view()

    def setCrystalType(self, crystal: int):
        call("apo_cuda_langevin_piston_integrator_set_crystal_type", self._h, _i(crystal))

    def setPressure(self, p):
        a = np.ascontiguousarray(p, np.float64).reshape(-1)
        call("apo_cuda_langevin_piston_integrator_set_pressure", self._h, _ptr(a), _sz(a.size))

    def setLangevinPistonMass(self, m):
        a = np.ascontiguousarray(m, np.float64).reshape(-1)
        call("apo_cuda_langevin_piston_integrator_set_langevin_piston_mass", self._h, _ptr(a),
             _sz(a.size))

    def getLangevinPistonMass(self) -> np.ndarray:
        a, n = np.zeros(3), _sz()
        call("apo_cuda_langevin_piston_integrator_get_langevin_piston_mass", _ptr(a), _sz(3),
             ctypes.byref(n), self._h)
        return a[:n.value]

    def setLangevinPistonFriction(self, g: float):
        call("apo_cuda_langevin_piston_integrator_set_langevin_piston_friction", self._h, _d(g))

    def setLangevinPistonFrictionSeed(self, seed: int):
        call("apo_cuda_langevin_piston_integrator_set_langevin_piston_friction_seed", self._h,
             ctypes.c_uint64(seed))

    def setRngSequencePos(self, pos: int):
        call("apo_cuda_langevin_piston_integrator_set_rng_sequence_pos", self._h,
             ctypes.c_ulonglong(pos))

    def getRngSequencePos(self) -> int:
        v = ctypes.c_ulonglong()
        call("apo_cuda_langevin_piston_integrator_get_rng_sequence_pos", ctypes.byref(v), self._h)
        return v.value

    def setReferenceTemperature(self, t: float):
        call("apo_cuda_langevin_piston_integrator_set_reference_temperature", self._h, _d(t))

    def useNoseHooverThermostat(self, flag: bool = True):
        call("apo_cuda_langevin_piston_integrator_use_nose_hoover_thermostat", self._h,
             ctypes.c_bool(flag))

    def setNoseHooverPistonMass(self, m: float):
        call("apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_mass", self._h, _d(m))

    def useOldTemperature(self, flag: bool = True):
        call("apo_cuda_langevin_piston_integrator_use_old_temperature", self._h, ctypes.c_bool(flag))

    def setMaxPredictorCorrectorIterations(self, n: int):
        call("apo_cuda_langevin_piston_integrator_set_max_predictor_corrector_iterations", self._h,
             _i(n))

    def setConstantSurfaceTension(self, flag: bool, tension: float = 0.0):
        call("apo_cuda_langevin_piston_integrator_set_constant_surface_tension", self._h,
             ctypes.c_bool(flag), _d(tension))

    def resetAverages(self):
        call("apo_cuda_langevin_piston_integrator_reset_averages", self._h)

    def _tensor(self, name) -> np.ndarray:
        a = np.zeros(9)
        call(name, _ptr(a), _sz(9), self._h)
        return a.reshape(3, 3)

    def getInstantaneousPressureTensor(self) -> np.ndarray:
        return self._tensor("apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_tensor")

    def getAveragePressureTensor(self) -> np.ndarray:
        return self._tensor("apo_cuda_langevin_piston_integrator_get_average_pressure_tensor")

    def getInstantaneousPressureScalar(self) -> float:
        v = _d()
        call("apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_scalar",
             ctypes.byref(v), self._h)
        return v.value

    def getAveragePressureScalar(self) -> float:
        v = _d()
        call("apo_cuda_langevin_piston_integrator_get_average_pressure_scalar", ctypes.byref(v),
             self._h)
        return v.value

    def _vector(self, what) -> np.ndarray:
        a, n = np.zeros(3), _sz()
        call(f"apo_cuda_langevin_piston_integrator_get_langevin_piston_{what}", _ptr(a), _sz(3),
             ctypes.byref(n), self._h)
        return a[:n.value]

    def getLangevinPistonOnStepPosition(self) -> np.ndarray:
        return self._vector("on_step_position")

    def getLangevinPistonHalfStepPosition(self) -> np.ndarray:
        return self._vector("half_step_position")

    def getLangevinPistonOnStepVelocity(self) -> np.ndarray:
        return self._vector("on_step_velocity")

    def getLangevinPistonDeltaPosition(self) -> np.ndarray:
        return self._vector("delta_position")

    def getLangevinPistonDeltaPressure(self) -> np.ndarray:
        return self._vector("delta_pressure")

    def getInstantaneousSurfaceTension(self) -> float:
        v = _d()
        call("apo_cuda_langevin_piston_integrator_get_instantaneous_surface_tension",
             ctypes.byref(v), self._h)
        return v.value

    def getCrystalType(self) -> int:
        v = _i()
        call("apo_cuda_langevin_piston_integrator_get_crystal_type", ctypes.byref(v), self._h)
        return v.value

    def getNoseHooverPistonState(self) -> np.ndarray:
        """(velocity, velocity one step back, force, force one step back)"""
        a = np.zeros(4)
        call("apo_cuda_langevin_piston_integrator_get_nose_hoover_piston_state", _ptr(a), _sz(4),
             self._h)
        return a

    def setNoseHooverPistonState(self, velocity, velocity_previous, force, force_previous):
        call("apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_state", self._h,
             _d(velocity), _d(velocity_previous), _d(force), _d(force_previous))


def rigid_water_fit(xyz: np.ndarray, waters: np.ndarray) -> np.ndarray:
    """Replaces every TIP3 water (O, H1, H2 index triples) by the rigid TIP3P
    template superposed on it (mass-weighted Kabsch fit)."""
    from .systems import _water_template, M_H, M_O
    t = _water_template()
    w = np.array([M_O, M_H, M_H])
    out = np.array(xyz, np.float64, copy=True)
    P = out[waters]                                   # (n,3,3)
    com = (w[None, :, None] * P).sum(1) / w.sum()
    Q = P - com[:, None, :]
    H = np.einsum("a,ai,naj->nij", w, t, Q)           # template^T W Q
    U, _, Vt = np.linalg.svd(H)
    d = np.sign(np.linalg.det(np.einsum("nij,njk->nik", U, Vt)))
    D = np.ones((len(d), 3))
    D[:, 2] = d
    Rm = np.einsum("nij,nj,njk->nik", U, D, Vt)
    out[waters] = com[:, None, :] + np.einsum("ai,nij->naj", t, Rm)
    return out


def relax(ctx: CharmmContext, waters=None, iterations: int = 150, max_step: float = 0.03):
    """Deterministic steepest-descent relaxation on the GPU force path: every
    iteration moves the atoms along -gradient, the largest move `max_step`
    Angstrom; TIP3 waters are refitted to the rigid geometry at the end.
    Used to remove the close contacts of freshly generated synthetic systems
    before dynamics."""
    x = ctx.getCoordinates()
    for _ in range(iterations):
        ctx.calculateForces(False, False, False)
        g = ctx.getForces()
        gmax = float(np.abs(g).max())
        if not np.isfinite(gmax) or gmax == 0.0:
            break
        x = x - (max_step / gmax) * g
        ctx.setCoordinates(x)
    if waters is not None and len(waters):
        x = rigid_water_fit(x, np.asarray(waters))
        ctx.setCoordinates(x)
    return x


def water_indices(sys) -> np.ndarray:
    """(n,3) atom indices of the OT-HT-HT waters of a System."""
    t = sys.atom_type
    return np.array([[i, i + 1, i + 2] for i in range(0, len(t) - 2)
                     if t[i] == "OT" and t[i + 1] == "HT" and t[i + 2] == "HT"], np.int64).reshape(-1, 3)


class Batch(_Handle):
    """Many independent systems advanced together (apo_batch_*): one launch
    per stage of a step for all systems, one CUDA graph per list segment.
    Each system keeps its own box, cutoffs, PME grid, LJ tables, velocity
    seed and noise stream."""
    _destroy = "apo_batch_destroy"

    def __init__(self, spline_order: int = 4, tiles_per_work: int = 8, precise: bool = False):
        super().__init__()
        call("apo_batch_create", ctypes.byref(self._h), _i(spline_order), _i(tiles_per_work),
             _i(int(precise)))
        self._keep = []          # PSF/PRM handles must outlive the batch set-up
        self._n = []

    def addSystem(self, psf: "CharmmPsf", prm: "CharmmParameters", box, kappa: float,
                  cutnb: float, ctonnb: float, ctofnb: float, nfft=(-1, -1, -1),
                  seed: int = 1) -> int:
        idx = _i()
        call("apo_batch_add_system", self._h, psf.handle, prm.handle, _d(box[0]), _d(box[1]),
             _d(box[2]), _d(kappa), _d(cutnb), _d(ctonnb), _d(ctofnb), _i(nfft[0]), _i(nfft[1]),
             _i(nfft[2]), ctypes.c_ulonglong(seed), ctypes.byref(idx))
        self._keep.append((psf, prm))
        return idx.value

    def initialize(self):
        call("apo_batch_initialize", self._h)
        n = _i()
        call("apo_batch_get_num_systems", ctypes.byref(n), self._h)
        self._n = [self.numAtoms(k) for k in range(n.value)]

    def numSystems(self) -> int:
        return len(self._n)

    def numAtoms(self, system: int = -1) -> int:
        v = _sz()
        call("apo_batch_get_num_atoms", ctypes.byref(v), self._h, _i(system))
        return int(v.value)

    def setCoordinates(self, system: int, xyz):
        a = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        call("apo_batch_set_coordinates", self._h, _i(system), _ptr(a), _sz(a.size))

    def _count(self, system: int) -> int:
        return sum(self._n) if system < 0 else self._n[system]

    def getCoordinates(self, system: int) -> np.ndarray:
        """system < 0: all systems' atoms, concatenated"""
        a = np.zeros(3 * self._count(system))
        call("apo_batch_get_coordinates", _ptr(a), _sz(a.size), self._h, _i(system))
        return a.reshape(-1, 3)

    def setVelocities(self, system: int, v):
        a = np.ascontiguousarray(v, np.float64).reshape(-1)
        call("apo_batch_set_velocities", self._h, _i(system), _ptr(a), _sz(a.size))

    def getVelocities(self, system: int) -> np.ndarray:
        a = np.zeros(3 * self._count(system))
        call("apo_batch_get_velocities", _ptr(a), _sz(a.size), self._h, _i(system))
        return a.reshape(-1, 3)

    def assignVelocities(self, temperature: float):
        call("apo_batch_assign_velocities", self._h, _d(temperature))

    def setLangevin(self, dt_ps: float, friction: float, temperature: float, seed: int):
        call("apo_batch_set_langevin", self._h, _d(dt_ps), _d(friction), _d(temperature),
             ctypes.c_ulonglong(seed))

    def propagate(self, steps: int):
        call("apo_batch_propagate", self._h, _i(steps))

    def calculateForces(self, energy: bool = True, virial: bool = False):
        call("apo_batch_calculate_forces", self._h, _i(int(energy)), _i(int(virial)))

    def getForces(self, system: int) -> np.ndarray:
        a = np.zeros(3 * self._count(system))
        call("apo_batch_get_forces", _ptr(a), _sz(a.size), self._h, _i(system))
        return a.reshape(-1, 3)

    def getEnergyComponents(self, system: int) -> Dict[str, float]:
        a = np.zeros(len(ENERGY_TERMS))
        call("apo_batch_get_energy_components", _ptr(a), _sz(a.size), self._h, _i(system))
        return dict(zip(ENERGY_TERMS, a.tolist()))

    def getTemperatures(self) -> np.ndarray:
        a = np.zeros(len(self._n))
        call("apo_batch_get_temperatures", _ptr(a), _sz(a.size), self._h)
        return a

    def autotune(self, steps: int = 20, candidates=None) -> int:
        t = _i()
        if candidates:
            c = (ctypes.c_int * len(candidates))(*candidates)
            call("apo_batch_autotune", ctypes.byref(t), self._h, _i(steps), c, _i(len(candidates)))
        else:
            call("apo_batch_autotune", ctypes.byref(t), self._h, _i(steps), None, _i(0))
        return t.value

    def getStream(self) -> int:
        v = _vp()
        call("apo_batch_get_stream", ctypes.byref(v), self._h)
        return v.value or 0

    def setComponentMask(self, mask: int):
        call("apo_batch_set_component_mask", self._h, _i(mask))

    def getDirectKernel(self) -> int:
        v = _i()
        call("apo_batch_get_direct_kernel", ctypes.byref(v), self._h)
        return v.value


def batch_from_systems(systems, workdir: str, seeds=None, spline_order: int = 4,
                       tiles_per_work: int = 8, precise: bool = False) -> "Batch":
    """Writes every apocharmm_b200.systems.System as CHARMM files under
    workdir, adds it to a new Batch with its own settings, initialises the
    batch and loads the coordinates."""
    from .systems import write_charmm_files
    b = Batch(spline_order, tiles_per_work, precise)
    for k, s in enumerate(systems):
        paths = write_charmm_files(s, os.path.join(workdir, f"sys{k}"))
        st = s.settings
        b.addSystem(CharmmPsf(paths["psf"]), CharmmParameters(paths["prm"]), s.box, st["kappa"],
                    st["cutnb"], st["ctonnb"], st["ctofnb"], st["nfft"],
                    seed=(seeds[k] if seeds is not None else 1000 + k))
    b.initialize()
    b.setCoordinates(-1, np.concatenate([np.asarray(s.pos, np.float64) for s in systems]))
    return b


def relax_batch(b: "Batch", waters_per_system, iterations: int = 150, max_step: float = 0.03):
    """relax() for every system of a batch at once: steepest descent with the
    largest move per system `max_step`, then the TIP3 refit."""
    n = b.numSystems()
    off = np.concatenate([[0], np.cumsum(b._n)])
    x = b.getCoordinates(-1)
    for _ in range(iterations):
        b.calculateForces(False, False)
        g = b.getForces(-1)
        for k in range(n):
            gk = g[off[k]:off[k + 1]]
            gmax = float(np.abs(gk).max())
            if np.isfinite(gmax) and gmax > 0.0:
                x[off[k]:off[k + 1]] -= (max_step / gmax) * gk
        b.setCoordinates(-1, x)
    for k in range(n):
        w = waters_per_system[k]
        if w is not None and len(w):
            x[off[k]:off[k + 1]] = rigid_water_fit(x[off[k]:off[k + 1]], np.asarray(w))
    b.setCoordinates(-1, x)
    return [x[off[k]:off[k + 1]].copy() for k in range(n)]


class Server(_Handle):
    """Request server with continuous batching (apo_server_*): MD-segment and
    energy/force requests admitted by free HBM, advanced together 20 steps at
    a time and re-batched as they arrive and finish; every request's result
    is the same alone and among others."""
    _destroy = "apo_server_destroy"
    PENDING, DONE, FAILED = 0, 1, 2

    def __init__(self, hbm_fraction: float = 0.5, spline_order: int = 4, precise: bool = False,
                 dt_ps: float = 0.002, friction: float = 1.0, temperature: float = 300.0,
                 seed: int = 1):
        super().__init__()
        call("apo_server_create", ctypes.byref(self._h), _d(hbm_fraction), _i(spline_order),
             _i(int(precise)), _d(dt_ps), _d(friction), _d(temperature), ctypes.c_ulonglong(seed))
        self._n = {}
        self._keep = {}

    def submit(self, kind: int, psf: "CharmmPsf", prm: "CharmmParameters", box, settings,
               xyz, seed: int, steps: int = 0) -> int:
        """kind 0: MD segment of `steps` steps, 1: energies and forces.
        settings: kappa, cutnb, ctonnb, ctofnb and nfft (as System.settings)."""
        a = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        rid = _i()
        nf = settings.get("nfft", (-1, -1, -1))
        call("apo_server_submit", ctypes.byref(rid), self._h, _i(kind), psf.handle, prm.handle,
             _d(box[0]), _d(box[1]), _d(box[2]), _d(settings["kappa"]), _d(settings["cutnb"]),
             _d(settings["ctonnb"]), _d(settings["ctofnb"]), _i(nf[0]), _i(nf[1]), _i(nf[2]),
             ctypes.c_ulonglong(seed), _ptr(a), _sz(a.size), ctypes.c_longlong(steps))
        self._n[rid.value] = a.size // 3
        self._keep[rid.value] = (psf, prm)
        return rid.value

    def poll(self, rid: int) -> int:
        st = _i()
        call("apo_server_poll", ctypes.byref(st), self._h, _i(rid))
        return st.value

    def wait(self, rid: int, timeout_s: float = -1.0) -> int:
        st = _i()
        call("apo_server_wait", ctypes.byref(st), self._h, _i(rid), _d(timeout_s))
        return st.value

    def _vec(self, name: str, rid: int) -> np.ndarray:
        a = np.zeros(3 * self._n[rid])
        call(name, _ptr(a), _sz(a.size), self._h, _i(rid))
        return a.reshape(-1, 3)

    def coordinates(self, rid: int) -> np.ndarray:
        return self._vec("apo_server_get_coordinates", rid)

    def velocities(self, rid: int) -> np.ndarray:
        return self._vec("apo_server_get_velocities", rid)

    def forces(self, rid: int) -> np.ndarray:
        return self._vec("apo_server_get_forces", rid)

    def energies(self, rid: int) -> Dict[str, float]:
        a = np.zeros(len(ENERGY_TERMS))
        call("apo_server_get_energy_components", _ptr(a), _sz(a.size), self._h, _i(rid))
        return dict(zip(ENERGY_TERMS, a.tolist()))

    def latency(self, rid: int) -> float:
        v = _d()
        call("apo_server_get_latency", ctypes.byref(v), self._h, _i(rid))
        return v.value

    def release(self, rid: int):
        call("apo_server_release", self._h, _i(rid))
        self._n.pop(rid, None)
        self._keep.pop(rid, None)

    def stats(self) -> Dict[str, float]:
        a = np.zeros(8)
        call("apo_server_get_stats", _ptr(a), _sz(8), self._h)
        return dict(zip(("system_steps", "simulated_ps", "rebuilds", "segments", "max_batch",
                         "busy_s", "reform_s", "energy_evals"), a.tolist()))
