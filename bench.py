"""Benchmark: MD throughput (ns/day) of the force/step path on one B200.

Workloads (--workload; the N=1 line uses chain23k):
  chain23k  23,558-atom solvated bead chain (62.23 A box, PME 64^3 order 6,
            cutoff 12 A, force switch 10-12 A, list 14 A, Langevin 300 K,
            gamma 1/ps, dt 2 fs, SETTLE)
  water12k  12,480-atom TIP3P box (50 A, PME 48^3 order 4, cutoff 10 A,
            switch 8-10 A, list 12 A, leapfrog NVE, dt 2 fs, SETTLE)
  water1m   999,999-atom TIP3P box (215.4 A, PME 216^3 order 4, cutoff 10 A,
            switch 8-10 A, list 11.5 A, Nose-Hoover 300 K, dt 2 fs, SETTLE)
All synthetic and seeded; the generated structure is relaxed by 150
deterministic steepest-descent iterations before dynamics.  One timed
iteration is one neighbour-list segment: a list rebuild plus 20 MD steps,
replayed from a captured CUDA graph.  L2 is flushed (a 256 MB device write)
before every timed iteration, outside the timed interval.

  value  ns/day from the sum of per-iteration CUDA-event times on the
         integrator's stream, max over ranks
  e2e    ns/day through the C ABI with host buffers: every iteration uploads
         coordinates and velocities from pinned host memory, propagates the
         segment and reads coordinates and velocities back
  roofline  direct-space kernel (FP32 pipe): 65 FLOP per in-cutoff pair over
         its CUDA-event time, against the FP32 FMA peak of the GPU at the SM
         clock sampled during the timed region (SMs x 128 lanes x 2 x clock)
  cpu_baseline  the FP64 CPU oracle (all host threads) on a bounded sample

--impl reference runs the reference engine's own build (oracle/_ref, compiled
from the reference sources for sm_100a by oracle/Makefile.ref) on the same
workload through its C++ API: the same generator and relaxation algorithm on
the reference's forces, then the same integrator for the same number of
steps.  The FP64 host oracle is timed beside it as the CPU baseline.  Without
that build (or without a GPU) the arm times the FP64 host oracle alone.
With torchrun (N>1) every rank of this arm but rank 0 exits at once; the
b200 arm runs one replica of the system per rank (replicas only: the path
has no collective).  `--gpus N` with N > 1 outside torchrun starts itself
under torchrun with N ranks; inside torchrun, N must equal WORLD_SIZE.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT_PS = 0.002
SEG = 20                       # MD steps per timed iteration (list cadence)
FLOP_PER_PAIR = 65
# DRAM bytes per launch of the direct-space kernel (dram__bytes_read.sum +
# dram__bytes_write.sum) from one ncu capture of the same kernel on the same
# workload (the inputs and the fixed-point force buffer stay in L2)
NB_TRAFFIC = {
    "chain23k": (2193920, "ncu capture of this kernel on this workload "
                          "(dram__bytes_read.sum + dram__bytes_write.sum)"),
    "chain23k_npt": (2193920, "ncu capture of this kernel on the same system at constant "
                              "volume (dram__bytes_read.sum + dram__bytes_write.sum)"),
}


def ns_per_day(steps: float, seconds: float) -> float:
    return 86400.0 * steps / seconds * DT_PS * 1e-3


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                mx = max(mx, float(p[1]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if p[4 + k].lower().startswith("active"):
                    reasons.add(name)
        busy = [v for v in sm if v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(value: float, world: int, device: str = "cuda") -> float:
    """The largest of every rank's value (each rank passes its own): a
    multi-GPU time is the slowest rank's.  Every rank must call it."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank: int) -> int:
    """Velocity seed of one replica: replicas differ, runs repeat."""
    return 2024 + rank


def bench_config(spec: dict, atoms: int) -> dict:
    """The `config` of a bench line: the same keys and values in both arms."""
    return {"workload": spec["desc"], "atoms": atoms, "md_steps_per_iteration": SEG,
            "dt_fs": DT_PS * 1e3}


def fp32_peak_tflops(sm_mhz: float, n_sm: int) -> float:
    """FP32 FMA peak: every SM issues 128 FMA lanes (2 FLOP) per clock."""
    return n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12


def relaunch_under_torchrun(n: int, argv) -> int:
    """Runs this script again under torchrun with one rank per GPU."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)
    return subprocess.run(cmd).returncode


WORKLOADS = {
    "chain23k": dict(factory="config_solvated_chain", integrator="langevin", friction=1.0,
                     desc="chain23k: 23,558-atom bead chain in TIP3P, 62.23 A box, PME 64^3 "
                          "order 6, cutoff 12 / switch 10-12 / list 14, Langevin 300 K "
                          "gamma 1/ps, dt 2 fs, SETTLE"),
    # the reference's leapfrog has no constraints (src/CudaLeapFrogIntegrator.cu:43-79):
    # its arm runs this workload with the Langevin integrator at zero friction
    # the same system at constant pressure (the reference's Langevin piston)
    "chain23k_npt": dict(factory="config_solvated_chain", integrator="piston", friction=20.0,
                         desc="chain23k_npt: the chain23k system at 1 atm, cubic Langevin piston "
                              "(mass 0.02 x total mass, friction 20/ps), Nose-Hoover 300 K, "
                              "dt 2 fs, SETTLE, a new box every step"),
    "water12k": dict(factory="config_small_water", integrator="leapfrog", friction=0.0,
                     ref_integrator="langevin",
                     desc="water12k: 12,480-atom TIP3P box, 50 A, PME 48^3 order 4, cutoff 10 "
                          "/ switch 8-10 / list 12, leapfrog NVE, dt 2 fs, SETTLE"),
    "water1m": dict(factory="config_large_water", integrator="nosehoover", friction=0.0,
                    desc="water1m: 999,999-atom TIP3P box, 215.4 A, PME 216^3 order 4, cutoff "
                         "10 / switch 8-10 / list 11.5, Nose-Hoover 300 K, dt 2 fs, SETTLE"),
}
RELAX_ITERATIONS = 150
RELAX_MAX_STEP = 0.03          # Angstrom, largest move per iteration


def make_system(name: str):
    from apocharmm_b200 import systems
    return getattr(systems, WORKLOADS[name]["factory"])()


def cpu_baseline(sys_obj, target_s: float = 10.0):
    """FP64 oracle: full force evaluations + position updates on all host
    threads, as many as fit in about `target_s` seconds (at least 2)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    st = sys_obj.settings
    o = oracle.Oracle(sys_obj, st["kappa"], st["ctofnb"], st["ctonnb"], st["nfft"], st["order"])
    threads = oracle.lib().or_max_threads()
    pos = np.array(sys_obj.pos)
    vel = np.zeros_like(pos)
    inv_m = 1.0 / np.asarray(sys_obj.mass)[:, None]
    t0 = time.perf_counter()
    o.evaluate(pos=pos, nthreads=threads)  # warm-up, also sizes the sample
    evals = int(min(200, max(2, round(target_s / max(1e-3, time.perf_counter() - t0)))))
    t0 = time.perf_counter()
    for _ in range(evals):
        E, grad = o.evaluate(pos=pos, nthreads=threads)
        vel -= (DT_PS / 0.0488882129) * grad * inv_m
        pos = pos + (DT_PS / 0.0488882129) * vel
    dt = time.perf_counter() - t0
    return {"value": ns_per_day(evals, dt), "unit": "ns/day", "cores": threads, "kind": "port",
            "sample": f"{evals} FP64 force evaluations (direct, 1-4, PME, bonded) + position "
                      f"updates of the {sys_obj.n_atoms}-atom workload, {dt:.1f} s"}


def _reference_build_run(args, s, spec, work):
    """Relaxes and propagates the workload with the reference engine's own
    build; returns the harness's JSON result."""
    import numpy as np
    from apocharmm_b200.api import rigid_water_fit, water_indices
    from apocharmm_b200.systems import write_charmm_files, write_crd
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    st = s.settings
    paths = write_charmm_files(s, work)
    common = [paths["psf"], paths["prm"], paths["crd"], str(s.box[0]), str(st["kappa"]),
              str(st["cutnb"]), str(st["ctonnb"]), str(st["ctofnb"]), *map(str, st["nfft"]),
              str(st["order"])]
    relaxed = os.path.join(work, "relaxed.txt")
    subprocess.run([harness, "relax", *common, str(RELAX_ITERATIONS), str(RELAX_MAX_STEP),
                    relaxed], check=True, timeout=1800, stdout=subprocess.DEVNULL)
    s.pos = rigid_water_fit(np.loadtxt(relaxed), water_indices(s))
    write_crd(s, paths["crd"])
    r = subprocess.run([harness, "md", *common, str(args.warmup * SEG), str(args.steps * SEG),
                        "2024", str(spec["friction"]), spec.get("ref_integrator", spec["integrator"])],
                       check=True, timeout=3600, stdout=subprocess.PIPE, text=True)
    return json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])


def _gpu_visible() -> bool:
    try:
        return subprocess.run(["nvidia-smi", "-L"], stdout=subprocess.DEVNULL,
                              stderr=subprocess.DEVNULL).returncode == 0
    except OSError:
        return False


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    spec = WORKLOADS[args.workload]
    s = make_system(args.workload)
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    ref = None
    reason = None
    if not os.path.exists(harness):
        reason = "reference build (oracle/_ref) not present"
    elif not _gpu_visible():
        reason = "no GPU visible"
    else:
        ref = _reference_build_run(args, s, spec, tempfile.mkdtemp(prefix="apo_ref_"))
    cb = cpu_baseline(s)
    line = {"impl": "reference", "metric": "ns/day", "unit": "ns/day",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "data": "synthetic (seeded generator)",
            "config": bench_config(spec, s.n_atoms)}
    if ref is not None:
        line.update({
            "value": ref["ns_per_day"], "ms_per_step": 1e3 * ref["seconds"] / args.steps,
            "dtype": "f32 (forces), f64 (integration)",
            "reference_build": dict(ref, build="reference sources compiled for sm_100a "
                                               "(oracle/Makefile.ref), driven through its C++ API"),
            "note": "the reference engine is GPU-only: value is its own build on this GPU, "
                    "timed on the host between device-wide synchronisations; cpu_baseline is "
                    "the FP64 host restatement of the same force/step path"})
    else:
        line.update({"value": cb["value"], "dtype": "f64",
                     "note": f"{reason}: value is the FP64 host restatement of the reference's "
                             "force/step path"})
    line["cpu_baseline"] = cb
    line["e2e"] = {"value": line["value"], "unit": "ns/day", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}
    print(json.dumps(line), flush=True)
    return 0


def _gen_batch_system(arg):
    """Process-pool worker: one system of the many-system workload."""
    seed, n_atoms = arg
    sys.path.insert(0, ROOT)
    from apocharmm_b200.systems import batch_system
    return batch_system(seed, n_atoms)


def run_batch(args):
    """Many-system workload: seeded systems (bead chain + TIP3P, atom counts
    log-uniform in 3,000-30,000, boxes at 0.997 g/cm^3, PME spacing <= 1 A,
    order 4, cutoff 10 A, Langevin 300 K, dt 2 fs, SETTLE) advanced together
    by the batch engine, against the same systems stepped one at a time in
    the plain form on the same GPU.  Both are timed with CUDA events over
    list-update segments; aggregate ns/day = simulated time of all systems
    per wall day."""
    import multiprocessing as mp

    import numpy as np
    rank, world, local = dist_env()
    t_start = time.perf_counter()

    def log(msg):
        print(f"[batch {time.perf_counter() - t_start:7.1f} s] {msg}", file=sys.stderr, flush=True)

    from apocharmm_b200.systems import batch_sizes
    sizes = batch_sizes(args.systems)
    with mp.get_context("spawn").Pool(min(len(sizes), os.cpu_count() or 1)) as pool:
        systems = pool.map(_gen_batch_system, [(1000 + k, n) for k, n in enumerate(sizes)],
                           chunksize=1)
    t_gen = time.perf_counter() - t_start
    log(f"generated {len(systems)} systems, {sum(s.n_atoms for s in systems)} atoms")
    import torch
    torch.cuda.set_device(local)
    from apocharmm_b200 import api
    work = tempfile.mkdtemp(prefix="apo_batch_")
    seeds = [5000 + k for k in range(len(systems))]
    b = api.batch_from_systems(systems, work, seeds=seeds, tiles_per_work=8,
                               precise=args.precise)
    log("batch initialised")
    waters = [api.water_indices(s) for s in systems]
    n_sys_all = len(systems)
    xs = api.relax_batch(b, waters, iterations=RELAX_ITERATIONS, max_step=RELAX_MAX_STEP)
    log("relaxed")
    # force error against FP64 on a sample of systems at the relaxed
    # coordinates; the one-by-one engine is checked at the same coordinates
    sample = sorted({0, n_sys_all // 3, 2 * n_sys_all // 3, n_sys_all - 1})
    b.calculateForces(False, False)
    errs, one_errs, grads = [], [], {}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        for k in sample:
            s = systems[k]
            st = s.settings
            Eo, Go = oracle.Oracle(s, st["kappa"], st["ctofnb"], st["ctonnb"], st["nfft"],
                                   st["order"]).evaluate(pos=xs[k])
            F = b.getForces(k)
            errs.append(float(np.sqrt(((F - Go) ** 2).sum() / (Go ** 2).sum())))
            grads[k] = Go
        log("force errors done")
    b.assignVelocities(300.0)
    b.setLangevin(DT_PS, 1.0, 300.0, 777)
    tpw = b.autotune(SEG, [4, 8, 16, 32])
    form = b.getDirectKernel()
    log(f"autotuned: {tpw} tiles per work item, kernel form {form}")
    stream = torch.cuda.ExternalStream(b.getStream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        b.propagate(SEG)
    torch.cuda.synchronize()
    seg_ms = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.propagate(SEG)
            e1.record(stream)
            e1.synchronize()
            seg_ms.append(e0.elapsed_time(e1))
    n_sys = len(systems)
    value = ns_per_day(args.steps * SEG * n_sys, sum(seg_ms) * 1e-3)
    log(f"timed: {sum(seg_ms) / args.steps:.2f} ms per segment, {value:.1f} ns/day")
    # end to end through the C ABI: all coordinates and velocities up and down per segment
    ntot = sum(s.n_atoms for s in systems)
    hx = torch.empty((ntot, 3), dtype=torch.float64, pin_memory=True)
    hv = torch.empty((ntot, 3), dtype=torch.float64, pin_memory=True)
    hx.numpy()[:] = b.getCoordinates(-1)
    hv.numpy()[:] = b.getVelocities(-1)
    iters = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(iters):
        api.call("apo_batch_set_coordinates", b.handle, api._i(-1), api._vp(hx.data_ptr()),
                 api._sz(3 * ntot))
        api.call("apo_batch_set_velocities", b.handle, api._i(-1), api._vp(hv.data_ptr()),
                 api._sz(3 * ntot))
        b.propagate(SEG)
        api.call("apo_batch_get_coordinates", api._vp(hx.data_ptr()), api._sz(3 * ntot), b.handle,
                 api._i(-1))
        api.call("apo_batch_get_velocities", api._vp(hv.data_ptr()), api._sz(3 * ntot), b.handle,
                 api._i(-1))
    e2e_s = time.perf_counter() - t0
    log("end to end done")
    # the same systems one at a time in the plain (single-system) engine,
    # from the files and relaxed coordinates the batch used
    one_ms = 0.0
    for k, s in enumerate(systems if args.one_steps > 0 else []):
        st = s.settings
        d = os.path.join(work, f"sys{k}")
        psf = api.CharmmPsf(os.path.join(d, f"{s.name}.psf"))
        prm = api.CharmmParameters(os.path.join(d, f"{s.name}.prm"))
        fm = api.ForceManager(psf, prm)
        fm.setBoxDimensions(s.box)
        fm.setKappa(st["kappa"])
        fm.setCutoff(st["cutnb"])
        fm.setCtonnb(st["ctonnb"])
        fm.setCtofnb(st["ctofnb"])
        fm.setFFTGrid(*st["nfft"])
        fm.setPmeSplineOrder(st["order"])
        fm.setPrecisionMode(args.precise)
        ctx = api.CharmmContext(fm)
        ctx.setCoordinates(xs[k])
        ctx.setRandomSeedForVelocities(seeds[k])
        ctx.assignVelocitiesAtTemperature(300.0)
        if k in grads:
            ctx.calculateForces(False, False, False)
            F = ctx.getForces()
            Go = grads[k]
            one_errs.append(float(np.sqrt(((F - Go) ** 2).sum() / (Go ** 2).sum())))
        integ = api.CudaLangevinThermostatIntegrator(DT_PS)
        integ.setThermostatFriction(1.0)
        integ.setReferenceTemperature(300.0)
        integ.setThermostatRngSeed(777)
        integ.setCharmmContext(ctx)
        integ.propagate(SEG)                       # capture + first replay
        st1 = torch.cuda.ExternalStream(ctx.getStream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st1)
        for _ in range(args.one_steps):
            integ.propagate(SEG)
        e1.record(st1)
        e1.synchronize()
        one_ms += e0.elapsed_time(e1)
        del integ, ctx, fm, prm, psf
        if k % 32 == 31:
            log(f"one by one: {k + 1} systems")
    one_value = ns_per_day(args.one_steps * SEG * n_sys, one_ms * 1e-3) if one_ms > 0 else None
    line = {
        "metric": "aggregate ns/day (many independent systems)", "value": value,
        "unit": "ns/day", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sum(seg_ms) / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (forces), f64 (integration)",
        "data": "synthetic (seeded generator)",
        "config": {"workload": f"batch{n_sys}: {n_sys} systems, bead chain (~10 %) in TIP3P, "
                               "atoms log-uniform 3,000-30,000, 0.997 g/cm^3, PME spacing "
                               "<= 1 A, order 4, cutoff 10 / switch 8-10 / list 12, Langevin "
                               "300 K gamma 1/ps, dt 2 fs, SETTLE",
                   "systems": n_sys, "atoms": ntot, "md_steps_per_iteration": SEG,
                   "form": "precision" if args.precise else "plain",
                   "tiles_per_work_autotuned": tpw,
                   "direct_kernel_autotuned": ["tile batches", "grouped queues"][form],
                   "l2": "flushed (256 MB device write) before every timed iteration"},
        "one_by_one": {"value": one_value, "unit": "ns/day",
                       "note": f"the same systems, one single-system context at a time, "
                               f"{args.one_steps} timed segments each after one warm-up segment",
                       "force_rel_rms_vs_fp64": one_errs},
        "batched_over_one_by_one": value / one_value if one_value else None,
        "force_rel_rms_vs_fp64": errs, "force_error_sample_systems": sample,
        "e2e": {"value": ns_per_day(iters * SEG * n_sys, e2e_s), "unit": "ns/day",
                "h2d_bytes_per_step": 2 * 3 * ntot * 8 / SEG,
                "d2h_bytes_per_step": 2 * 3 * ntot * 8 / SEG},
        "clocks": clocks.summary(), "generation_s": t_gen,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """Serving workload: a seeded Poisson request stream (mean 50 requests/s),
    70 % MD segments (U[100, 5000] steps) and 30 % single energy/force
    evaluations, each on its own system (bead chain + TIP3P, atoms
    log-uniform in 2,000-100,000, 0.997 g/cm^3, PME spacing <= 1 A, order 4,
    cutoff 10 A), Langevin 300 K, dt 2 fs.  Requests are submitted to the
    server at their arrival times; latency is arrival -> result.  Aggregate
    ns/day = simulated time of all MD requests over the wall time from the
    first arrival to the last result."""
    import multiprocessing as mp

    import numpy as np
    rank, world, local = dist_env()
    t_start = time.perf_counter()

    def log(msg):
        print(f"[serve {time.perf_counter() - t_start:7.1f} s] {msg}", file=sys.stderr, flush=True)

    rng = np.random.default_rng(4242)
    nreq = args.requests
    sizes = [int(v) for v in np.exp(rng.uniform(np.log(2000), np.log(100000), nreq))]
    kinds = (rng.uniform(size=nreq) >= 0.7).astype(int)          # 1 = energy/force
    steps = rng.integers(100, 5001, nreq)
    arrivals = np.cumsum(rng.exponential(1.0 / 50.0, nreq))
    with mp.get_context("spawn").Pool(min(nreq, os.cpu_count() or 1)) as pool:
        systems = pool.map(_gen_batch_system, [(2000 + k, n) for k, n in enumerate(sizes)],
                           chunksize=1)
    log(f"generated {nreq} systems, {sum(s.n_atoms for s in systems)} atoms")
    import torch
    torch.cuda.set_device(local)
    from apocharmm_b200 import api
    from apocharmm_b200.systems import write_charmm_files
    work = tempfile.mkdtemp(prefix="apo_serve_")
    b = api.batch_from_systems(systems, os.path.join(work, "relax"))
    xs = api.relax_batch(b, [api.water_indices(s) for s in systems],
                         iterations=RELAX_ITERATIONS, max_step=RELAX_MAX_STEP)
    b.close()
    del b
    handles = []
    for k, s in enumerate(systems):
        p = write_charmm_files(s, os.path.join(work, f"r{k}"))
        handles.append((api.CharmmPsf(p["psf"]), api.CharmmParameters(p["prm"])))
    log("relaxed, files written")
    srv = api.Server(hbm_fraction=0.8, spline_order=4, precise=args.precise, dt_ps=DT_PS,
                     friction=1.0, temperature=300.0, seed=31)
    ids = []
    t0 = time.perf_counter()
    with ClockSampler(local) as clocks:
        for k in range(nreq):
            delay = arrivals[k] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            s = systems[k]
            ids.append(srv.submit(int(kinds[k]), handles[k][0], handles[k][1], s.box, s.settings,
                                  xs[k], 7000 + k, int(steps[k])))
        for rid in ids:
            if srv.wait(rid, 3600.0) != api.Server.DONE:
                raise RuntimeError(f"request {rid} failed")
    wall = time.perf_counter() - t0
    lat = np.array([srv.latency(r) for r in ids])
    md = kinds == 0
    st = srv.stats()
    sim_ns = float(sum(int(steps[k]) for k in range(nreq) if md[k])) * DT_PS * 1e-3
    value = sim_ns / (wall / 86400.0)
    log(f"served: wall {wall:.1f} s, p50 {np.percentile(lat, 50):.3f} s, "
        f"p99 {np.percentile(lat, 99):.3f} s")
    # force error against FP64 for the smallest energy/force requests
    errs = []
    same = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        ek = sorted([k for k in range(nreq) if not md[k]], key=lambda k: sizes[k])[:2]
        for k in ek:
            s = systems[k]
            stt = s.settings
            Eo, Go = oracle.Oracle(s, stt["kappa"], stt["ctofnb"], stt["ctonnb"], stt["nfft"],
                                   stt["order"]).evaluate(pos=xs[k])
            F = srv.forces(ids[k])
            errs.append(float(np.sqrt(((F - Go) ** 2).sum() / (Go ** 2).sum())))
        # the smallest MD request again, alone on a fresh server
        k = min([k for k in range(nreq) if md[k]], key=lambda k: sizes[k])
        alone = api.Server(hbm_fraction=0.8, spline_order=4, precise=args.precise, dt_ps=DT_PS,
                           friction=1.0, temperature=300.0, seed=31)
        s = systems[k]
        rid = alone.submit(0, handles[k][0], handles[k][1], s.box, s.settings, xs[k], 7000 + k,
                           int(steps[k]))
        alone.wait(rid, 3600.0)
        same = bool(np.array_equal(alone.coordinates(rid), srv.coordinates(ids[k])))
        alone.close()
    line = {
        "metric": "serving: aggregate ns/day with p50/p99 latency", "value": value,
        "unit": "ns/day", "n_gpus": 1, "steps": nreq, "warmup": 0,
        "ms_per_step": 1e3 * wall / max(1, nreq), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (forces), f64 (integration)",
        "data": "synthetic (seeded generator and request stream)",
        "config": {"workload": f"serve{nreq}: Poisson 50 req/s, 70 % MD U[100, 5000] steps, 30 % "
                               "energy/force, atoms log-uniform 2,000-100,000, bead chain in "
                               "TIP3P, PME spacing <= 1 A, order 4, cutoff 10 A, Langevin 300 K, "
                               "dt 2 fs", "requests": nreq, "md_requests": int(md.sum()),
                   "atoms": int(sum(sizes)), "hbm_fraction": 0.8},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "p50_md": float(np.percentile(lat[md], 50)) if md.any() else None,
                      "p50_energy": float(np.percentile(lat[~md], 50)) if (~md).any() else None},
        "wall_s": wall, "server": st, "force_rel_rms_vs_fp64": errs,
        "smallest_md_request_same_alone": same, "clocks": clocks.summary(),
    }
    srv.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def make_integrator(api, spec, rank):
    kind = spec["integrator"]
    if kind == "langevin":
        integ = api.CudaLangevinThermostatIntegrator(DT_PS)
        integ.setThermostatFriction(spec["friction"])
        integ.setReferenceTemperature(300.0)
        integ.setThermostatRngSeed(777 + rank)
    elif kind == "leapfrog":
        integ = api.CudaLeapFrogIntegrator(DT_PS)
    elif kind == "piston":
        integ = api.CudaLangevinPistonIntegrator(DT_PS)
        integ.setCrystalType(integ.CUBIC)
        integ.setReferenceTemperature(300.0)
        integ.setLangevinPistonFriction(spec["friction"])
        integ.setLangevinPistonFrictionSeed(777 + rank)
    else:
        integ = api.CudaNoseHooverIntegrator(DT_PS)
        integ.setReferenceTemperature(300.0)
    return integ


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100, help="timed iterations (20 MD steps each)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="chain23k",
                    choices=sorted(WORKLOADS) + ["batch", "serve"])
    ap.add_argument("--requests", type=int, default=40, help="serve workload: requests")
    ap.add_argument("--systems", type=int, default=256, help="batch workload: number of systems")
    ap.add_argument("--one-steps", type=int, default=2,
                    help="batch workload: timed segments per system in the one-by-one baseline "
                         "(0: skip the baseline)")
    ap.add_argument("--precise", action="store_true", help="precision form")
    ap.add_argument("--pme-tensor-copies", type=int, default=1, choices=[0, 1],
                    help="z-pencil slabs by tiled tensor copies (1) or plain loads (0)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--tiles-per-work", type=int, default=8,
                    help="j-tiles per direct-space work item")
    ap.add_argument("--items-per-warp", type=int, default=None,
                    help="direct-space work items per warp before it retires (0: persistent "
                         "grid; default: the library's)")
    ap.add_argument("--direct-kernel", type=int, default=0, choices=[0, 1, 2],
                    help="direct-space kernel form: 0 tile batches, 1 grouped queues, 2 octet lists")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if "WORLD_SIZE" in os.environ:
        if int(os.environ["WORLD_SIZE"]) != args.gpus:
            print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={os.environ['WORLD_SIZE']}",
                  file=sys.stderr)
            return 2
    elif args.gpus > 1:
        return relaunch_under_torchrun(args.gpus, sys.argv[1:])
    if args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no "
                              "serving layer"}))
            return 0
        return run_serve(args)
    if args.workload == "batch":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no "
                              "many-system engine; the one-by-one baseline is in the b200 line"}))
            return 0
        return run_batch(args)
    if args.impl == "reference":
        return run_reference_arm(args)

    import numpy as np
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)

    from apocharmm_b200 import api
    spec = WORKLOADS[args.workload]
    s = make_system(args.workload)
    work = tempfile.mkdtemp(prefix=f"apo_bench_{rank}_")
    psf, prm, fm, ctx = api.system_context(s, work, precise=args.precise,
                                           tiles_per_work=args.tiles_per_work,
                                           items_per_warp=args.items_per_warp)
    fm.setDirectKernel(args.direct_kernel)
    fm.setPmeTensorCopies(bool(args.pme_tensor_copies))
    # remove the close contacts of the generated structure (deterministic)
    s.pos = api.relax(ctx, api.water_indices(s), iterations=RELAX_ITERATIONS,
                      max_step=RELAX_MAX_STEP)
    ctx.setRandomSeedForVelocities(replica_seed(rank))
    ctx.assignVelocitiesAtTemperature(300.0)

    # force error of this configuration against the FP64 oracle (rank 0)
    force_err = None
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        ctx.calculateForces(False, True, False)
        F = ctx.getForces()
        st = s.settings
        Eo, Go = oracle.Oracle(s, st["kappa"], st["ctofnb"], st["ctonnb"], st["nfft"],
                               st["order"]).evaluate()
        force_err = float(np.sqrt(((F - Go) ** 2).sum() / (Go ** 2).sum()))

    n_pairs_cut = _count_pairs(ctx, s.settings["ctofnb"])

    ctx.resetNeighborList()
    api.call("apo_charmm_context_set_kernel_timing", ctx.handle, api._i(1))
    integ = make_integrator(api, spec, rank)
    integ.setCharmmContext(ctx)

    stream = torch.cuda.ExternalStream(ctx.getStream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        integ.propagate(SEG)

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    seg_ms, nb_ms, nb_launch = [], 0.0, 0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            integ.propagate(SEG)
            e1.record(stream)
            e1.synchronize()
            seg_ms.append(e0.elapsed_time(e1))
            t = api.ctypes.c_double()
            n = api.ctypes.c_int()
            api.call("apo_charmm_context_get_kernel_time", api.ctypes.byref(t), api.ctypes.byref(n),
                     ctx.handle)
            nb_ms += t.value
            nb_launch += n.value
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(seg_ms), world)
    if world > 1:
        torch.distributed.barrier()
    md_steps = args.steps * SEG
    value = ns_per_day(md_steps * world, total_ms * 1e-3)
    n_pairs_end = _count_pairs(ctx, s.settings["ctofnb"])
    lc = [api.ctypes.c_int() for _ in range(3)]
    api.call("apo_charmm_context_get_list_counts", *[api.ctypes.byref(v) for v in lc], ctx.handle)
    list_counts = {"slots": lc[0].value, "tiles": lc[1].value, "work_items": lc[2].value}

    # end-to-end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        n = s.n_atoms
        hx = torch.empty(3 * n, dtype=torch.float64, pin_memory=True)
        hv = torch.empty(3 * n, dtype=torch.float64, pin_memory=True)
        hx.numpy()[:] = ctx.getCoordinates().reshape(-1)
        hv.numpy()[:] = ctx.getVelocities().reshape(-1)
        lib = api.lib()
        iters = max(3, args.steps // 2)
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        for _ in range(iters):
            api.call("apo_charmm_context_set_coordinates_xyz", ctx.handle,
                     api._vp(hx.data_ptr()), api._sz(3 * n))
            api.call("apo_charmm_context_set_velocities", ctx.handle,
                     api._vp(hv.data_ptr()), api._sz(3 * n))
            integ.propagate(SEG)
            api.call("apo_charmm_context_get_coordinates", api._vp(hx.data_ptr()), api._sz(3 * n),
                     ctx.handle)
            api.call("apo_charmm_context_get_velocities", api._vp(hv.data_ptr()), api._sz(3 * n),
                     ctx.handle)
        el = max_over_ranks(time.perf_counter() - t0, world)
        e2e = {"value": ns_per_day(iters * SEG * world, el), "unit": "ns/day",
               "h2d_bytes_per_step": 2 * 3 * n * 8 / SEG, "d2h_bytes_per_step": 2 * 3 * n * 8 / SEG,
               "note": "per 20-step segment: coordinates+velocities up (pinned), propagate, "
                       "coordinates+velocities down; bytes given per MD step"}

    if rank == 0:
        clk = clocks.summary()
        n_sm = torch.cuda.get_device_properties(local).multi_processor_count
        peak = fp32_peak_tflops(clk["sm_mhz"] or 1965.0, n_sm)
        avg_nb_s = (nb_ms / max(1, nb_launch)) * 1e-3
        pairs_avg = 0.5 * (n_pairs_cut + n_pairs_end)
        achieved = pairs_avg * FLOP_PER_PAIR / avg_nb_s / 1e12 if avg_nb_s > 0 else None
        cb = None
        if not args.no_cpu_baseline:
            cb = cpu_baseline(s)
        kps = integ.getKernelsPerStep()
        if spec["integrator"] == "piston":  # the sorted coordinates refreshed every step
            launches = args.steps * (12 + SEG * (8 + kps))
        else:
            launches = args.steps * (12 + SEG * (7 + kps))
        line = {
            "metric": "ns/day", "value": value, "unit": "ns/day", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (forces), f64 (integration)", "data": "synthetic (seeded generator)",
            "config": bench_config(spec, s.n_atoms),
            "engine": {"form": "precision" if args.precise else "plain",
                       "direct_kernel": ["tile batches", "grouped queues", "octet lists"][args.direct_kernel],
                       "tiles_per_work": args.tiles_per_work,
                       "items_per_warp": args.items_per_warp,
                       "pme_tensor_copies": fm.getPmeTensorCopies()},
            "l2": "flushed (256 MB device write) before every timed iteration, outside the "
                  "timed interval",
            "parallelism": f"replicas x{world}",
            "md_steps_timed": md_steps,
            "neighbor_list": list_counts,
            "force_rel_rms_vs_fp64": force_err,
            "roofline": {"kernel": "direct-space tile kernel", "bound": "fp32",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": NB_TRAFFIC.get(args.workload, (None, None))[0],
                         "traffic_source": NB_TRAFFIC.get(args.workload, (None, None))[1],
                         "work": f"{FLOP_PER_PAIR} FLOP x {pairs_avg:.0f} in-cutoff pairs per launch",
                         "launch_ms": avg_nb_s * 1e3, "launches_timed": nb_launch,
                         "peak_source": f"{n_sm} SMs x 128 FP32 lanes x 2 FLOP x the median SM "
                                        f"clock sampled in the timed region ({clk['sm_mhz']} MHz)"},
            "clocks": clk,
            "e2e": e2e,
            "gpu_launches": launches,
            "cpu_baseline": cb,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def _count_pairs(ctx, radius: float) -> int:
    from apocharmm_b200 import api
    n = api._sz()
    api.call("apo_charmm_context_get_neighbor_pairs", None, api._sz(0), api.ctypes.byref(n),
             api._d(radius), ctx.handle)
    return int(n.value)


if __name__ == "__main__":
    sys.exit(main())
