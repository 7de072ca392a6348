#!/usr/bin/env python
"""Benchmark of the KS-Hamiltonian hot path on B200.

Workload (one "step"): H|psi> on the 64-atom diamond supercell -- cubic
a = 20.52 bohr, 64^3 grid, 128 orbitals, 256 Gaussian KB projectors -- in mixed
precision (complex64 FFT/pointwise, FP64 projection accumulators).  Reported
beside it: the same apply in FP64, ETRS steps/s on the same system, and the
error of the mixed result against the FP64 path and the CPU FP64 oracle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun: every rank applies H to its own 128 orbitals (the
path is independent per orbital, no data-path collective: weak scaling).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "inq-wannier-fork_b200"))

import numpy as np  # noqa: E402

METRIC = "orbital H-applies/s"
UNIT = "orbital-applies/s"
WORKLOAD = ("64-atom diamond supercell: cubic a=20.52 bohr, 64^3 grid, 128 orbitals, 256 Gaussian KB "
            "projectors (s+p, radius 3 bohr), Gamma point; one step = one H|psi> on all 128 orbitals")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--orbitals", type=int, default=128)
    ap.add_argument("--etrs-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bounded CPU-baseline sample length")
    ap.add_argument("--no-cells", dest="cells", action="store_false", help="skip the 16-cell batch measurement")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false", help="skip the adjoint measurement")
    ap.add_argument("--no-cfg4", dest="cfg4", action="store_false",
                    help="skip the large-cell (144^3, 480 orbitals) section")
    return ap.parse_args()


# ------------------------------------------------------------------ distributed plumbing
def dist_setup(ngpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_pg(world, local):
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180), device_id=torch.device("cuda", local))
    return dist if world > 1 else None


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, x: float) -> float:
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # the timed region starts only once the sampler is producing lines
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        busy = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ inputs
def build_inputs(M, seed=0):
    from pinq_b200 import systems

    lattice = systems.cubic(20.52)
    nr = (64, 64, 64)
    pos = systems.diamond_positions(10.26, 2)
    V = systems.gaussian_potential(lattice, nr, pos)
    psi = systems.random_orbitals(lattice, nr, M, 25.0, seed)
    return lattice, nr, pos, V, psi


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), float(d.get("bf16_tflops", 1590.0)), "measured"
    return 6650.0, 1590.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of each kernel from the committed ncu summaries:
    lines 'traffic <kernel> <bytes_per_launch>' in profiles/*.txt."""
    out = {}
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return out
    for f in sorted(os.listdir(pdir)):
        if not f.endswith(".txt"):
            continue
        for line in open(os.path.join(pdir, f)):
            parts = line.split()
            if len(parts) == 3 and parts[0] == "traffic":
                try:
                    out[parts[1]] = float(parts[2])
                except ValueError:
                    pass
    return out


# ------------------------------------------------------------------ CPU baseline (oracle)
def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), recorded beside CPU timings."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def cpu_baseline(lattice, nr, pos, V, seconds, steps=None, warmup=0):
    """The oracle's FP64 H|psi> (C++, OpenMP over orbitals, all host threads) on a
    bounded sample of the same workload: as many orbitals as threads."""
    import oracle

    oracle.build()
    threads = oracle.num_threads()
    from pinq_b200 import systems

    Ms = max(1, min(128, threads))
    psi = systems.random_orbitals(lattice, nr, Ms, 25.0, 7)
    o = oracle.System(lattice, nr)
    o.set_potential(V)
    o.set_projectors(o.build_gaussian_kb(pos))
    for _ in range(warmup):
        o.apply_h(psi)
    times = []
    t_end = time.perf_counter() + seconds
    n = 0
    while True:
        t0 = time.perf_counter()
        o.apply_h(psi)
        times.append(time.perf_counter() - t0)
        n += 1
        if (steps is not None and n >= steps) or (steps is None and time.perf_counter() > t_end):
            break
    total = sum(times)
    # the median apply (every apply after the warm-ups is a repetition of the same work)
    return {"value": Ms / statistics.median(times), "unit": UNIT, "cores": threads, "cpu_model": cpu_model(),
            "kind": "port",
            "sample": f"oracle FP64 H|psi> on {Ms} of the 128 orbitals of the same 64^3 / 64-atom system, "
                      f"median of {n} applies after {warmup} warm-ups ({total:.1f} s)"}, times


def _timed_ms(fn, K, W):
    import torch

    for _ in range(W):
        fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(K):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e)


def bench_cells(args, local):
    """cfg3: 16 uneven cells (grids 24..48^3, 8..64 orbitals, 2..16 atoms), mixed
    precision; one CUDA graph (one branch per cell) and one persistent launch over a
    device work queue, against cell-by-cell launches."""
    import torch

    import pinq_b200 as pb
    from pinq_b200 import systems

    hams, xs, ys = [], [], []
    for c in systems.cfg3_cells(seed=0):
        h = pb.KSHamiltonian(c["lattice"], c["nr"], "mixed", device=local)
        h.set_scalar_potential(systems.gaussian_potential(c["lattice"], c["nr"], c["positions"]))
        h.set_gaussian_projectors(c["positions"])
        h.reserve(c["M"])
        x = torch.as_tensor(systems.random_orbitals(c["lattice"], c["nr"], c["M"], 25.0, c["seed"])).to(
            "cuda", torch.complex64)
        hams.append(h)
        xs.append(x)
        ys.append(torch.empty_like(x))
    batch = pb.CellBatch(hams, mode="graph")
    K = max(20, args.steps // 4)
    ms_graph = _timed_ms(lambda: batch.apply(xs, ys), K, 3)
    # the persistent form: one kernel over (cell, pass, tiles) work items from a device queue
    pbatch = pb.CellBatch(hams, mode="persistent")
    ms_pers = _timed_ms(lambda: pbatch.apply(xs, ys), K, 3)
    pbatch.status()
    pinfo = pbatch.info()
    pbatch.close()

    def seq():
        for h, x, y in zip(hams, xs, ys):
            h.apply(x, y)

    ms_seq = _timed_ms(seq, K, 3)
    # every cell's launch schedule picked by the autotuner, then the faster launch form
    t0 = time.perf_counter()
    scheds = batch.autotune([x.shape[1] for x in xs])
    batch.set_mode("auto")
    form, form_ms = batch.autotune_form(xs, ys)
    tune_s = time.perf_counter() - t0
    ms_tuned = _timed_ms(lambda: batch.apply(xs, ys), K, 3)
    batch.status()
    norb = sum(x.shape[1] for x in xs)
    return {"ncells": len(hams), "grids": [h.nr[0] for h in hams], "orbitals": norb, "steps": K,
            "graph_orbital_applies_per_s": norb * K / (ms_graph * 1e-3),
            "persistent_orbital_applies_per_s": norb * K / (ms_pers * 1e-3),
            "persistent_work_items": pinfo["items"], "persistent_ctas": pinfo["ctas"],
            "sequential_orbital_applies_per_s": norb * K / (ms_seq * 1e-3),
            "graph_speedup": ms_seq / ms_graph,
            "autotuned_form": form, "autotuned_form_ms": form_ms,
            "autotuned_orbital_applies_per_s": norb * K / (ms_tuned * 1e-3),
            "autotune_speedup_over_default_graph": ms_graph / ms_tuned, "autotune_s": tune_s,
            "schedules": [list(sc) for sc in scheds], "precision": "mixed"}


def bench_adjoint(args, local):
    """cfg2: ETRS forward (200 steps, dt 0.05, 16 orbitals on the 32^3 / 8-atom cell,
    checkpoints every 20) and its adjoint, FP64 and mixed; wall times of the
    device-synchronised calls."""
    import torch

    import pinq_b200 as pb
    from pinq_b200 import systems
    from pinq_b200.adjoint import DipolePropagation

    cfg = systems.config("cfg2")
    out = {"config": "cfg2: a=10.26, 32^3, 8 atoms, 16 orbitals, dt=0.05, 200 steps, checkpoint every 20, "
                     "Fourier sphere mask on", "steps": cfg["steps"],
           "ratio": "(forward keeping what the backward needs + backward, better of 2) / plain forward (best of 3)",
           "timing": "wall clock around device-synchronised calls"}
    for precision in ("fp64", "mixed"):
        h = pb.KSHamiltonian(cfg["lattice"], cfg["nr"], precision, device=local)
        h.set_scalar_potential(cfg["V"])
        h.set_gaussian_projectors(cfg["positions"])
        h.set_fourier_sphere_mask(True)
        dt = torch.complex128 if precision == "fp64" else torch.complex64
        psi0 = torch.as_tensor(cfg["psi"]).to("cuda", dt)
        res = {}
        # one plain-forward baseline per precision, the best of three runs, shared by
        # both modes (the plain forward is the same ETRS run in either mode)
        base = DipolePropagation(h, psi0, cfg["occ"], cfg["dt"], cfg["checkpoint_every"], store_powers=False)
        base.forward(cfg["amplitudes"], keep=False)
        t_plain = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            base.forward(cfg["amplitudes"], keep=False)
            torch.cuda.synchronize()
            t_plain.append(time.perf_counter() - t0)
        del base
        t_fwd = min(t_plain)
        for mode, store in (("checkpointed", False), ("stored_powers", True)):
            prop = DipolePropagation(h, psi0, cfg["occ"], cfg["dt"], cfg["checkpoint_every"], store_powers=store)
            prop.forward(cfg["amplitudes"], keep=True)  # warm-up
            prop.backward()
            best = None
            for _ in range(2):  # the better of two (forward keeping + backward) runs
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                d = prop.forward(cfg["amplitudes"], keep=True)
                torch.cuda.synchronize()
                t2 = time.perf_counter()
                gA, gV = prop.backward()
                torch.cuda.synchronize()
                t3 = time.perf_counter()
                if best is None or t3 - t1 < best[2] - best[0]:
                    best = (t1, t2, t3)
            t1, t2, t3 = best
            res[mode] = {"forward_s": t_fwd, "forward_keep_s": t2 - t1, "backward_s": t3 - t2,
                         "total_over_forward": (t3 - t1) / t_fwd, "dipole": d,
                         "grad_amplitudes_norm": float(gA.norm()), "grad_V_norm": float(gV.norm()),
                         "_gA": gA.cpu().numpy(), "_gV": gV.cpu().numpy()}
            del prop
        out[precision] = {"forward_steps_per_s": cfg["steps"] / res["checkpointed"]["forward_s"], "modes": res}
    out["mixed_vs_fp64"] = {}
    for mode in ("checkpointed", "stored_powers"):
        g64, g32 = out["fp64"]["modes"][mode], out["mixed"]["modes"][mode]
        out["mixed_vs_fp64"][mode] = {
            "dipole_rel": abs(g32["dipole"] - g64["dipole"]) / max(1e-300, abs(g64["dipole"])),
            "grad_amplitudes_rel": float(np.linalg.norm(g32["_gA"] - g64["_gA"]) / np.linalg.norm(g64["_gA"])),
            "grad_V_rel": float(np.linalg.norm(g32["_gV"] - g64["_gV"]) / np.linalg.norm(g64["_gV"]))}
    for p in ("fp64", "mixed"):
        for mode in ("checkpointed", "stored_powers"):
            del out[p]["modes"][mode]["_gA"], out[p]["modes"][mode]["_gV"]
    return out


def bench_cfg4(args, local):
    """Large cell: cubic a=30, 144^3, 240 atoms on a jittered shell (radius 6.7), 960
    projectors, 480 orbitals (11.5 GB in complex64, 23 GB in complex128), inputs made on
    the device (plane waves within ecut 30 Ha, the library's inverse FFT and
    orthonormalisation).  H|psi> and ETRS steps/s in both precisions, the LDA SCF ETRS
    step and the TD-MLWF step in mixed precision, device memory, the mixed-vs-FP64
    error of H|psi> on the same (complex64) input orbitals, and the adjoint gradient
    (50 steps, checkpoints every 10) of 16 of the orbitals in both precisions."""
    import torch

    import pinq_b200 as pb
    from pinq_b200 import systems
    from pinq_b200.adjoint import DipolePropagation

    lattice = systems.cubic(30.0)
    nr = (144, 144, 144)
    pos = systems.shell_positions(240, 6.7, 0.05, (15.0, 15.0, 15.0), seed=0)
    V = systems.gaussian_potential_device(lattice, nr, pos, device=f"cuda:{local}")
    vion_d = torch.as_tensor(V, dtype=torch.float64, device=f"cuda:{local}").contiguous()
    M = 480
    out = {"config": "cfg4: cubic a=30, 144^3, 240 atoms on a jittered shell r=6.7 (Fibonacci sphere), "
                     "960 projectors, ecut 30 Ha, 480 orbitals", "timing": "CUDA events; SCF ETRS and TD-MLWF: "
                     "wall clock around synchronised calls"}
    x_err = None  # the first 32 orbitals of the FP64 block, rounded to complex64: the common input
    y_err = {}
    for precision in ("fp64", "mixed"):
        torch.cuda.empty_cache()
        torch.cuda.reset_peak_memory_stats()
        h = pb.KSHamiltonian(lattice, nr, precision, device=local)
        h.set_scalar_potential(V)
        kb = h.set_gaussian_projectors(pos, 3.0, 1.0, 1.5, -0.7)
        x = systems.random_orbitals_device(h, M, 30.0, seed=3)
        if x_err is None:
            x_err = x[:, :32].to(torch.complex64).cpu()
        xe = x_err.to(device=x.device, dtype=x.dtype)
        y_err[precision] = h.apply(xe).to(torch.complex128).cpu()
        del xe
        y = torch.empty_like(x)
        for _ in range(2):
            h.apply(x, y)
        ms = _timed_ms(lambda: h.apply(x, y), 5, 1) / 5
        # the propagators need the Fourier-sphere mask on the kinetic term here: 1/2 |G_max|^2
        # dt / 2 is about 8 on this grid, far past the Taylor step's stability bound
        h.set_fourier_sphere_mask(True)
        cov = [h.cart_to_cov(np.array([a, 0.0, 0.0])) for a in (0.0, 0.01, -0.01, 0.02)]
        ms_etrs = _timed_ms(lambda: h.etrs_step_(x, 0.05, cov[1], cov[2]), 2, 1) / 2
        res = {"apply_ms": ms, "orbital_applies_per_s": M / (ms * 1e-3),
               "etrs_steps_per_s": 1.0 / (ms_etrs * 1e-3), "sphere_points": int(kb["counts"].sum())}
        if precision == "mixed":
            occ = np.full(M, 2.0)
            rho = h.density(x, occ)
            h.ks_potential(rho, vion_d, 2, energies=False)
            h.etrs_scf_step_(x, rho, 0.05, cov[0], cov[1], occ, vion_d, 2)  # warm-up
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            its = [h.etrs_scf_step_(x, rho, 0.05, cov[n], cov[n + 1], occ, vion_d, 2)[0] for n in (1, 2)]
            torch.cuda.synchronize()
            res["scf_etrs_lda"] = {"steps_per_s": 2 / (time.perf_counter() - t0), "scf_iterations": its}
            t0 = time.perf_counter()
            _, spreads, sweeps = h.mlwf_step_(x)
            torch.cuda.synchronize()
            res["tdmlwf_step"] = {"s": time.perf_counter() - t0, "jade_sweeps": sweeps, "maxsweep": 100,
                                  "states": "random plane-wave states after 5 ETRS steps (delocalised: JADE "
                                            "runs to maxsweep)"}
        res["propagation"] = "Fourier-sphere mask on the kinetic term (inqb_set_fourier_sphere_mask)"
        free, total = torch.cuda.mem_get_info()
        res.update({"device_memory_in_use_gb": (total - free) / 1e9,
                    "torch_peak_gb": torch.cuda.max_memory_allocated() / 1e9})
        out[precision] = res
        del x, y, h
    out["mixed_vs_fp64_apply_rel_norm_32_orbitals"] = float((y_err["mixed"] - y_err["fp64"]).norm() /
                                                            y_err["fp64"].norm())
    out["error_input"] = "the same 32 orbitals (the FP64 block rounded to complex64) through both precisions"
    # adjoint on 16 orbitals: 50 steps, checkpoints every 10
    amps = np.random.default_rng(9).normal(0.0, 0.01, 50)
    grads = {}
    for precision in ("fp64", "mixed"):
        torch.cuda.empty_cache()
        h = pb.KSHamiltonian(lattice, nr, precision, device=local)
        h.set_scalar_potential(V)
        h.set_gaussian_projectors(pos, 3.0, 1.0, 1.5, -0.7)
        h.set_fourier_sphere_mask(True)
        psi0 = systems.random_orbitals_device(h, 16, 30.0, seed=4)
        prop = DipolePropagation(h, psi0, np.full(16, 2.0), 0.05, 10)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d = prop.forward(amps, keep=True)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        gA, gV = prop.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        grads[precision] = (d, gA.cpu().numpy(), gV.cpu().numpy())
        out[precision]["adjoint_16_orbitals"] = {"forward_s": t1 - t0, "backward_s": t2 - t1,
                                                 "total_over_forward": (t2 - t0) / (t1 - t0)}
        del prop, psi0, h
    (d64, a64, v64), (d32, a32, v32) = grads["fp64"], grads["mixed"]
    out["adjoint_mixed_vs_fp64"] = {"dipole_rel": abs(d32 - d64) / abs(d64),
                                    "grad_amplitudes_rel": float(np.linalg.norm(a32 - a64) / np.linalg.norm(a64)),
                                    "grad_V_rel": float(np.linalg.norm(v32 - v64) / np.linalg.norm(v64))}
    return out


def run_reference(args):
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return 0
    lattice, nr, pos, V, _ = build_inputs(2, 0)
    res, times = cpu_baseline(lattice, nr, pos, V, seconds=args.cpu_seconds, steps=args.steps,
                              warmup=args.warmup)
    med = statistics.median(times)
    line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": len(times),
            "warmup": args.warmup, "ms_per_step": 1e3 * med, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "precision": "fp64", "sample_orbitals_per_step":
                       int(round(res["value"] * med))},
            "impl": "reference", "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def run_ours(args):
    import torch

    world, rank, local = dist_setup(args.gpus)
    dist = make_pg(world, local)
    import pinq_b200 as pb

    M = args.orbitals
    lattice, nr, pos, V, psi64 = build_inputs(M, seed=rank)
    N = int(np.prod(nr))

    h32 = pb.KSHamiltonian(lattice, nr, "mixed", device=local)
    h64 = pb.KSHamiltonian(lattice, nr, "fp64", device=local)
    for h in (h32, h64):
        h.set_scalar_potential(V)
        kb = h.set_gaussian_projectors(pos, 3.0, 1.0, 1.5, -0.7)
        h.reserve(M)
    nent = int(kb["counts"].sum())
    x64 = torch.as_tensor(psi64).to("cuda")
    x32 = x64.to(torch.complex64)
    y32 = torch.empty_like(x32)
    y64 = torch.empty_like(x64)

    # -- error of the mixed path against the FP64 path and the oracle (all orbitals)
    h32.apply(x32, y32)
    h64.apply(x64, y64)
    torch.cuda.synchronize()
    err_fp64 = float((y32.to(torch.complex128) - y64).norm() / y64.norm())
    err_oracle = None
    if rank == 0:
        import oracle

        o = oracle.System(lattice, nr)
        o.set_potential(V)
        o.set_projectors(o.build_gaussian_kb(pos))
        # every orbital of the workload (the oracle's H|psi> costs about 23 ms per
        # orbital and thread at 64^3)
        sub = np.ascontiguousarray(psi64)
        ref = o.apply_h(sub)
        mixed = y32.cpu().numpy().astype(np.complex128)
        fp64 = y64.cpu().numpy()
        eps_ref = o.band_energies(sub, ref)
        eps32 = h32.band_energies(x32, y32)
        eps64 = h64.band_energies(x64, y64)
        err_oracle = {"mixed_rel_norm": float(np.linalg.norm(mixed - ref) / np.linalg.norm(ref)),
                      "fp64_rel_max": float(np.abs(fp64 - ref).max() / np.abs(ref).max()),
                      "band_energies_mixed_rel_max": float(np.abs(eps32 - eps_ref).max() / np.abs(eps_ref).max()),
                      "band_energies_fp64_rel_max": float(np.abs(eps64 - eps_ref).max() / np.abs(eps_ref).max()),
                      "orbitals_checked": int(sub.shape[1])}

    def timed(fn, K, W):
        for _ in range(W):
            fn()
        barrier(dist)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(K):
            fn()
        e.record()
        torch.cuda.synchronize()
        barrier(dist)
        return max_over_ranks(dist, s.elapsed_time(e))

    K, W = args.steps, max(3, args.warmup)
    # -- headline: mixed H|psi>, device-resident inputs (268 MB > L2), live per-pass events
    clocks = ClockSampler(local)
    for _ in range(W):  # warm-up, untimed
        h32.apply(x32, y32)
    clocks.start()
    h32.timing_start(K)  # CUDA events around the three passes of each timed apply
    barrier(dist)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(K):
        h32.apply(x32, y32)
    e.record()
    torch.cuda.synchronize()
    barrier(dist)
    ms = max_over_ranks(dist, s.elapsed_time(e))
    clk = clocks.stop()
    pass_ms, napplies = h32.timing_stop()

    # -- the two forms of the KB projection (deterministic both): fused into the first
    # tile pass (the default, timed above) and its own gather-and-contract kernel
    # (tcgen05 TF32 tensor cores with a split-precision correction in the mixed
    # precision, CUDA cores in FP64); per-pass CUDA-event times
    proj_forms = {}
    Kp = max(5, K // 4)
    for name, h, x, y in (("mixed", h32, x32, y32), ("fp64", h64, x64, y64)):
        for form in ("fused", "kernel"):
            h.set_projection_mode(form)
            for _ in range(W):
                h.apply(x, y)
            torch.cuda.synchronize()
            h.timing_start(Kp)
            for _ in range(Kp):
                h.apply(x, y)
            pms, pn = h.timing_passes()
            proj_forms[f"{name}_{form}"] = {"apply_ms": float(sum(pms)) / pn,
                                            "passes_ms": {"projection_kernel": pms[0] / pn, "tile_fwd": pms[1] / pn,
                                                          "tile_x": pms[2] / pn, "tile_inv": pms[3] / pn}}
        h.set_projection_mode("fused")
    proj_forms["engines"] = {"fused": "CUDA cores inside the first tile pass: FP32 products, FP64 sums per "
                                      "(plane, half, atom), fixed-order finish in the second pass",
                             "kernel_mixed": "tcgen05.mma kind::tf32, M=128 N=16, 3xTF32 split, FP64 sums per "
                                             "32-point chunk",
                             "kernel_fp64": "CUDA cores, FP64"}

    # -- FP64 H|psi>
    ms64 = timed(lambda: h64.apply(x64, y64), max(3, K // 2), W)
    k64 = max(3, K // 2)
    # -- ETRS steps (mixed and FP64) on the same system, A_x changing every step
    amps = np.random.default_rng(5).normal(0.0, 0.01, args.etrs_steps + W + 2)
    xe32 = x32.clone()
    xe64 = x64.clone()
    cov = [h32.cart_to_cov(np.array([a, 0.0, 0.0])) for a in amps]
    it = {"n": 0}

    def etrs(h, x):
        n = it["n"] % (len(cov) - 1)
        h.etrs_step_(x, 0.05, cov[n], cov[n + 1])
        it["n"] += 1

    ms_etrs32 = timed(lambda: etrs(h32, xe32), args.etrs_steps, W)
    ms_etrs64 = timed(lambda: etrs(h64, xe64), args.etrs_steps, W)

    # -- the 3-D FFT alone: the library's forward transform (tile passes) against cuFFT's
    # batched C2C (torch.fft.fftn over the three grid axes of the same [N][M] block), a
    # comparison point only; 2 N M b algorithmic bytes per transform
    fft = {}
    Kf = max(5, K // 10)
    for name, h, x in (("mixed", h32, x32), ("fp64", h64, x64)):
        yf = torch.empty_like(x)
        ms_ours = timed(lambda: h.to_fourier(x, yf), Kf, W)
        xv = x.view(nr[0], nr[1], nr[2], x.shape[1])
        ms_cufft = timed(lambda: torch.fft.fftn(xv, dim=(0, 1, 2)), Kf, W)
        nb = 2.0 * x.numel() * x.element_size()
        fft[name] = {"ours_ms": ms_ours / Kf, "cufft_ms": ms_cufft / Kf,
                     "ours_GBps": nb / (ms_ours / Kf * 1e-3) / 1e9, "cufft_GBps": nb / (ms_cufft / Kf * 1e-3) / 1e9,
                     "cufft_over_ours": ms_cufft / ms_ours}
        del yf
    if rank == 0:
        import scipy.fft

        xs16 = x64[:, :16].cpu().numpy().reshape(nr[0], nr[1], nr[2], 16)
        nthr = os.cpu_count() or 1
        scipy.fft.fftn(xs16, axes=(0, 1, 2), workers=nthr)
        t0 = time.perf_counter()
        for _ in range(3):
            scipy.fft.fftn(xs16, axes=(0, 1, 2), workers=nthr)
        t_sp = (time.perf_counter() - t0) / 3
        fft["cpu_scipy"] = {"kind": "scipy.fft twin", "cores": nthr, "sample": "16 of the 128 orbitals, complex128",
                            "ms": 1e3 * t_sp, "orbital_transforms_per_s": 16 / t_sp}
    fft["timing"] = "CUDA events over device-resident blocks; cuFFT plan made in the warm-up"

    # -- Crank-Nicolson steps (steepest-descent sweeps to a residual of 1e-10), 2 steps each
    cn = {}
    for name, h, x in (("mixed", h32, x32), ("fp64", h64, x64)):
        xc = x[:, :32].clone()
        h.crank_nicolson_step_(xc, 0.05, cov[0], cov[1], 300, 1e-10)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sweeps = [h.crank_nicolson_step_(xc, 0.05, cov[n], cov[n + 1], 300, 1e-10)[0] for n in range(2)]
        torch.cuda.synchronize()
        cn[f"{name}_steps_per_s"] = 2 / (time.perf_counter() - t0)
        cn[f"{name}_sweeps_per_step"] = sweeps
    cn.update({"orbitals": 32, "dt": 0.05, "tol": 1e-10, "H_applies_per_sweep": 10,
               "timing": "wall clock around device-synchronised calls (one read-back per sweep)"})

    # -- ETRS with the LDA self-consistency loop (Hartree + LDA exchange-correlation
    # rebuilt from the density on the device), all 128 orbitals, from the same start
    scf = {}
    vion_d = torch.as_tensor(V, dtype=torch.float64, device="cuda")
    occ_all = np.full(x64.shape[1], 2.0)
    n_scf = 3
    for name, h, x in (("mixed", h32, x32), ("fp64", h64, x64)):
        xs = x.clone()
        rho_s = h.density(xs, occ_all)
        h.ks_potential(rho_s, vion_d, 2, energies=False)
        h.etrs_scf_step_(xs, rho_s, 0.05, cov[0], cov[1], occ_all, vion_d, 2)  # warm-up step
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        its = []
        for n in range(1, 1 + n_scf):
            k_, en_ = h.etrs_scf_step_(xs, rho_s, 0.05, cov[n], cov[n + 1], occ_all, vion_d, 2)
            its.append(k_)
        torch.cuda.synchronize()
        scf[f"{name}_steps_per_s"] = n_scf / (time.perf_counter() - t0)
        scf[f"{name}_scf_iterations"] = its
        scf[f"{name}_energies"] = en_
        scf[f"{name}_dipole"] = h.dipole(rho_s).tolist()
        h.set_scalar_potential(V)
    scf["mixed_vs_fp64_energy_rel"] = {k: abs(scf["mixed_energies"][k] - scf["fp64_energies"][k]) /
                                       max(abs(scf["fp64_energies"][k]), 1e-300) for k in scf["fp64_energies"]}
    scf.update({"theory": "LDA (Hartree + Slater exchange + Perdew-Zunger correlation)", "orbitals": int(x64.shape[1]),
                "dt": 0.05, "nscf": 5, "threshold": 5e-5, "steps": n_scf,
                "H_applies_per_step": "4 + 4 per SCF iteration",
                "timing": "wall clock around device-synchronised calls (one read-back per SCF iteration)"})

    # -- e2e through the host-buffer C-ABI call (pinned host memory, copies in the timed region)
    xh = x32.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    Ke = max(3, K // 4)
    for _ in range(2):
        h32.apply_host(xh, yh)
    barrier(dist)
    t0 = time.perf_counter()
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record()
    for _ in range(Ke):
        h32.apply_host(xh, yh)
    e2.record()
    torch.cuda.synchronize()
    barrier(dist)
    ms_e2e = max_over_ranks(dist, s2.elapsed_time(e2))
    wall_e2e = time.perf_counter() - t0

    # -- TD-MLWF after a step (mlwf_properties::calculate): the six matrices, JADE, the
    # rotation of all 128 orbitals, centres and spreads; per-phase CUDA-event times
    # states: 128 Gaussians (sigma 1 bohr) on the 64 atoms and 64 bond midpoints,
    # orthonormalised and mixed by a seeded unitary, built on the device
    mlwf = {}
    lat_t = torch.tensor(np.asarray(lattice, float).reshape(3, 3), dtype=torch.float64, device="cuda")
    fr = [torch.tensor(np.where(np.arange(n) >= (n + 1) // 2, np.arange(n) - n, np.arange(n)) / n,
                       dtype=torch.float64, device="cuda") for n in nr]
    fx, fy, fz = torch.meshgrid(fr[0], fr[1], fr[2], indexing="ij")
    rr = torch.stack([fx.reshape(-1), fy.reshape(-1), fz.reshape(-1)], 1) @ lat_t
    centres_w = np.concatenate([pos, pos + 10.26 / 8.0])
    loc = torch.empty((rr.shape[0], len(centres_w)), dtype=torch.complex128, device="cuda")
    for j, c in enumerate(centres_w):
        d = rr - torch.tensor(c, dtype=torch.float64, device="cuda")
        d -= 20.52 * torch.round(d / 20.52)
        loc[:, j] = torch.exp(-(d * d).sum(1) / 2.0)
    h64.orthonormalize_(loc)
    g_mix = torch.Generator(device="cpu").manual_seed(11)
    qm, _ = torch.linalg.qr(torch.randn(len(centres_w), len(centres_w), dtype=torch.complex128, generator=g_mix))
    loc = loc @ qm.to("cuda")
    del rr, fx, fy, fz
    for name, h, x in (("mixed", h32, loc.to(torch.complex64)), ("fp64", h64, loc)):
        xm = x.clone()
        t0 = time.perf_counter()
        _, _, k_first = h.mlwf_step_(xm)  # the first transform un-mixes the states
        torch.cuda.synchronize()
        mlwf[f"{name}_first_ms"] = 1e3 * (time.perf_counter() - t0)
        mlwf[f"{name}_first_jade_sweeps"] = k_first
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n_m = 3
        sw = []
        for _ in range(n_m):
            _, spreads_m, k_ = h.mlwf_step_(xm)
            sw.append(k_)
        torch.cuda.synchronize()
        mlwf[f"{name}_ms_per_step"] = 1e3 * (time.perf_counter() - t0) / n_m
        mlwf[f"{name}_jade_sweeps"] = sw
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(n_m):
            h.mlwf_matrices(xm)
        s1.record()
        torch.cuda.synchronize()
        ms_g = s0.elapsed_time(s1) / n_m
        M_ = xm.shape[1]
        mlwf[f"{name}_matrices_ms"] = ms_g
        # 3 weighted Gram products: 3 N M^2 complex multiply-adds = 24 N M^2 flops
        mlwf[f"{name}_matrices_tflops"] = 24.0 * xm.shape[0] * M_ * M_ / (ms_g * 1e-3) / 1e12
        mlwf[f"{name}_mean_spread"] = float(np.mean(spreads_m))
    mlwf.update({"states": "128 Gaussians (sigma 1 bohr) on the 64 atoms and 64 bond midpoints, orthonormalised "
                           "and mixed by a seeded unitary; steps after the first start in the localised gauge",
                 "orbitals": int(x64.shape[1]), "maxsweep": 100, "tol": 1e-8,
                 "timing": "step: wall clock around synchronised calls (one read-back per JADE sweep); "
                           "matrices: CUDA events"})

    # -- the oracle (CPU, FP64, all host threads) on bounded samples of the same two
    # workloads, reported beside them: one SCF ETRS step of 16 orbitals, and the TD-MLWF
    # matrices + JADE for 32 of the localised states
    if rank == 0:
        import oracle

        o = oracle.System(lattice, nr)
        o.set_potential(V)
        o.set_projectors(o.build_gaussian_kb(pos))
        ps = np.ascontiguousarray(x64[:, :16].cpu().numpy())
        occ16 = np.full(16, 2.0)
        rho16 = o.density(ps, occ16)
        o.ks_potential(rho16, V, 2)
        t0 = time.perf_counter()
        _, _, it_c, _ = o.etrs_scf_step(ps, rho16, 0.05, cov[1], cov[2], occ16, V, 2)
        t_c = time.perf_counter() - t0
        scf["cpu_reference"] = {"kind": "port", "cores": oracle.num_threads(), "sample": "one SCF ETRS step of 16 of "
                                "the 128 orbitals (oracle, FP64)", "seconds": t_c, "scf_iterations": it_c,
                                "orbital_steps_per_s": 16 / t_c}
        scf["mixed_orbital_steps_per_s"] = scf["mixed_steps_per_s"] * x64.shape[1]
        # 32 of the states as the TD-MLWF steps left them (localised gauge, FP64)
        ls = np.ascontiguousarray(xm[:, :32].cpu().numpy())
        t0 = time.perf_counter()
        a_c = o.mlwf_matrices(ls)
        t1 = time.perf_counter()
        _, _, _, sw_c = oracle.jade(a_c)
        t2 = time.perf_counter()
        mlwf["cpu_reference"] = {"kind": "port", "cores": oracle.num_threads(), "sample": "matrices and JADE for 32 of "
                                 "the 128 states in the localised gauge (oracle, FP64)", "matrices_s": t1 - t0, "jade_s": t2 - t1,
                                 "jade_sweeps": sw_c}
        del o

    # -- checkpoint in INQ's restart layout: all 128 orbitals (complex128 files) + density
    ckpt = None
    if rank == 0:
        import shutil

        from pinq_b200.checkpoint import RealTimeResults, load_checkpoint, save_checkpoint

        cdir = tempfile.mkdtemp(prefix="inqb_ckpt_")
        try:
            occ_c = np.full(x64.shape[1], 2.0)
            rho_c = h64.density(x64, occ_c)
            res_c = RealTimeResults()
            res_c.record(0, 0.0, 0.0, (0.0, 0.0, 0.0))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            save_checkpoint(cdir, h64, x64, occ_c, rho_c, res_c)
            t_save = time.perf_counter() - t0
            back_c = torch.empty_like(x64)
            rho_b = torch.empty_like(rho_c)
            t0 = time.perf_counter()
            load_checkpoint(cdir, h64, back_c, rho_b)
            torch.cuda.synchronize()
            t_load = time.perf_counter() - t0
            nbytes = x64.numel() * 16 + rho_c.numel() * 8
            ckpt = {"bytes": int(nbytes), "save_s": t_save, "load_s": t_load,
                    "save_GBps": nbytes / t_save / 1e9, "load_GBps": nbytes / t_load / 1e9,
                    "exact_round_trip": bool(torch.equal(back_c, x64) and torch.equal(rho_b, rho_c)),
                    "layout": "INQ restart layout (one complex128 file per state + occupations + density)",
                    "storage": "local temporary directory of the GPU host"}
        finally:
            shutil.rmtree(cdir, ignore_errors=True)

    cells = bench_cells(args, local) if args.cells else None
    adj = bench_adjoint(args, local) if args.adjoint else None
    big = bench_cfg4(args, local) if args.cfg4 and world == 1 else None

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    hbm, bf16, peak_kind = peaks()
    b = 8  # bytes per complex64
    bT = 4
    L = 4
    rec = 32  # bytes of one sphere-entry record (phase, L radial values, offset, segment)
    alg = {  # algorithmic bytes per launch
        # orbitals in, Fourier tiles out, the entry records once
        "tile_fwd": 2 * N * M * b + nent * rec,
        # Fourier tiles in and out
        "tile_x": 2 * N * M * b,
        # Fourier tiles and orbitals in, H psi out, V, the records and the per-point index once
        "tile_inv": 3 * N * M * b + N * bT + nent * rec + 4 * N,
    }
    per_launch_ms = {k: pass_ms[i] / max(1, napplies) for i, k in enumerate(["tile_fwd", "tile_x", "tile_inv"])}
    kernels = {}
    traffic = profiled_traffic()
    for k in alg:
        t = per_launch_ms[k] * 1e-3
        gbs = alg[k] / t / 1e9 if t > 0 else 0.0
        kernels[k] = {"ms_per_launch": per_launch_ms[k], "algorithmic_bytes": alg[k], "achieved_gbs": gbs,
                      "frac": gbs / hbm, "traffic": traffic.get(k)}
    dom = max(kernels, key=lambda k: kernels[k]["ms_per_launch"])
    d = kernels[dom]
    B_H = 2 * N * M * b + N * bT + nent * L * bT
    apply_ms = ms / K
    value = world * M * K / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": apply_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Gaussian orbitals, Gaussian local potential and KB projectors)",
        "config": {"workload": WORKLOAD, "precision": "mixed: complex64 FFT/pointwise, FP64 projection sums",
                   "grid": list(nr), "orbitals_per_gpu": M, "atoms": len(pos), "projectors": 4 * len(pos),
                   "sphere_points": nent, "l2": "inputs larger than L2 (268 MB orbital block > 126 MB L2)",
                   "parallelism": f"orbital replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": d["achieved_gbs"], "peak": hbm, "unit": "GB/s",
                     "frac": d["frac"], "traffic": d["traffic"], "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": d["algorithmic_bytes"]},
        "roofline_apply": {"B_H_bytes": B_H, "achieved_gbs": B_H / (apply_ms * 1e-3) / 1e9,
                           "frac": B_H / (apply_ms * 1e-3) / 1e9 / hbm},
        "kernels": kernels,
        "e2e": {"value": world * M * Ke / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": N * M * b,
                "d2h_bytes_per_step": N * M * b, "wall_s": wall_e2e, "call": "inqb_apply_h_host"},
        "gpu_launches": 3 * K,
        "clocks": clk,
        "fp64": {"value": world * M * k64 / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64 / k64,
                 "speedup_mixed_over_fp64": (ms64 / k64) / apply_ms},
        "etrs": {"mixed_steps_per_s": world * args.etrs_steps / (ms_etrs32 * 1e-3),
                 "fp64_steps_per_s": world * args.etrs_steps / (ms_etrs64 * 1e-3),
                 "H_applies_per_step": 8, "dt": 0.05},
        "fft": fft,
        "projection_forms": proj_forms,
        "crank_nicolson": cn,
        "etrs_scf": scf,
        "checkpoint": ckpt,
        "mlwf": mlwf,
        "error": {"mixed_vs_fp64_gpu_rel_norm": err_fp64, "vs_oracle": err_oracle},
    }
    if cells is not None:
        line["cells"] = cells
    if adj is not None:
        line["adjoint"] = adj
    if big is not None:
        line["cfg4"] = big
    if world == 1:
        try:
            res, _ = cpu_baseline(lattice, nr, pos, V, seconds=args.cpu_seconds, warmup=2)
            line["cpu_baseline"] = res
        except Exception as ex:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(ex)}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
