#!/usr/bin/env python
"""Throughput of the fused D3Q19 step on B200 (MLUPS), one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl wt|reference]

Workload (default): the 256x128x128 channel with a 15-degree-yawed
superellipsoid hull (80x30x24 cells, 20000 triangles with a seeded bump
field, voxelised on the GPU by Voxel.build), u0 = 0.06, Re = 2000 on the length
(tau = 0.5072), TRT Lambda = 3/16, Smagorinsky Cs = 0.1, free-slip side
planes, seeded +-1e-4 velocity noise. A "step" is one lattice time step
over all 4,194,304 cells; MLUPS counts every cell (the reference's
convention, js/main.js:621).

* value      kernel throughput: K steps of one wt_step call, inputs resident
             in HBM, CUDA events on the library's stream.
* e2e        the same metric through the public per-step call a host makes
             (LBM.step(): parameters pushed, one step, the force read back
             to host memory, synchronous).
* fp16dev    the half-deviation storage form on the same workload.
* accuracy   pair-averaged Cd / Cl of FP32, FP16-dev and FP64 storage after
             the workload's 10000 steps (average over the last 2000).
* roofline   152 (FP32) algorithmic bytes per cell update over the measured
             HBM copy bandwidth.
* cpu_baseline  the CPU oracle (the reference arithmetic in C, OpenMP z-slabs
             as js/pool.js decomposes them) timed on this host's cores.

--impl reference times that CPU implementation alone on the same workload.
Multi-GPU (torchrun): every rank runs an independent replica (the reference
has no exchange step to shard); value = all cells of all ranks / max time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = ("MLUPS FP32 vs FP16-store at |ΔCd|<1% vs FP64; "
          "adjoint grad time / forward time")
BYTES_PER_CELL = {"f32": 152, "f16dev": 76, "f64": 304}
FALLBACK_HBM_GBS = 6650.0

from windtunnel_b200.workloads import WORKLOADS, channel_lattice  # noqa: E402


# ---------------------------------------------------------------------------- set-up
def setup_gpu(wl, storage, math_mode="fast", kernel="auto"):
    return channel_lattice(wl, storage, math_mode, kernel)


def setup_oracle(wl):
    """The workload on the CPU oracle: the same hull voxelised by the oracle's
    Voxel.build (bit-identical to the GPU's), the same lookup, parameters
    and seeded state."""
    from oracle.oracle import OracleLBM, lookup_mask, voxel_build as oracle_voxel_build
    from windtunnel_b200.workloads import hull_triangles, placement, set_params
    o = OracleLBM(wl["nx"], wl["ny"], wl["nz"], "f32", side_bc=wl["side_bc"])
    set_params(o, wl)
    b = wl["body"]
    grid, info = oracle_voxel_build(hull_triangles(b, wl["seed"]), b["res"])
    M, P, box = placement(wl, info["ext"])
    mask = lookup_mask(grid, info["min"], info["inv"], M, P, b["scale"], wl["nx"], wl["ny"],
                       wl["nz"], box)
    o.voxelize_mask(box, mask)
    o.init_eq_noise(wl["seed"], wl["amp"])
    return o


def host_cpus() -> list[int]:
    try:
        return sorted(os.sched_getaffinity(0))
    except AttributeError:
        return list(range(os.cpu_count() or 1))


def host_threads() -> int:
    """Hardware threads this process may run on."""
    return len(host_cpus())


def physical_cores() -> int:
    """Distinct (package, core) pairs among the CPUs this process may run on;
    the hardware-thread count when the topology is not readable."""
    seen = set()
    for c in host_cpus():
        t = Path(f"/sys/devices/system/cpu/cpu{c}/topology")
        try:
            seen.add((t.joinpath("physical_package_id").read_text().strip(),
                      t.joinpath("core_id").read_text().strip()))
        except OSError:
            return host_threads()
    return len(seen) or host_threads()


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return self
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()
        time.sleep(0.3)   # first sample before the region starts
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=5)
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "power_w_max": max(power) if power else None, "samples": len(sm),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------- helpers
def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel_tag: str) -> float | None:
    """DRAM bytes per launch from the committed ncu summary of this kernel, if any."""
    p = ROOT / "profiles" / f"{kernel_tag}.md"
    try:
        m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", p.read_text())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class Dist:
    """One rank per GPU from the torchrun environment: barriers and the max of
    a time over ranks. backend "nccl" (the GPU runs) or "gloo" (CPU ranks,
    which the tests use)."""

    def __init__(self, backend: str = "nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = False

    def init(self):
        import datetime

        import torch
        if self.backend == "nccl":
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch.distributed as dist
            kw = {"device_id": torch.device("cuda", self.local)} if self.backend == "nccl" else {}
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=180), **kw)
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        import torch.distributed as dist
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


def whole_job_mlups(world: int, cells: int, steps: int, ms_max: float) -> float:
    """Replicas: every rank steps its own lattice of `cells` cells, so the job
    updates world x cells x steps cells in the slowest rank's time."""
    return world * cells * steps / (ms_max * 1e-3) / 1e6


def timed_steps(sim, K: int, dist: Dist) -> tuple[float, int]:
    """K steps in one wt_step call, CUDA events on the library stream; (ms, launches)."""
    import torch
    stream = torch.cuda.ExternalStream(sim.stream)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = sim.launch_count
    dist.barrier()
    torch.cuda.synchronize()
    start.record(stream)
    sim.step_forces(K)
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    return start.elapsed_time(end), sim.launch_count - l0


def e2e_steps(sim, K: int, dist: Dist, batch: int = 1) -> float:
    """K steps through the public calls, `batch` steps per call: push the
    parameters, step, read the force series to host. batch = 1 is
    LBM.step() (js/lbm.js:285-291) once per step; batch = 16 is
    Pool.step(16) (js/pool.js:97-125), the reference's batched executor."""
    import torch
    stream = torch.cuda.ExternalStream(sim.stream)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p = sim.params()
    dist.barrier()
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(K // batch):
        sim.set_params(u0=p.u0, tau=p.tau)   # the host's per-call parameter push
        if batch == 1:
            sim.step()
            _ = sim.force                     # force of this step, in host memory
        else:
            _ = sim.step_forces(batch)        # per-step force series, in host memory
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    return start.elapsed_time(end)


def pair_avg_coeff(forces, u0, area, window):
    import numpy as np
    f = np.asarray(forces, np.float64)
    pa = 0.5 * (f[1:] + f[:-1])
    q = 0.5 * u0 * u0 * area
    w = pa[-window:]
    return float(w[:, 0].mean() / q), float(w[:, 1].mean() / q)


ACCURACY_FORMS = (("f64", "f64", "exact", None), ("f32", "f32", "fast", None),
                  ("f16dev", "f16dev", "fast", "nearest"),
                  ("f16dev_stochastic", "f16dev", "fast", "stochastic"))


def accuracy_study(wl, replicas: int = 4, steps: int | None = None,
                   window: int | None = None) -> dict:
    """Cd / Cl of every storage form against float64 storage, as ensemble means.

    The hull's wake at Re 2000 is chaotic: two arithmetic forms (float32
    included) follow different trajectories after a few thousand steps, so
    one run's window average carries a sampling error of several percent of
    Cd. Each form therefore runs `replicas` seeded copies of the workload
    (initial velocity noise seeds seed, seed+1, ...; the same seeds for every
    form) for the configuration's step count and takes the pair-averaged
    coefficients over the last `window` steps of each (js/main.js:113-127).
    A form's Cd is the mean over its replicas with the standard error
    std / sqrt(replicas); its error against float64 (and float32) is the mean
    of the per-seed differences, with their standard error."""
    import numpy as np

    from windtunnel_b200.stats import window_coefficients
    steps = steps or wl["accuracy_steps"]
    window = window or wl["accuracy_window"]
    out = {"workload": wl["name"], "steps": steps, "window": window, "replicas": replicas,
           "seeds": [wl["seed"] + k for k in range(replicas)],
           "statistic": "mean over seeded replicas of the pair-averaged coefficient over "
                        "the last `window` steps; sem = std / sqrt(replicas)"}
    per, first = {}, {}
    for name, storage, mm, rounding in ACCURACY_FORMS:
        sim = setup_gpu(wl, storage, mm)
        if rounding:
            sim.set_params(f16_rounding=rounding)
        cd, cl = [], []
        t0 = time.time()
        for k in range(replicas):
            sim.init_eq_noise(wl["seed"] + k, wl["amp"])
            F = sim.step_forces(steps)
            c = window_coefficients(F, wl["u0"], sim.frontalArea, window)
            cd.append(c["cd"])
            cl.append(c["cl"])
            if k == 0:
                first[name] = (F, sim.frontalArea)
        sim.close()
        per[name] = (np.array(cd), np.array(cl))
        e = {"cd": float(np.mean(cd)), "cl": float(np.mean(cl)),
             "cd_sem": float(np.std(cd, ddof=1) / math.sqrt(replicas)) if replicas > 1 else None,
             "cl_sem": float(np.std(cl, ddof=1) / math.sqrt(replicas)) if replicas > 1 else None,
             "cd_replicas": [round(v, 6) for v in cd], "wall_s": round(time.time() - t0, 2)}
        if rounding:
            e["rounding"] = rounding
        out[name] = e
    # the storage error before the flow separates the trajectories: the
    # first seed's pair-averaged Cd over consecutive 500-step windows, every
    # form against float64 from the same initial state
    F64, area = first["f64"]
    q = 0.5 * wl["u0"] ** 2 * area
    def wcd(F, a, b):
        pa = 0.5 * (F[1:, 0] + F[:-1, 0])
        return float(pa[a:b].mean() / q)
    rows = []
    for a in range(0, steps - 1, 500):
        b = min(a + 500, steps - 1)
        ref = wcd(F64, a, b)
        rows.append({"steps": [a, b + 1], "cd_f64": ref,
                     **{f"dcd_rel_{n}": (wcd(first[n][0], a, b) - ref) / abs(ref)
                        for n in first if n != "f64"}})
    out["seed0_windows"] = rows
    for ref in ("f64", "f32"):
        rcd, rcl = per[ref]
        for name, (cd, cl) in per.items():
            if name == ref or (ref == "f32" and name == "f64"):
                continue
            dcd, dcl = cd - rcd, cl - rcl
            sem = float(np.std(dcd, ddof=1) / math.sqrt(replicas)) if replicas > 1 else None
            out[name][f"dcd_rel_vs_{ref}"] = float(np.mean(dcd) / np.mean(rcd))
            out[name][f"dcd_rel_vs_{ref}_sem"] = sem / abs(float(np.mean(rcd))) if sem else None
            out[name][f"dcl_vs_{ref}_over_cd"] = float(np.mean(dcl) / np.mean(rcd))
    return out


def long_window_accuracy(wl, steps: int, spinup: int | None = None, block: int = 10000,
                         forms: list[str] | None = None, noise_seed: int | None = None) -> dict:
    """Cd / Cl of each storage form over one long window, against float64.

    One trajectory per form from the workload's seed (or `noise_seed` for the
    initial velocity noise, the body unchanged): `spinup` steps (the
    configuration's step count) and then `steps` steps whose pair-averaged
    drag and lift (js/main.js:113-127) are summed into blocks of `block`
    steps. A form's Cd is the mean over its blocks; its standard error is
    std(block means) / sqrt(blocks), the batch-means estimate behind the
    reference's blocking SEM (js/main.js:163-212), given for block lengths 1,
    2, 5 and 10 times `block` so that its plateau shows that the blocks are
    long enough to be independent. The forms' trajectories separate within
    the spin-up, so the error of a form against float64 (or float32) has the
    standard error sqrt(sem_a^2 + sem_b^2). Each form's entry is printed
    to stderr as it completes."""
    import numpy as np

    spinup = wl["accuracy_steps"] if spinup is None else spinup
    nb = steps // block
    steps = nb * block
    chunk = block * max(1, 200000 // block)
    seed = wl["seed"] if noise_seed is None else noise_seed
    out = {"workload": wl["name"], "seed": seed, "spinup": spinup, "steps": steps,
           "block": block,
           "statistic": "pair-averaged coefficient over `steps` steps after `spinup`; sem = "
                        "std(block means) / sqrt(blocks)"}
    per = {}
    for name, storage, mm, rounding in ACCURACY_FORMS:
        if forms and name not in forms:
            continue
        sim = setup_gpu(wl, storage, mm)
        if rounding:
            sim.set_params(f16_rounding=rounding)
        if noise_seed is not None:
            sim.init_eq_noise(noise_seed, wl["amp"])
        q = 0.5 * wl["u0"] ** 2 * sim.frontalArea
        t0 = time.time()
        last = sim.step_forces(spinup)[-1] if spinup else np.zeros(3)
        sums = np.zeros((nb, 2))
        done = 0
        while done < steps:
            F = sim.step_forces(min(chunk, steps - done))
            pa = 0.5 * (F + np.vstack([last[None, :], F[:-1]]))
            sums[done // block:(done + len(F)) // block] = \
                pa[:, :2].reshape(-1, block, 2).sum(axis=1)
            last = F[-1]
            done += len(F)
        sim.close()
        means = sums / (block * q)
        cd = float(means[:, 0].mean())
        cl = float(means[:, 1].mean())

        def sem(col, m):
            k = nb // m
            if k < 2:
                return None
            b = col[:k * m].reshape(k, m).mean(axis=1)
            return float(np.std(b, ddof=1) / math.sqrt(k))
        e = {"cd": cd, "cl": cl, "cd_sem": sem(means[:, 0], 1), "cl_sem": sem(means[:, 1], 1),
             "cd_sem_by_block": {str(m * block): sem(means[:, 0], m) for m in (1, 2, 5, 10)},
             "wall_s": round(time.time() - t0, 1)}
        if rounding:
            e["rounding"] = rounding
        per[name] = e
        out[name] = e
        print(json.dumps({name: e}), file=sys.stderr, flush=True)
    for ref in ("f64", "f32"):
        if ref not in per:
            continue
        r = per[ref]
        for name, e in per.items():
            if name == ref or (ref == "f32" and name == "f64"):
                continue
            e[f"dcd_rel_vs_{ref}"] = (e["cd"] - r["cd"]) / abs(r["cd"])
            e[f"dcd_rel_vs_{ref}_sem"] = math.hypot(e["cd_sem"], r["cd_sem"]) / abs(r["cd"])
            e[f"dcl_vs_{ref}_over_cd"] = (e["cl"] - r["cl"]) / abs(r["cd"])
    return out


def steady_accuracy(wl) -> dict:
    """The storage error alone, on a steady wake: one run per form, Cd / Cl
    over the last window steps against float64 storage."""
    from windtunnel_b200.stats import window_coefficients
    out = {"workload": wl["name"], "steps": wl["accuracy_steps"],
           "window": wl["accuracy_window"]}
    ref = None
    for name, storage, mm, rounding in ACCURACY_FORMS:
        sim = setup_gpu(wl, storage, mm)
        if rounding:
            sim.set_params(f16_rounding=rounding)
        c = window_coefficients(sim.step_forces(wl["accuracy_steps"]), wl["u0"], sim.frontalArea,
                                wl["accuracy_window"])
        sim.close()
        e = {"cd": c["cd"], "cl": c["cl"]}
        if ref is None:
            ref = e
        else:
            e["dcd_rel_vs_f64"] = abs(e["cd"] - ref["cd"]) / abs(ref["cd"])
        out[name] = e
    return out


# ---------------------------------------------------------------------------- adjoint
ADJOINT_WORKLOADS = {
    "design128": dict(
        name="128x64x64 channel, 32^3 partial-bounce-back design box at (40,32,32), Re=100",
        nx=128, ny=64, nz=64, u0=0.05, tau=0.53, csm=0.1, lam=3 / 16, les=True,
        side_bc="freeslip", box=(24, 16, 16, 56, 48, 48), centre=(40.0, 32.0, 32.0),
        radius=10.0, width=1.5, noise=0.05, seed=1234, amp=1e-4, steps=1500, window=500,
        checkpoint=50, storage="f32", fd_cells=16, fd_eps=1e-3),
    "design384": dict(
        name="384x160x160 channel, 64^3 partial-bounce-back design box at (120,80,80), Re=1000",
        nx=384, ny=160, nz=160, u0=0.05, tau=0.506, csm=0.1, lam=3 / 16, les=True,
        side_bc="freeslip", box=(88, 48, 48, 152, 112, 112), centre=(120.0, 80.0, 80.0),
        radius=20.0, width=1.5, noise=0.05, seed=1234, amp=1e-4, steps=4000, window=1000,
        checkpoint=0, storage="f16dev", fd_cells=0, fd_eps=0.0),
}


def design_field(aw) -> "np.ndarray":
    """s = (1 - tanh((|x - c| - r) / w)) / 2 + U(-noise, noise), clipped to [0, 1]."""
    import numpy as np
    x0, y0, z0, x1, y1, z1 = aw["box"]
    zz, yy, xx = np.meshgrid(np.arange(z0, z1) + 0.5, np.arange(y0, y1) + 0.5,
                             np.arange(x0, x1) + 0.5, indexing="ij")
    cx, cy, cz = aw["centre"]
    r = np.sqrt((xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2)
    rng = np.random.default_rng(aw["seed"])
    s = 0.5 * (1 - np.tanh((r - aw["radius"]) / aw["width"]))
    s = s + rng.uniform(-aw["noise"], aw["noise"], r.shape)
    return np.clip(s, 0.0, 1.0)


def design_lattice(aw, storage, math_mode="fast", s=None, seed=None):
    from windtunnel_b200 import LBM
    sim = LBM(aw["nx"], aw["ny"], aw["nz"], storage=storage, math=math_mode,
              side_bc=aw["side_bc"])
    sim.set_params(u0=aw["u0"], tau=aw["tau"], csm=aw["csm"], les=int(aw["les"]),
                   **{"lambda": aw["lam"]})
    sim.init_eq_noise(aw["seed"] if seed is None else seed, aw["amp"])
    sim.set_solid_fraction(aw["box"], design_field(aw) if s is None else s)
    return sim


def adjoint_study(aw) -> dict:
    """Adjoint gradient time over forward time on a design-box workload, with
    gradient checks: FP64 central differences (when fd_cells > 0), the FP64
    adjoint, and the FP32-storage adjoint against the workload's storage form."""
    import numpy as np
    import torch
    N, W, C = aw["steps"], aw["window"], aw["checkpoint"]
    out = {"workload": aw["name"], "steps": N, "window": W, "storage": aw["storage"],
           "objective": "mean drag (Fx) over the last window steps"}
    # plain forward of the same lattice (events on the library stream)
    sim = design_lattice(aw, aw["storage"])
    sim.step_forces(3)
    sim.close()
    sim = design_lattice(aw, aw["storage"])
    st = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    F = sim.step_forces(N)
    e1.record(st)
    e1.synchronize()
    t_fwd = e0.elapsed_time(e1)
    J_fwd = float(F[-W:, 0].mean())
    sim.close()
    # gradient: forward sweep with checkpoints + recompute + adjoint
    sim = design_lattice(aw, aw["storage"])
    free0 = torch.cuda.mem_get_info()[0]
    e0.record(st := torch.cuda.ExternalStream(sim.stream))
    J, g, stats = sim.adjoint(N, W, 0, C)
    e1.record(st)
    e1.synchronize()
    t_adj = e0.elapsed_time(e1)
    sim.close()
    t_grad = stats["forward_ms"] + stats["backward_ms"]
    out.update(forward_ms=round(t_fwd, 2), gradient_ms=round(t_grad, 2),
               forward_sweep_ms=round(stats["forward_ms"], 2),
               backward_ms=round(stats["backward_ms"], 2),
               ratio=round(stats["backward_ms"] / t_fwd, 3),
               ratio_definition="t(adjoint incl. recompute) / t(one forward run of the same "
                                "steps); gradient_over_forward adds the checkpointing "
                                "forward sweep (device time of both sweeps); "
                                "gradient_call_ms is the whole call on the stream's "
                                "clock, the device-memory allocation of its "
                                "checkpoints included",
               gradient_over_forward=round(t_grad / t_fwd, 3),
               gradient_call_ms=round(t_adj, 2),
               checkpoint_interval=stats["segment"], checkpoints=stats["checkpoints"],
               adjoint_device_bytes=stats["device_bytes"],
               device_free_before_bytes=int(free0), J=J, J_plain_forward=J_fwd)
    # the same call again on a lattice that kept the first call's memory (an
    # optimisation loop): no allocation inside the call
    sim = design_lattice(aw, aw["storage"])
    start = sim.get_state()
    sim.adjoint(N, W, 0, C, keep=True)
    sim.set_state(start)
    e0.record(st := torch.cuda.ExternalStream(sim.stream))
    _, g_kept, _ = sim.adjoint(N, W, 0, C, keep=True)
    e1.record(st)
    e1.synchronize()
    out["gradient_call_ms_kept_memory"] = round(e0.elapsed_time(e1), 2)
    out["kept_memory_same_gradient"] = bool(np.array_equal(g_kept, g))
    sim.close()
    # every state stored (no recomputation) when they fit in the free memory
    pop = 19 * aw["nx"] * aw["ny"] * aw["nz"] * {"f32": 4, "f16dev": 2, "f64": 8}[aw["storage"]]
    if C != N and pop * (N + 3) <= 0.75 * free0:
        sim = design_lattice(aw, aw["storage"])
        e0.record(st := torch.cuda.ExternalStream(sim.stream))
        _, g_all, st_all = sim.adjoint(N, W, 0, N)
        e1.record(st)
        e1.synchronize()
        t_all = e0.elapsed_time(e1)
        sim.close()
        t_g = st_all["forward_ms"] + st_all["backward_ms"]
        out["store_all"] = dict(gradient_ms=round(t_g, 2),
                                forward_sweep_ms=round(st_all["forward_ms"], 2),
                                backward_ms=round(st_all["backward_ms"], 2),
                                ratio=round(st_all["backward_ms"] / t_fwd, 3),
                                gradient_over_forward=round(t_g / t_fwd, 3),
                                gradient_call_ms=round(t_all, 2),
                                adjoint_device_bytes=st_all["device_bytes"],
                                same_gradient=bool(np.array_equal(g_all, g)))
    # the same gradient with float32 storage (for the half-storage forward) or float64
    ref_storage = "f32" if aw["storage"] == "f16dev" else "f64"
    sim = design_lattice(aw, ref_storage, "exact" if ref_storage == "f64" else "fast")
    Jr, gr, _ = sim.adjoint(N, W, 0, C)
    sim.close()
    cos = float((g * gr).sum() / (np.linalg.norm(g) * np.linalg.norm(gr)))
    out[f"vs_{ref_storage}_adjoint"] = {
        "cosine": cos, "rel_l2": float(np.linalg.norm(g - gr) / np.linalg.norm(gr)),
        "J_rel": abs(J - Jr) / abs(Jr)}
    if aw["storage"] == "f16dev":
        # the same agreement within the horizon over which a gradient of the
        # separated wake is reproducible at all (1000 steps, J over the last
        # 250), beside two float32 runs whose initial noise differs
        h = adjoint_horizon_study(aw, horizons=(1000,), window=250)["horizons"][0]
        out["vs_f32_adjoint_1000_steps"] = {"window": 250, **h}
    if aw["fd_cells"]:
        rng = np.random.default_rng(aw["seed"] + 1)
        s0 = design_field(aw)
        eps = aw["fd_eps"]
        # seeded cells whose +-eps perturbation stays inside [0, 1]
        free = np.argwhere((s0 > eps) & (s0 < 1 - eps))
        pick = free[rng.choice(len(free), aw["fd_cells"], replace=False)]
        rows = []
        for idx in map(tuple, pick):
            js = []
            for sgn in (1, -1):
                sv = s0.copy()
                sv[idx] += sgn * eps
                fsim = design_lattice(aw, "f64", "exact", s=sv)
                js.append(float(fsim.step_forces(N)[-W:, 0].mean()))
                fsim.close()
            fd = (js[0] - js[1]) / (2 * eps)
            rows.append((g[idx], gr[idx], fd))
        rows = np.array(rows)
        scale = np.abs(rows[:, 2]).max()
        out["fd_check"] = {
            "cells": aw["fd_cells"], "eps": eps, "fd": "central, float64 storage + arithmetic",
            "max_rel_err_adjoint": float(np.max(np.abs(rows[:, 0] - rows[:, 2]) /
                                                np.maximum(np.abs(rows[:, 2]), 1e-300))),
            "max_err_over_max_fd_adjoint": float(np.max(np.abs(rows[:, 0] - rows[:, 2])) / scale),
            "max_rel_err_f64_adjoint": float(np.max(np.abs(rows[:, 1] - rows[:, 2]) /
                                                    np.maximum(np.abs(rows[:, 2]), 1e-300))),
            "max_err_over_max_fd_f64_adjoint": float(np.max(np.abs(rows[:, 1] - rows[:, 2])) /
                                                     scale)}
    else:
        # drag of the storage form against a float64 run of the same case
        sim = design_lattice(aw, "f64", "exact")
        F64 = sim.step_forces(N)
        sim.close()
        J64 = float(F64[-W:, 0].mean())
        # Cd is J over the same dynamic pressure and area: the relative errors coincide
        out["cd_rel_err_vs_f64"] = abs(J_fwd - J64) / abs(J64)
    return out


def adjoint_horizon_study(aw, horizons=(250, 500, 1000, 2000, 4000), window=250) -> dict:
    """How far the half-storage and float32-storage gradients of one design
    workload agree, against the horizon N (J = mean drag over the last
    `window` steps of N): cosine and relative L2 of dJ/ds, and the relative
    difference of J. Beside it, the same comparison between two float32
    runs whose initial velocity noise differs (seed and seed + 1): the
    agreement two trajectories of one arithmetic keep once the flow has
    separated them, which the half/float32 pair cannot beat."""
    import numpy as np

    def grad(storage, N, seed=None):
        sim = design_lattice(aw, storage, seed=seed)
        J, g, _ = sim.adjoint(N, window, 0, 0)
        sim.close()
        return J, g

    def agree(a, b):
        (Ja, ga), (Jb, gb) = a, b
        return {"cosine": float((ga * gb).sum() / (np.linalg.norm(ga) * np.linalg.norm(gb))),
                "rel_l2": float(np.linalg.norm(ga - gb) / np.linalg.norm(gb)),
                "J_rel": abs(Ja - Jb) / abs(Jb)}

    rows = []
    for N in horizons:
        f32 = grad("f32", N)
        rows.append({"steps": N, "half_vs_f32": agree(grad("f16dev", N), f32),
                     "f32_reseeded_vs_f32": agree(grad("f32", N, aw["seed"] + 1), f32)})
    return {"workload": aw["name"], "window": window,
            "objective": "mean drag over the last window steps", "horizons": rows}


def cpu_baseline(wl, budget_s: float = 24.0) -> dict:
    """The CPU oracle (the reference's arithmetic, z-slabs split over threads as
    js/pool.js splits them) on this host, bounded to about `budget_s` seconds.

    Thread counts follow the reference's own in-app benchmark
    (js/main.js:595-663): one core, then 2, half and all-but-one of the
    hardware threads (at most 16 workers, js/main.js:626-628), best of three
    timings each; the all-threads point is added when it is not among them.
    Each timing is a sample of interior z-planes sized to the budget
    (step_sample: one step's collide/stream/boundary work on those planes).
    `value` is the best point, as the reference's benchmark keeps its best
    worker count."""
    o = setup_oracle(wl)
    hc = host_threads()
    tries = [1] + sorted({v for v in (2, max(2, hc >> 1), max(2, hc - 1)) if 2 <= v <= 16})
    if hc not in tries:
        tries.append(hc)
    nx, ny, nz = wl["nx"], wl["ny"], wl["nz"]
    per = budget_s / len(tries)
    sweep = []
    for t in tries:
        t0 = time.perf_counter()
        o.step_sample(1, nz - 1, t)            # warms the thread team; sizes the sample
        t_full = time.perf_counter() - t0
        planes = int((nz - 2) * (per / 10.0) / max(t_full, 1e-6))
        planes = max(min(t, nz - 2), min(nz - 2, planes))
        best = 0.0
        for _ in range(3):
            cells = 0
            t0 = time.perf_counter()
            for _ in range(3):
                cells += o.step_sample(1, 1 + planes, t)
            best = max(best, cells / (time.perf_counter() - t0) / 1e6)
        sweep.append({"threads": t, "mlups": round(best, 2), "planes": planes})
    o.close()
    top = max(sweep, key=lambda e: e["mlups"])
    return {"value": top["mlups"], "unit": "MLUPS", "cores": top["threads"], "kind": "port",
            "physical_cores": physical_cores(), "hardware_threads": hc,
            "single_thread": sweep[0]["mlups"], "sweep": sweep,
            "sample": f"best of 3 x 3 steps per thread count, each step on interior z-planes "
                      f"[1, 1+planes) of the {nx}x{ny}x{nz} workload (oracle: float64 "
                      f"arithmetic, float32 storage, z-slabs as js/pool.js), {cpu_model()}"}


# ---------------------------------------------------------------------------- arms
def workload_config(wl, world: int) -> dict:
    """The `config` object both arms print: what the workload is, not how an
    arm computes it."""
    n = wl["nx"] * wl["ny"] * wl["nz"]
    return {"workload": wl["name"], "lattice": f"{wl['nx']}x{wl['ny']}x{wl['nz']}", "cells": n,
            "storage": "f32", "tau": wl["tau"], "u0": wl["u0"], "les_cs": wl["csm"],
            "trt_lambda": wl["lam"], "side_bc": wl["side_bc"],
            "l2": f"inputs larger than L2: two {19 * n * 4 / 1e6:.1f} MB population buffers "
                  f"per lattice",
            "parallelism": f"replicas{world}" if world > 1 else "single GPU"}


def timed_form(wl, storage, math_mode, K, W, dist, rounding=None) -> float:
    """Max over ranks of the event time (ms) of K steps of one storage / arithmetic form."""
    sim = setup_gpu(wl, storage, math_mode)
    if rounding:
        sim.set_params(f16_rounding=rounding)
    sim.step_forces(W)
    ms, _ = timed_steps(sim, K, dist)
    sim.close()
    return dist.max(ms)


def run_wt(args) -> None:
    import torch
    dist = Dist()
    dist.init()
    wl = WORKLOADS[args.workload]
    n = wl["nx"] * wl["ny"] * wl["nz"]
    K, W = args.steps, args.warmup
    peak, peak_kind = measured_peaks()

    sim = setup_gpu(wl, "f32", "fast")
    sim.step_forces(W)
    clocks = ClockSampler(torch.cuda.current_device()).start() if dist.rank == 0 else None
    ms, launches = timed_steps(sim, K, dist)
    clk = clocks.stop() if clocks else None
    ms_max = dist.max(ms)
    value = whole_job_mlups(dist.world, n, K, ms_max)

    # public batched path (host buffers, one synchronisation per call), at
    # least 16 steps whatever K is
    sim.step_forces(W)
    ke = max(16, max(W, K // 4) // 16 * 16)
    e2e_ms = dist.max(e2e_steps(sim, ke, dist, batch=16))
    e2e1_ms = dist.max(e2e_steps(sim, ke, dist, batch=1))
    if not (e2e_ms > 0 and e2e1_ms > 0):
        raise RuntimeError(f"end-to-end timing of {ke} steps gave {e2e_ms} / {e2e1_ms} ms")
    from windtunnel_b200._lib import wt_params
    import ctypes
    h2d = ctypes.sizeof(wt_params)
    e2e_val = whole_job_mlups(dist.world, n, ke, e2e_ms)
    e2e1_val = whole_job_mlups(dist.world, n, ke, e2e1_ms)
    sim.close()

    # half-deviation storage (nearest and stochastic rounding) and the
    # reference's own arithmetic (float64 collision in js/lbm.js's operation
    # order, float32 storage) on the same workload
    ms16 = timed_form(wl, "f16dev", "fast", K, W, dist)
    ms16s = timed_form(wl, "f16dev", "fast", K, W, dist, rounding="stochastic")
    msx = timed_form(wl, "f32", "exact", K, W, dist)
    v16 = whole_job_mlups(dist.world, n, K, ms16)
    v16s = whole_job_mlups(dist.world, n, K, ms16s)
    vx = whole_job_mlups(dist.world, n, K, msx)

    def achieved(form, t_ms):
        return BYTES_PER_CELL[form] * n * K / (t_ms * 1e-3) / 1e9

    a32, a16 = achieved("f32", ms), achieved("f16dev", ms16)
    shape = f"{wl['nx']}x{wl['ny']}x{wl['nz']}"
    traffic = profiled_traffic(f"k_step_pair_f32_{shape}")
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": dist.world,
        "steps": K, "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(wl, dist.world),
        "kernel": "pair (two cells per thread, one aligned load and store of the pair per "
                  "direction, packed float32x2 collision; WT_KERNEL_AUTO), float32 collision "
                  "(WT_MATH_FAST)",
        "roofline": {"bound": "hbm", "achieved": round(a32, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(a32 / peak, 4), "traffic": traffic,
                     "peak_source": peak_kind,
                     "bytes_per_cell": BYTES_PER_CELL["f32"],
                     "note": "achieved = 152 B x cells x steps / event time of the K-step call",
                     "fp16dev_achieved": round(a16, 1),
                     "fp16dev_frac": round(a16 / peak, 4),
                     "fp16dev_bytes_per_cell": BYTES_PER_CELL["f16dev"],
                     "fp16dev_traffic": profiled_traffic(
                         f"k_step_pair_f16_{shape}")},
        "e2e": {"value": round(e2e_val, 1), "unit": "MLUPS",
                "h2d_bytes_per_step": h2d / 16, "d2h_bytes_per_step": 3 * 8 + 4 / 16,
                "steps": ke,
                "path": "Pool.step(16) per call (js/pool.js:97-125): wt_set_params + "
                        "wt_step(16) + the 16-step force series to host",
                "per_step_call": {"value": round(e2e1_val, 1), "unit": "MLUPS",
                                  "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 3 * 8 + 4,
                                  "path": "LBM.step() per step: wt_set_params + wt_step(1) + "
                                          "force to host"}},
        "gpu_launches": launches,
        "fp16dev_value": round(v16, 1),
        "fp16dev_over_fp32": round(v16 / value, 3),
        "fp16dev_roofline_frac": round(a16 / peak, 4),
        "fp16dev_stochastic_value": round(v16s, 1),
        "fp16dev_stochastic_over_fp32": round(v16s / value, 3),
        "exact_f32_value": round(vx, 1),
        "fp16dev": {"value": round(v16, 1), "unit": "MLUPS", "ms_per_step": ms16 / K,
                    "rounding": "nearest", "over_fp32": round(v16 / value, 3),
                    "roofline_frac": round(a16 / peak, 4)},
        "fp16dev_stochastic": {"value": round(v16s, 1), "unit": "MLUPS",
                               "ms_per_step": ms16s / K, "rounding": "stochastic",
                               "over_fp32": round(v16s / value, 3),
                               "roofline_frac": round(achieved("f16dev", ms16s) / peak, 4)},
        "exact_f32": {"value": round(vx, 1), "unit": "MLUPS", "ms_per_step": msx / K,
                      "arithmetic": "float64 collision in js/lbm.js's operation order, no FMA "
                                    "contraction, float32 storage (WT_MATH_EXACT): bit-identical "
                                    "to the reference; the like-for-like arm against the CPU "
                                    "port",
                      "roofline_frac": round(achieved("f32", msx) / peak, 4)},
        "clocks": clk,
    }
    if args.accuracy and dist.rank == 0:
        line["accuracy"] = accuracy_study(wl, replicas=args.replicas)
        line["accuracy_steady"] = steady_accuracy(WORKLOADS["sphere128"])
    if args.adjoint and dist.rank == 0:
        line["adjoint"] = adjoint_study(ADJOINT_WORKLOADS["design128"])
        if args.adjoint_scale:
            line["adjoint_scale"] = adjoint_study(ADJOINT_WORKLOADS["design384"])
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl)
    dist.barrier()
    dist.close()
    if dist.rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args) -> None:
    """The reference's CPU path (the oracle port) on this host's cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]
    K, W = args.steps, args.warmup
    threads = host_threads()
    o = setup_oracle(wl)
    nx, ny, nz = wl["nx"], wl["ny"], wl["nz"]
    # size each timed step as a z-slab sample so the whole run stays within the budget
    t0 = time.perf_counter()
    o.step_sample(1, nz - 1, threads)
    t_full = time.perf_counter() - t0
    budget = args.reference_budget
    planes = nz - 2
    if (K + W) * t_full > budget:
        planes = max(threads, int((nz - 2) * budget / ((K + W) * t_full)))
        planes = min(planes, nz - 2)
    z0, z1 = 1, 1 + planes
    for _ in range(W):
        o.step_sample(z0, z1, threads)
    cells = 0
    t0 = time.perf_counter()
    for _ in range(K):
        cells += o.step_sample(z0, z1, threads)
    dt = time.perf_counter() - t0
    value = cells / dt / 1e6
    sample = (f"each step: interior z-planes [{z0},{z1}) of the {nx}x{ny}x{nz} lattice "
              f"({nx * ny * planes} cells, stepSlab + boundaries), {threads} threads, "
              f"{cpu_model()}")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": "MLUPS",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": K, "warmup": W,
        "ms_per_step": dt * 1e3 / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(wl, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": round(value, 2), "unit": "MLUPS", "cores": threads,
                         "kind": "port", "sample": sample, "physical_cores": physical_cores(),
                         "hardware_threads": host_threads()},
        "e2e": {"value": round(value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference is browser JavaScript (js/lbm.js); no JS engine exists on this "
                "host, so its arithmetic is timed through the C restatement in oracle/"}),
        flush=True)


def run_study(args) -> None:
    """`--study accuracy`: the accuracy ensemble on --workload with --replicas
    seeds per form; `--study accuracy-long`: one --long-steps window per form
    (--forms); `--study adjoint-horizon`: the half-vs-float32 gradient
    agreement of the 384x160x160 differentiation workload against horizon."""
    import torch
    torch.cuda.set_device(0)
    if args.study == "accuracy":
        res = accuracy_study(WORKLOADS[args.workload], replicas=args.replicas)
    elif args.study == "accuracy-long":
        res = long_window_accuracy(WORKLOADS[args.workload], args.long_steps,
                                   forms=args.forms.split(",") if args.forms else None,
                                   noise_seed=args.seed)
    else:
        res = adjoint_horizon_study(ADJOINT_WORKLOADS["design384"])
    print(json.dumps(res), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["wt", "reference"], default="wt")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="channel256")
    ap.add_argument("--no-accuracy", dest="accuracy", action="store_false")
    ap.add_argument("--replicas", type=int, default=4,
                    help="seeded replicas per storage form in the accuracy ensemble")
    ap.add_argument("--study", choices=["accuracy", "accuracy-long", "adjoint-horizon"],
                    help="run one study alone and print its JSON (no timing line)")
    ap.add_argument("--long-steps", type=int, default=3000000,
                    help="averaged steps per form of --study accuracy-long")
    ap.add_argument("--seed", type=int, default=None,
                    help="initial velocity-noise seed of --study accuracy-long (the body "
                         "stays the workload's; default: the workload's seed)")
    ap.add_argument("--forms", default=None,
                    help="comma-separated storage forms of --study accuracy-long "
                         "(f64,f32,f16dev,f16dev_stochastic; default all)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false")
    ap.add_argument("--no-adjoint-scale", dest="adjoint_scale", action="store_false")
    ap.add_argument("--reference-budget", type=float, default=90.0,
                    help="seconds of timed CPU work for --impl reference")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.study:
        run_study(args)
    else:
        run_wt(args)


if __name__ == "__main__":
    main()
