#!/usr/bin/env python
"""Benchmark of the D2Q9 time step (LLALBM's perform_lbm loop body) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one lattice-Boltzmann time step of the whole lattice.  The default
workload is the 4096 x 4096 random porous channel (BGK tau 0.8, Zou-He
velocity inlet u = 0.02, Zou-He pressure outlet rho = 1, 30 % solid discs of
radius 3..12): its 2.4 GB FP64 state is far larger than L2, so every step reads
HBM and the roofline fraction is meaningful.  `value` is MLUPS of the plain
FP64 drop-in path (lattice nodes x steps / device time), with the FP32- and
FP16-shifted storage forms reported beside it.

Multi-GPU runs (torchrun, one rank per GPU) advance an independent replica of
the lattice on every GPU (no data-path collective); `value` sums all replicas
and the time is the maximum over ranks.

--impl reference times the reference's own OpenMP CPU path (LLALBM's
perform_lbm compiled from its headers, oracle/_ref/ref_runner_fast) on the
host cores, rank 0 only.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "latticeboltzmannmethod-fonnesu-grassi-guffanti_b200")
sys.path.insert(0, os.path.join(PKG, "python"))

import llb_workloads as W  # noqa: E402

METRIC = "MLUPS (D2Q9 lattice updates per second, all nodes)"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
REF_FAST = os.path.join(ROOT, "oracle", "_ref", "ref_runner_fast")


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def workload(name: str, size: int = 4096) -> dict:
    if name == "porous4096":
        return dict(name=name if size == 4096 else f"porous{size}",
                    desc=f"random porous channel {size}x{size}, 30% solid discs r 3..12, BGK tau 0.8, "
                    "Zou-He velocity inlet u=0.02, Zou-He pressure outlet rho=1",
                    types=lambda: W.porous_types(size, size), collision=0, tau=0.8, tau_even=0.8, tau_odd=0.8,
                    inlet=("const", 0.02, 0.0), outlet_bc=2, rho_out=1.0, ref_args=[
                        "--collision", "bgk", "--tau", "0.8", "--inlet", "zh", "--outlet", "zhp",
                        "--inlet-u", "const:0.02:0", "--outlet-u", "pressure"])
    if name == "cylinder1024x256":
        te = 3.0 * (0.05 * 40 / 200) + 0.5
        to = 0.25 * (1.0 / (te - 0.5)) + 0.5
        return dict(name=name, desc="cylinder vortex street 1024x256, r=20 at (200,131), TRT magic 1/4, "
                    "parabolic Zou-He inlet u_max=0.05, Zou-He pressure outlet rho=1",
                    types=lambda: W.cylinder_types(), collision=1, tau=te, tau_even=te, tau_odd=to,
                    inlet=("parabolic", 0.05, 1, 254), outlet_bc=2, rho_out=1.0, ref_args=[
                        "--collision", "trt", "--tau-even", repr(te), "--magic", "0.25", "--inlet", "zh",
                        "--outlet", "zhp", "--inlet-u", "parabolic:0.05:1:254", "--outlet-u", "pressure"])
    if name in ("cavity129", "cavity"):
        n = 129 if name == "cavity129" else size
        return dict(name=f"cavity{n}", desc=f"lid-driven cavity {n}x{n}, BGK tau 0.884, lid u=(0.1,0)",
                    types=lambda: W.cavity_types(n), collision=0, tau=0.884, tau_even=0.884, tau_odd=0.884,
                    inlet=("const", 0.1, 0.0), outlet_bc=0, rho_out=1.0, ref_args=[
                        "--collision", "bgk", "--tau", "0.884", "--inlet", "zh", "--outlet", "zh",
                        "--inlet-u", "const:0.1:0"])
    raise SystemExit(f"unknown workload {name}")


def workload_config(wl: dict, types: np.ndarray, world: int) -> dict:
    """The `config` object of a bench line, the same for both arms: the
    workload, its lattice and its active (fluid, inlet, outlet) node count."""
    R, C = types.shape
    n_active = int(np.isin(types, (W.FLUID, W.INLET, W.OUTLET)).sum())
    return {"workload": wl["name"], "description": wl["desc"], "rows": R, "cols": C, "active_nodes": n_active,
            "storage": "f64", "pattern": "AB (ping-pong)",
            "parallelism": f"replicas x{world}" if world > 1 else "one lattice",
            "l2": "resident state 2 x 9 x 8 B x nodes, far larger than L2: no flush needed"
            if R * C >= 1 << 20 else "L2-resident lattice"}


def open_table(wl: dict, nodes: dict) -> np.ndarray:
    ni, no = len(nodes["inlet"]), len(nodes["outlet"])
    tab = np.zeros((1, ni + no, 2))
    kind = wl["inlet"][0]
    if kind == "const":
        tab[0, :ni] = wl["inlet"][1:3]
    else:
        umax, i0, i1 = wl["inlet"][1:]
        tab[0, :ni, 0] = [W.parabolic_u(int(i), umax, i0, i1) for i in nodes["inlet"][:, 0]]
    if wl["outlet_bc"] == 2:
        tab[0, ni:] = (wl["rho_out"], 0.0)
    return tab


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, period_ms: int = 50):
        self.samples = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(index), "-lms", str(period_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.perf_counter(), [x.strip() for x in line.split(",")]))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0: float, t1: float) -> dict:
        inside = [s for t, s in self.samples if t0 <= t <= t1]
        window = "timed"
        if len(inside) < 3:
            inside = [s for _, s in self.samples]
            window = "run (timed region shorter than the sampling period)"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(s[1]) for s in inside if num(s[1]) is not None]
        mx = [num(s[2]) for s in inside if num(s[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for s in inside for n, v in zip(names, s[5:9]) if v.strip().lower() == "active"})
        pw = [num(s[3]) for s in inside if num(s[3]) is not None]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside), "window": window,
                "power_w_max": max(pw) if pw else None}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------
class Dist:
    """One process per GPU (torchrun environment); replicas, timing = max over
    ranks.  backend "gloo" runs the same logic on CPU tensors."""

    def __init__(self, gpus: int, backend: str = "nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist
            from datetime import timedelta

            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = f"cuda:{self.local}"
            dist.init_process_group(backend, timeout=timedelta(seconds=300))
            self.pg = dist
            self.torch = torch

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU arms
# ---------------------------------------------------------------------------
def reference_cpu(wl: dict, types: np.ndarray, warmup: int, steps: int) -> dict:
    """The reference's perform_lbm (OpenMP policies, all host threads) on the
    same lattice: oracle/_ref/ref_runner_fast fed through Lattice::reinit."""
    if not os.path.exists(REF_FAST):
        return None
    R, C = types.shape
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        raw = os.path.join(d, "types.u8")
        np.ascontiguousarray(types.T).tofile(raw)  # column-major grid
        cmd = [REF_FAST, "--types-raw", raw, str(R), str(C), "--policy", "omp", "--threads", str(threads),
               *wl["ref_args"], "--timing", "--warmup", str(warmup), "--steps", str(steps), "--out", d]
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        p = subprocess.run(cmd, capture_output=True, text=True, cwd=d, env=env, timeout=1800)
        if p.returncode != 0:
            return {"error": p.stderr[-500:]}
        line = [ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1]
        r = json.loads(line)
    mlups = R * C * steps / r["seconds"] / 1e6
    return {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": "reference",
            "sample": f"LLALBM perform_lbm, OMPPolicy (OMPBGK/TRT, OMPBounceBack, OMPZouHe + Zou-He pressure "
                      f"policy), {R}x{C} lattice, {steps} timed steps after {warmup} warm-up, "
                      f"g++ -O3 -march=x86-64-v3 -fopenmp, {threads} threads",
            "seconds": r["seconds"], "steps": steps}


def problem_wl(kind: str, collision: int, tau: float, u: float, outlet_bc: int, rows: int) -> dict:
    """Reference-runner arguments of one batched or served problem."""
    col = (["--collision", "bgk", "--tau", repr(tau)] if collision == 0 else
           ["--collision", "trt", "--tau-even", repr(tau), "--magic", "0.25"])
    if kind == "cavity":
        bc = ["--inlet", "zh", "--outlet", "zh", "--inlet-u", f"const:{u!r}:0"]
    elif kind == "cylinder":
        bc = ["--inlet", "zh", "--outlet", "zhp", "--inlet-u", f"parabolic:0.05:1:{rows - 2}", "--outlet-u",
              "pressure"]
    else:
        bc = ["--inlet", "zh", "--outlet", "zhp" if outlet_bc == 2 else "zh", "--inlet-u", f"const:{u!r}:0",
              "--outlet-u", "pressure" if outlet_bc == 2 else "const:0:0"]
    return {"ref_args": col + bc}


def reference_sample(items, warmup: int, steps: int) -> dict:
    """The reference's OpenMP path over a sample of independent problems, one
    after another (one Lattice per problem): node updates / summed time."""
    work, secs, names = 0, 0.0, []
    for wl, types in items:
        r = reference_cpu(wl, types, warmup, steps)
        if r is None or "error" in r:
            return r
        work += types.shape[0] * types.shape[1] * steps
        secs += r["seconds"]
        names.append(f"{types.shape[0]}x{types.shape[1]}")
        cores = r["cores"]
    return {"value": work / secs / 1e6, "unit": "MLUPS", "cores": cores, "kind": "reference",
            "sample": f"LLALBM perform_lbm, OMPPolicy, problems {', '.join(names)} one after another, "
                      f"{steps} timed steps each after {warmup} warm-up, {cores} threads",
            "seconds": secs, "steps": steps}


def oracle_cpu(wl: dict, types: np.ndarray, steps: int) -> dict:
    """Fallback when the reference could not be compiled: the C restatement."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import harness as H  # test infrastructure, used here only as the CPU baseline

    lists = H.classify(types)
    p = H.Params(collision=wl["collision"], tau=wl["tau"], tau_even=wl["tau_even"], tau_odd=wl["tau_odd"],
                 outlet_bc=wl["outlet_bc"], rho_out=wl["rho_out"])
    ins = "const:%r:0" % wl["inlet"][1] if wl["inlet"][0] == "const" else "parabolic:%r:%d:%d" % wl["inlet"][1:]
    table = H.open_values(lists, ins, "pressure" if wl["outlet_bc"] == 2 else "const:0:0", 1)
    t0 = time.perf_counter()
    H.run_oracle(lists, p, steps, table)
    s = time.perf_counter() - t0
    R, C = types.shape
    return {"value": R * C * steps / s / 1e6, "unit": "MLUPS", "cores": 1, "kind": "port",
            "sample": f"C restatement of the reference step, {R}x{C}, {steps} steps (incl. setup), 1 thread"}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def bytes_per_step(storage_bytes: int, n_active: int, n_nodes: int, steps_per_pass: int = 1) -> int:
    """Algorithmic HBM bytes of one step: 9 populations read and 9 written per
    active node, plus the 1-byte node mask of every node, once per pass over
    the lattice (a two-steps-per-pass kernel moves them once for two steps)."""
    return (18 * storage_bytes * n_active + n_nodes) // steps_per_pass


PAIR_CONFIGS = (3, 4, 5)  # pipeline configurations that advance two steps per pass


def make_lattice(L, wl, nodes, R, C, storage, device):
    g = L.CudaLattice(R, C, nodes["fluid"], nodes["wall"], nodes["inlet"], nodes["inlet_side"], nodes["outlet"],
                      nodes["outlet_side"], nodes["obstacle"], nodes["obstacle_dirs"], collision=wl["collision"],
                      tau=wl["tau"], tau_even=wl["tau_even"], tau_odd=wl["tau_odd"], outlet_bc=wl["outlet_bc"],
                      storage=storage, device=device)
    g.set_open_values(open_table(wl, nodes))
    return g


def time_form(L, wl, nodes, R, C, storage, device, warmup, steps, dist, pipeline=None, launch_shape=None):
    g = make_lattice(L, wl, nodes, R, C, storage, device)
    if pipeline is not None:
        g.set_pipeline(pipeline)
    if launch_shape is not None:
        g.set_launch_shape(launch_shape)
    g.init()
    g.step(warmup)
    g.synchronize()
    dist.barrier()
    g.synchronize()
    t0 = time.perf_counter()
    g.record(0)
    g.step(steps)
    g.record(1)
    g.synchronize()
    t1 = time.perf_counter()
    dist.barrier()
    ms = dist.max(g.elapsed_ms(0, 1))
    g.check_numerics()
    g.step(1, macro=True)
    rho, u = g.macro()
    return g, ms, (t0, t1), u


def drag_lift(L, wl, nodes, R, C, device, steps, every=100):
    """Drag and lift of every storage form, sampled every `every` steps with
    the compensated FP64 reduction, against the FP64 run: drag relative to
    itself, lift relative to its amplitude, over the second half of the run
    (the developed street)."""
    hist = {}
    for storage in (0, 1, 2):
        g = make_lattice(L, wl, nodes, R, C, storage, device)
        g.init()
        g.set_force_points(nodes["obstacle"], nodes["obstacle_dirs"])
        h, done = [], 1
        while done + every <= steps:
            g.step(every)
            done += every
            h.append(g.flow_forces())
        g.close()
        hist[storage] = np.array(h)
    half = len(hist[0]) // 2
    lift64, drag64 = hist[0][half:, 0], hist[0][half:, 1]
    out = {"steps": steps, "every": every, "drag_mean_f64": float(drag64.mean()),
           "lift_amplitude_f64": float(np.abs(lift64).max())}
    for storage, name in ((1, "f32s"), (2, "f16s")):
        lift, drag = hist[storage][half:, 0], hist[storage][half:, 1]
        out[name] = {"drag_mean": float(drag.mean()),
                     "drag_max_rel_err": float(np.max(np.abs(drag - drag64) / np.abs(drag64))),
                     "lift_max_err_rel_amplitude": float(np.max(np.abs(lift - lift64)) / np.abs(lift64).max())}
    return out


def shifted_accuracy(L, wl, nodes, R, C, device, steps):
    """Velocity error of the shifted storage forms against the FP64 run of the
    same lattice after `steps` steps (config 3 states 20 000): relative L2
    over the active nodes, u of both components, unrounded."""
    act = np.zeros((C, R), dtype=bool)
    for k in ("fluid", "inlet", "outlet"):
        act[nodes[k][:, 1], nodes[k][:, 0]] = True
    us = {}
    for storage in (0, 1, 2):
        g = make_lattice(L, wl, nodes, R, C, storage, device)
        g.init()
        g.step(steps - 1, macro=True)
        g.check_numerics()
        us[storage] = g.macro()[1][:, act]
        g.close()
    ref = us[0]
    norm = float(np.sqrt((ref ** 2).sum()))
    out = {"steps": steps, "lattice": wl["name"], "oracle": "the FP64 path on the GPU (bit-exact with the reference)"}
    for storage, name in ((1, "f32s"), (2, "f16s")):
        out[name] = {"u_rel_l2_vs_f64": float(np.sqrt(((us[storage] - ref) ** 2).sum())) / norm,
                     "u_max_abs_diff": float(np.abs(us[storage] - ref).max())}
    return out


def open_flow(L, device, steps, warmup):
    """The plain FP64 path on open flow: the 4096 x 4096 lid cavity (HBM-bound,
    default kernel) and config 1 (129 x 129 cavity, L2-resident and
    launch-bound: microseconds per step over 2000 graph-replayed steps)."""
    class One:  # single-process timing (no ranks)
        world = 1

        @staticmethod
        def barrier():
            pass

        @staticmethod
        def max(x):
            return x

    out = {}
    peak = (json.load(open(PEAKS_FILE)).get("hbm_gbs") if os.path.exists(PEAKS_FILE) else None) or FALLBACK_HBM_GBS
    for name, size, k in (("cavity", 4096, max(steps, 100)), ("cavity129", 129, 2000)):
        wl = workload(name, size)
        types = wl["types"]()
        nodes = L.classify(types)
        R, C = types.shape
        n_active = len(nodes["fluid"]) + len(nodes["inlet"]) + len(nodes["outlet"])
        g, ms, _, _ = time_form(L, wl, nodes, R, C, 0, device, warmup, k, One)
        per = ms / k
        spp = 2 if g.pipeline in PAIR_CONFIGS else 1
        bps = bytes_per_step(8, n_active, R * C)          # the metric's bytes of one step
        out[wl["name"]] = {"mlups": round(R * C / per / 1e3, 1), "us_per_step": round(per * 1e3, 3),
                           "steps": k, "pipeline": g.pipeline, "gb_s": round(bps / per / 1e6, 1),
                           "frac_of_measured_hbm": round(bps / per / 1e6 / peak, 4)}
        if spp == 2:
            out[wl["name"]]["note"] = ("two steps per pass: the kernel moves the bytes of one step per two steps, "
                                       "so its own DRAM traffic is half of gb_s")
        g.close()
    out["cavity129"]["note"] = "config 1: 16 641 nodes, L2-resident, launch-bound; the HBM fraction does not apply"
    return out


def reference_parity(L, wl, types, nodes, device, steps=3):
    """The plain FP64 path against the reference itself on the bench's own
    lattice: LLALBM's perform_lbm with the Serial policies
    (oracle/_ref/ref_runner, the parity build without FMA contraction) for
    `steps` steps, compared bit for bit with the CUDA path after the same
    steps (populations S_t, u and rho of every node)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_runner")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_runner was not built"}
    R, C = types.shape
    with tempfile.TemporaryDirectory() as d:
        raw = os.path.join(d, "types.u8")
        np.ascontiguousarray(types.T).tofile(raw)
        cmd = [exe, "--types-raw", raw, str(R), str(C), "--policy", "serial", *wl["ref_args"],
               "--steps", str(steps), "--out", d]
        t0 = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, text=True, cwd=d, timeout=3600)
        secs = time.perf_counter() - t0
        if p.returncode != 0:
            return {"unavailable": "reference runner failed: " + p.stderr[-200:]}
        ref_pop = np.fromfile(os.path.join(d, "populations.f64")).reshape(9, C, R)
        ref_u = np.fromfile(os.path.join(d, "u.f64")).reshape(2, C, R)
        ref_rho = np.fromfile(os.path.join(d, "rho.f64")).reshape(C, R)
    g = make_lattice(L, wl, nodes, R, C, 0, device)
    g.init()
    g.step(steps - 1, macro=True)
    pop = g.populations()
    rho, u = g.macro()
    pipeline = g.pipeline
    g.close()
    act = np.zeros((C, R), dtype=bool)
    for k in ("fluid", "inlet", "outlet"):
        act[nodes[k][:, 1], nodes[k][:, 0]] = True
    dpop = float(np.abs(pop[:, act] - ref_pop[:, act]).max())
    return {"config": wl["name"], "steps": steps, "max_abs_df": dpop,
            "max_abs_du": float(np.abs(u - ref_u).max()), "max_abs_drho": float(np.abs(rho - ref_rho).max()),
            "bit_exact": bool(np.array_equal(pop[:, act], ref_pop[:, act]) and np.array_equal(u, ref_u)
                              and np.array_equal(rho, ref_rho)),
            "active_nodes": int(act.sum()), "gpu_pipeline": pipeline,
            "reference": "LLALBM perform_lbm, SerialPolicy (BGK, BounceBack, ZouHe + Zou-He pressure policy), "
                         "g++ -O2 -ffp-contract=off", "reference_seconds": round(secs, 1)}


def run_ours(a, dist):
    import llalbm_cuda as L

    wl = workload(a.workload, a.size)
    types = wl["types"]()
    R, C = types.shape
    nodes = L.classify(types)
    n_active = len(nodes["fluid"]) + len(nodes["inlet"]) + len(nodes["outlet"])
    dev = dist.local
    sampler = ClockSampler(dev)
    forms = {}
    head = None
    for storage, name, sb in ((0, "f64", 8), (1, "f32s", 4), (2, "f16s", 2)):
        if name != "f64" and name not in a.forms.split(","):  # the FP64 path is the headline: always timed
            continue
        g, ms, (t0, t1), u = time_form(L, wl, nodes, R, C, storage, dev, a.warmup, a.steps, dist, a.pipeline,
                                       a.launch_shape)
        per = ms / a.steps
        spp = 2 if g.pipeline in PAIR_CONFIGS else 1
        bps = bytes_per_step(sb, n_active, R * C, spp)
        form = {"mlups": dist.world * R * C / per / 1e3, "ms_per_step": per, "gb_s": bps / per / 1e6,
                "bytes_per_step": bps, "pipeline": g.pipeline, "steps_per_pass": spp}
        if storage == 0:
            head = (g, ms, t0, t1)
        else:
            # the forms' velocity error is measured after the configuration's
            # full step count (shifted_accuracy), not after these few steps
            g.close()
        forms[name] = form
    g, ms, t0, t1 = head
    clocks = sampler.summary(t0, t1)

    # end to end through the C ABI with host buffers: every step copies its
    # boundary values from pinned host memory and reads back the step's
    # stability flag (the reference's per-step LLALBM_DEBUG NaN scan); the
    # read-back of step n is awaited after step n + 1 is queued.
    try:
        import torch
        pinned = torch.empty((1, g.n_open, 2), dtype=torch.float64, pin_memory=True).numpy()
    except Exception:
        pinned = np.empty((1, g.n_open, 2))
    pinned[...] = open_table(wl, nodes)
    e2e_steps = max(1, min(a.steps, 200))

    def e2e_run(n):
        for q in range(n):
            g.set_open_values(pinned, g.t)
            g.step(1)
            g.check_numerics_begin(q % 2)
            if q > 0:
                g.check_numerics_end((q - 1) % 2)
        g.check_numerics_end((n - 1) % 2)

    e2e_run(3)
    dist.barrier()
    t_e = time.perf_counter()
    e2e_run(e2e_steps)
    e_s = dist.max(time.perf_counter() - t_e)
    g.close()
    sampler.stop()
    forces = None
    if wl["name"] == "cylinder1024x256" and a.force_steps > 0:
        forces = drag_lift(L, wl, nodes, R, C, dev, a.force_steps)

    f64 = forms["f64"]
    peaks = {}
    if os.path.exists(PEAKS_FILE):
        peaks = json.load(open(PEAKS_FILE))
    peak = peaks.get("hbm_gbs") or FALLBACK_HBM_GBS
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        traffic = json.load(open(tfile)).get(f"{wl['name']}_f64_bytes_per_launch")
    line = {
        "metric": METRIC, "value": round(f64["mlups"], 1), "unit": "MLUPS", "n_gpus": dist.world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(f64["ms_per_step"], 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(wl, types, dist.world),
        "roofline": {"bound": "hbm", "achieved": round(f64["gb_s"], 1), "peak": peak, "unit": "GB/s",
                     "frac": round(f64["gb_s"] / peak, 4), "traffic": traffic,
                     "peak_source": "measured" if peaks.get("hbm_gbs") else "fallback",
                     "algorithmic_bytes_per_launch": f64["bytes_per_step"] * f64["steps_per_pass"],
                     "steps_per_launch": f64["steps_per_pass"]},
        "forms": {k: {kk: (round(vv, 6) if isinstance(vv, float) else vv) for kk, vv in v.items()}
                  for k, v in forms.items()},
        "e2e": {"value": round(dist.world * R * C * e2e_steps / e_s / 1e6, 1), "unit": "MLUPS",
                "h2d_bytes_per_step": int(pinned.nbytes), "d2h_bytes_per_step": 4, "steps": e2e_steps,
                "path": "C ABI per step: llb_set_open_values (pinned host) + llb_step + llb_check_numerics_begin; "
                        "the step's flag read back (llb_check_numerics_end) after the next step is queued"},
        "gpu_launches": a.steps,
        "clocks": clocks,
    }
    if forces:
        line["drag_lift"] = forces
    return line, wl, types


def output_writer(L, device, size=1024, every=1000, saves=4):
    """Saves of u on output steps (perform_lbm's write_lattice_file,
    Lattice.hpp:370-374) on a size x size lid cavity: steps with the macro
    output on the save steps and no files, the same run writing each file
    before stepping on (the reference's order: copy, format, write), and the
    same run through the asynchronous writer (the copy enqueued on the
    lattice's stream, files written by native threads while the next steps
    run; the final flush is inside the timed region)."""
    import shutil
    import tempfile

    wl = workload("cavity", size)
    types = wl["types"]()
    nodes = L.classify(types)
    R, C = types.shape
    out = {"lattice": f"cavity{size}", "steps_between_saves": every, "saves": saves}
    tmp = tempfile.mkdtemp(prefix="llb_out_")
    try:
        for mode in ("none", "sync", "async"):
            g = make_lattice(L, wl, nodes, R, C, 0, device)
            w = L.OutputWriter(tmp) if mode != "none" else None
            g.init()
            g.step(50)
            g.synchronize()
            t0 = time.perf_counter()
            for n in range(saves):
                g.step(every - 1)
                g.step(1, macro=True)
                if w:
                    w.save_u(g, n)
                    if mode == "sync":
                        w.flush()
            if w:
                w.flush()
            g.synchronize()
            s = time.perf_counter() - t0
            out[f"mlups_{mode}"] = round(R * C * every * saves / s / 1e6, 1)
            if w:
                st = w.stats()
                out[f"write_s_per_file_{mode}"] = round(st["write_s"] / max(st["files"], 1), 4)
                w.close()
            g.close()
        out["file_bytes"] = sum(os.path.getsize(os.path.join(tmp, f)) for f in os.listdir(tmp)) // (2 * saves)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def batch_add(b, L, prob, storage):
    """Adds one config-4 problem to a batch (or creates it alone when b is None)."""
    types = prob["make_types"]()
    n = L.classify(types)
    ni, no = len(n["inlet"]), len(n["outlet"])
    tab = np.zeros((1, ni + no, 2))
    tab[0, :ni, 0] = prob["u"]
    if prob["outlet_bc"] == 2:
        tab[0, ni:] = (1.0, 0.0)
    kw = dict(collision=1 if prob["trt"] else 0, tau=prob["tau"], tau_even=prob["tau"], tau_odd=prob["tau_odd"],
              outlet_bc=prob["outlet_bc"])
    R, C = types.shape
    args = (R, C, n["fluid"], n["wall"], n["inlet"], n["inlet_side"], n["outlet"], n["outlet_side"],
            n["obstacle"], n["obstacle_dirs"])
    active = len(n["fluid"]) + ni + no
    if b is None:
        g = L.CudaLattice(*args, storage=storage, **kw)
        g.set_open_values(tab)
        return g, active
    return b.add(*args, open_values=tab, **kw), active


def batch_accuracy(L, probs, device, steps=5000, sample=8):
    """Velocity error of the batched FP32-shifted form against the FP64 path on
    config 4's own step count: a sample of the problems (half cavities, half
    channels, spread over the list) run `steps` steps in an FP32-shifted
    batch and in an FP64 batch (bit-exact with the reference); relative L2 of
    u over the active nodes, per problem."""
    cav = [p for p in probs if p["kind"] == "cavity"]
    chan = [p for p in probs if p["kind"] != "cavity"]
    half = max(1, sample // 2)
    pick = cav[:: max(1, len(cav) // half)][:half] + chan[:: max(1, len(chan) // half)][:half]
    us = {}
    for storage in (L.STORE_F64, L.STORE_F32S):
        with L.CudaBatch(storage=storage, device=device) as b:
            slots = [batch_add(b, L, p, storage)[0] for p in pick]
            b.step(steps - 1)
            b.synchronize()
            us[storage] = [b.lattice(s).compute_macro()[1] for s in slots]
    errs = []
    for p, u64, u32 in zip(pick, us[L.STORE_F64], us[L.STORE_F32S]):
        errs.append(float(np.sqrt(((u32 - u64) ** 2).sum() / max((u64 ** 2).sum(), 1e-300))))
    return {"steps": steps, "problems": [f"{p['kind']} {p['rows']}x{p['cols']}" for p in pick],
            "u_rel_l2_vs_f64": errs, "max": max(errs), "median": float(np.median(errs))}


def run_batch(a, dist):
    """Config 4: 256 uneven problems advanced as one batch (FP32-shifted,
    autotuned launch shape) against each problem alone through the plain FP64
    path."""
    import llalbm_cuda as L

    probs = W.batch_problems()[:a.lattices]
    nodes = sum(p["rows"] * p["cols"] for p in probs)
    b = L.CudaBatch(storage=L.STORE_F32S, device=dist.local)
    active = 0
    for p in probs:
        _, act = batch_add(b, L, p, L.STORE_F32S)
        active += act
    if a.batch_layout is None:
        by, spl, tune_ms = b.tune(8)
    else:  # a fixed layout and launch shape (profiling), no tuner
        b.set_layout({"auto": 0, "compact": 1, "dense": 2}[a.batch_layout])
        by, spl, tune_ms = a.batch_block_y, a.batch_spl, 0.0
        b.set_config(by, spl)
    layout = {0: "auto", 1: "compact", 2: "dense"}[b.layout]
    b.step(a.warmup)
    b.synchronize()
    dist.barrier()
    sampler = ClockSampler(dist.local)
    t0 = time.perf_counter()
    b.record(0)
    b.step(a.steps)
    b.record(1)
    b.synchronize()
    t1 = time.perf_counter()
    ms = dist.max(b.elapsed_ms(0, 1))
    sampler.stop()
    batched = dist.world * nodes * a.steps / ms / 1e3
    b.close()
    # plain FP64 path, one problem at a time, same lattices (100 timed steps
    # after 20 warm ones per problem, so the sum is stable from box to box)
    k_plain = 100
    plain_ms = 0.0
    for p in probs:
        g, _ = batch_add(None, L, p, L.STORE_F64)
        g.init()
        g.step(20)
        g.synchronize()
        g.record(0)
        g.step(k_plain)
        g.record(1)
        plain_ms += g.elapsed_ms(0, 1)
        g.close()
    plain = nodes * k_plain / plain_ms / 1e3
    accuracy = batch_accuracy(L, probs, dist.local) if a.batch_accuracy_steps > 0 else None
    bps = 18 * 4 * active + nodes
    peak = (json.load(open(PEAKS_FILE)).get("hbm_gbs") if os.path.exists(PEAKS_FILE) else None) or FALLBACK_HBM_GBS
    per = ms / a.steps
    return {
        "metric": METRIC, "value": round(batched, 1), "unit": "MLUPS", "n_gpus": dist.world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(per, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (shifted storage)", "data": "synthetic",
        "config": {"workload": "batch256" if len(probs) == 256 else f"batch256[:{len(probs)}]", "lattices": len(probs), "nodes": nodes, "active_nodes": active,
                   "description": "256 problems, nx 64..1024 step 32, aspect 1..4, half lid cavities, half "
                                  "channels with 0-8 discs, tau U[0.55,1.5], BGK/TRT 50/50",
                   "launch": {"block_y": by, "steps_per_launch": spl, "layout": layout,
                              "autotuned_ms_per_step": round(tune_ms, 4)}},
        "roofline": {"bound": "hbm", "achieved": round(bps / per / 1e6, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(bps / per / 1e6 / peak, 4), "traffic": None},
        "plain_f64": {"mlups": round(plain, 1), "steps_per_problem": k_plain,
                      "path": "each problem alone through llb_step (FP64, the lattice's default step kernel)"},
        "batched_over_plain_f64": round(batched / plain, 3),
        "accuracy": accuracy,
        "gpu_launches": (a.steps + spl - 1) // spl, "clocks": sampler.summary(t0, t1),
    }


# ---------------------------------------------------------------------------
# served solve stream (config 5)
# ---------------------------------------------------------------------------
def serve_prepare(L, reqs):
    """Node lists and boundary values of every request, built before any clock
    starts (a client holds its lattice description before it submits)."""
    cache = {}
    out = []
    for r in reqs:
        key = (r["kind"], r["rows"], r["cols"])
        if key not in cache:
            n = L.classify(r["make_types"]())
            cache[key] = (n, len(n["fluid"]) + len(n["inlet"]) + len(n["outlet"]))
        n, active = cache[key]
        out.append(dict(req=r, lists=n, active=active, table=W.serve_open_values(r, n)))
    return out


def serve_submit(server, p, steps=None):
    r, n = p["req"], p["lists"]
    return server.submit(r["rows"], r["cols"], n["fluid"], n["wall"], n["inlet"], n["inlet_side"], n["outlet"],
                         n["outlet_side"], n["obstacle"], n["obstacle_dirs"], steps=steps or r["steps"],
                         collision=r["collision"], tau=r["tau"], tau_even=r["tau_even"], tau_odd=r["tau_odd"],
                         outlet_bc=r["outlet_bc"], open_values=p["table"])


def serve_stream(L, prepared, arrivals, storage, mode, budget, warmup, max_chunk=256):
    """Submits every request at its arrival time (a feeder thread), collects
    every result (rho and u copied to host memory); latency = done - submitted."""
    import queue as Q

    with L.CudaServer(storage=storage, mode=mode, budget_bytes=budget, max_chunk_steps=max_chunk) as s:
        small = sorted(prepared, key=lambda p: p["req"]["rows"] * p["req"]["cols"])[:max(warmup, 1)]
        for p in small:                                   # warm-up: module load, first graphs
            rid = serve_submit(s, p, steps=200)
            s.wait(rid, 600)
            s.result(rid, fields=False)
        st0 = s.stats()
        ids = Q.Queue()
        t_start = time.perf_counter() + 0.02

        def feeder():
            for q, p in enumerate(prepared):
                delay = t_start + arrivals[q] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                ids.put((q, serve_submit(s, p)))
        th = threading.Thread(target=feeder)
        th.start()
        times = [None] * len(prepared)
        peak = 0
        for _ in prepared:
            q, rid = ids.get()
            while True:
                try:
                    s.wait(rid, 0.05)
                    break
                except L.LLBError as e:
                    if e.code != -9:
                        raise
                    peak = max(peak, s.stats()["bytes_in_use"])
            rho, u, times[q] = s.result(rid)
        th.join()
        st = s.stats()
    sub = np.array([t[0] for t in times])
    adm = np.array([t[1] for t in times])
    done = np.array([t[2] for t in times])
    lat = done - sub
    span = float(done.max() - sub.min())
    work = sum(p["req"]["rows"] * p["req"]["cols"] * p["req"]["steps"] for p in prepared)
    pct = {f"p{q}": round(float(np.percentile(lat, q)), 4) for q in (50, 95, 99)}
    busy = float(np.sum(done - adm)) if mode == L.SERVE_SEQUENTIAL else None
    return {"mlups": round(work / span / 1e6, 1), "span_s": round(span, 3), "latency_s": pct,
            "busy_mlups": None if busy is None else round(work / busy / 1e6, 1),
            "latency_mean_s": round(float(lat.mean()), 4), "queue_wait_mean_s": round(float((adm - sub).mean()), 4),
            "node_updates": work, "peak_bytes_in_use": int(peak), "chunks": st["chunks"] - st0["chunks"],
            "batch_steps": st["batch_steps"] - st0["batch_steps"],
            "worker_s": {k: round(st[k] - st0[k], 3) for k in ("admit_s", "wait_s", "retire_s")},
            "t0": float(sub.min()), "t1": float(done.max())}


def run_serve(a, dist):
    """Config 5: a Poisson stream of requests served by continuous batching
    (FP32-shifted) and, as the comparison, the same stream through the plain
    FP64 path one request at a time."""
    import llalbm_cuda as L

    reqs = W.serve_requests(a.requests)
    prepared = serve_prepare(L, reqs)
    budget = 120 * 10**9
    # engine throughput: every request of the stream resident in one batch, device-timed steps
    with L.CudaBatch(storage=L.STORE_F32S, device=dist.local) as b:
        for p in prepared:
            r, n = p["req"], p["lists"]
            b.add(r["rows"], r["cols"], n["fluid"], n["wall"], n["inlet"], n["inlet_side"], n["outlet"],
                  n["outlet_side"], n["obstacle"], n["obstacle_dirs"], collision=r["collision"], tau=r["tau"],
                  tau_even=r["tau_even"], tau_odd=r["tau_odd"], outlet_bc=r["outlet_bc"], open_values=p["table"])
        b.set_layout(L.LAYOUT_AUTO)      # the server's lanes' layout and shape
        b.set_config(2, 1)
        b.step(32)
        b.synchronize()
        b.record(0)
        b.step(128)
        b.record(1)
        cap_ms = b.elapsed_ms(0, 1)
    nodes = sum(p["req"]["rows"] * p["req"]["cols"] for p in prepared)
    resident = nodes * 128 / cap_ms / 1e3
    # capacity of the server: the whole stream submitted at once (the server is
    # never idle; admission, chunking, retirement and the tail included)
    burst = serve_stream(L, prepared, np.zeros(len(prepared)), L.STORE_F32S, L.SERVE_BATCHED, budget, a.warmup,
                         a.max_chunk)
    cal = {"mlups": burst["mlups"]}
    capacity = cal["mlups"] * 1e6
    mean_work = np.mean([p["req"]["rows"] * p["req"]["cols"] * p["req"]["steps"] for p in prepared])
    rate = 0.7 * capacity / mean_work
    arrivals = W.poisson_arrivals(len(prepared), rate)
    sampler = ClockSampler(dist.local)
    batched = serve_stream(L, prepared, arrivals, L.STORE_F32S, L.SERVE_BATCHED, budget, a.warmup, a.max_chunk)
    clocks = sampler.summary(batched["t0"] - time.monotonic() + time.perf_counter(),
                             batched["t1"] - time.monotonic() + time.perf_counter())
    plain = serve_stream(L, prepared, arrivals, L.STORE_F64, L.SERVE_SEQUENTIAL, budget, a.warmup)
    sampler.stop()
    peak = (json.load(open(PEAKS_FILE)).get("hbm_gbs") if os.path.exists(PEAKS_FILE) else None) or FALLBACK_HBM_GBS
    bytes_total = sum((18 * 4 * p["active"] + p["req"]["rows"] * p["req"]["cols"]) * p["req"]["steps"]
                      for p in prepared)
    gbs = bytes_total / batched["span_s"] / 1e9
    h2d = sum(16 * (len(p["lists"]["fluid"]) + len(p["lists"]["wall"]) + len(p["lists"]["inlet"]) +
                    len(p["lists"]["outlet"]) + len(p["lists"]["obstacle"])) + p["table"].nbytes for p in prepared)
    d2h = sum(24 * p["req"]["rows"] * p["req"]["cols"] for p in prepared)
    strip = lambda d: {k: v for k, v in d.items() if k not in ("t0", "t1")}
    return {
        "metric": METRIC, "value": round(batched["mlups"], 1), "unit": "MLUPS", "n_gpus": dist.world,
        "steps": len(prepared), "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (shifted storage)", "data": "synthetic",
        "config": {"workload": "serve", "requests": len(prepared),
                   "description": "Poisson arrivals; side log-uniform 128..2048 (multiple of 16); steps uniform "
                                  "1k..20k; cavity / cylinder channel / porous channel 1:1:1; FP32-shifted; "
                                  "120 GB admission budget; arrival rate 0.7 x the measured capacity",
                   "rate_per_s": round(rate, 4), "capacity_mlups": round(cal["mlups"], 1),
                   "capacity_is": "the batched FP32-shifted server on the whole stream submitted at once: node "
                                  "updates / (last done - first submitted)",
                   "resident_batch_mlups": round(resident, 1),
                   "resident_batch_is": "all requests of the stream resident in one FP32-shifted batch, 128 "
                                        "device-timed batch steps (the engine without serving overheads)",
                   "value_is": "node updates of all requests / (last done - first submitted), wall clock through "
                               "the C ABI server with host buffers in and out",
                   "steps_field": "number of requests"},
        "serve": {"batched_f32s": strip(batched), "plain_f64_sequential": strip(plain),
                  "mlups_ratio": round(batched["mlups"] / plain["mlups"], 3),
                  "capacity_ratio": round(cal["mlups"] / plain["busy_mlups"], 3),
                  "capacity_ratio_is": "batched FP32-shifted capacity / plain FP64 throughput while busy "
                                       "(node updates / summed per-request service time)"},
        "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(gbs / peak, 4), "traffic": None,
                     "note": "algorithmic bytes of all requests over the stream's wall-clock span (offered load "
                             "0.7 of capacity)"},
        "e2e": {"value": round(batched["mlups"], 1), "unit": "MLUPS", "h2d_bytes_per_step": int(h2d / len(prepared)),
                "d2h_bytes_per_step": int(d2h / len(prepared)),
                "path": "llb_server_submit (node lists + boundary values from host memory) ... llb_server_result "
                        "(rho, u to host memory); per request"},
        "gpu_launches": batched["batch_steps"] + 4 * len(prepared), "clocks": clocks,
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="porous4096",
                    choices=("porous4096", "cylinder1024x256", "cavity129", "cavity", "batch256", "serve"))
    ap.add_argument("--pipeline", type=int, default=None,
                    help="plain path step kernel: -1 one thread per node, -2 active-sector list, 0..2 and 6 TMA "
                         "configurations, 3..5 two steps per pass (default: per lattice)")
    ap.add_argument("--launch-shape", type=int, default=None, help="columns per block of the one-thread kernel")
    ap.add_argument("--lattices", type=int, default=256,
                    help="batch256 workload: the first N of the 256 problems (smaller batches for profiling)")
    ap.add_argument("--batch-layout", choices=("auto", "compact", "dense"), default=None,
                    help="batch workload: fixed layout (with --batch-block-y / --batch-spl) instead of the autotuner")
    ap.add_argument("--batch-block-y", type=int, default=2)
    ap.add_argument("--batch-spl", type=int, default=1)
    ap.add_argument("--requests", type=int, default=96, help="requests in the served stream (workload serve)")
    ap.add_argument("--max-chunk", type=int, default=256,
                    help="served stream: steps per chunk of the batched server's lanes, at most")
    ap.add_argument("--size", type=int, default=4096, help="lattice side of the porous and cavity workloads")
    ap.add_argument("--forms", default="f64,f32s,f16s", help="storage forms to time (f64 always first)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="porous workload: skip the batched and served summaries")
    ap.add_argument("--force-steps", type=int, default=50000,
                    help="steps of the config-2 drag/lift comparison of the storage forms (0: skip)")
    ap.add_argument("--batch-accuracy-steps", type=int, default=5000,
                    help="batch workload: steps of the FP32-shifted vs FP64 error run on a sample (0: skip)")
    ap.add_argument("--accuracy-steps", type=int, default=20000,
                    help="porous workload: steps of the shifted forms' velocity-error run against FP64")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)

    if a.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        w = min(a.warmup, 5)
        if a.workload in ("batch256", "serve"):
            # a sample of the independent problems, each through its own Lattice
            if a.workload == "batch256":
                probs = W.batch_problems()[:6]
                items = [(problem_wl(p["kind"], int(p["trt"]), p["tau"], p["u"], p["outlet_bc"], p["rows"]),
                          p["make_types"]()) for p in probs]
                desc = "256 uneven problems (sample of 6)"
            else:
                reqs = W.serve_requests(a.requests)[:6]
                items = [(problem_wl(r["kind"], r["collision"], r["tau_even"], r["lid"] or 0.02, r["outlet_bc"],
                                     r["rows"]), r["make_types"]()) for r in reqs]
                desc = "served request stream (sample of 6 requests)"
            k = max(1, min(a.steps, 20))
            r = reference_sample(items, w, k)
            wl = {"name": a.workload, "desc": desc, "config": {"workload": a.workload, "description": desc}}
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_runner_fast was not built"}))
                return
        else:
            wl = workload(a.workload, a.size)
            types = wl["types"]()
            # K timed steps of the whole lattice after W warm-up steps, as the
            # GPU arm, as long as they stay within about 40 steps of the 4096^2
            # lattice (~2 minutes on 16 host threads); beyond that, fewer
            # steps, reported as such
            cap = max(2, 40 * 4096 * 4096 // (types.shape[0] * types.shape[1]))
            w = min(a.warmup, max(1, cap // 8))
            k = max(1, min(a.steps, cap - w))
            r = reference_cpu(wl, types, w, k)
            if r is None:
                r = oracle_cpu(wl, types, k)
        if "error" in r:
            print(json.dumps({"impl": "reference", "unavailable": "reference runner failed: " + r["error"][-200:]}))
            return
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": round(r["value"], 3), "unit": "MLUPS",
            "n_gpus": 0, "steps": k, "warmup": w, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": wl["config"] if "config" in wl else workload_config(wl, types, 1),
            "cpu_baseline": r, "e2e": {"value": round(r["value"], 3), "unit": "MLUPS",
                                       "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }), flush=True)
        return

    dist = Dist(a.gpus)
    if a.workload in ("batch256", "serve"):
        line = run_batch(a, dist) if a.workload == "batch256" else run_serve(a, dist)
        if dist.rank == 0:
            print(json.dumps(line), flush=True)
        dist.close()
        return
    line, wl, types = run_ours(a, dist)
    if dist.world == 1 and a.workload == "porous4096" and not a.no_extras:
        # the batched and served FP32-shifted forms beside the plain FP64 path
        import copy
        ab = copy.copy(a)
        ab.steps = min(max(a.steps, 100), 300)
        bl = run_batch(ab, dist)
        line["batched"] = {"workload": "batch256", "mlups_f32s": bl["value"], "plain_f64_mlups": bl["plain_f64"]["mlups"],
                           "ratio": bl["batched_over_plain_f64"], "roofline_frac": bl["roofline"]["frac"],
                           "steps": ab.steps, "launch": bl["config"]["launch"], "accuracy": bl["accuracy"]}
        asv = copy.copy(a)
        asv.requests = a.requests
        sl = run_serve(asv, dist)
        sv = sl["serve"]
        line["served"] = {"workload": "serve", "requests": asv.requests, "rate_per_s": sl["config"]["rate_per_s"],
                          "capacity_mlups_f32s": sl["config"]["capacity_mlups"],
                          "resident_batch_mlups_f32s": sl["config"]["resident_batch_mlups"],
                          "f32s_batched": {k: sv["batched_f32s"][k] for k in ("mlups", "latency_s", "chunks",
                                                                               "batch_steps", "worker_s")},
                          "f64_plain_sequential": {k: sv["plain_f64_sequential"][k] for k in ("mlups", "busy_mlups",
                                                                                              "latency_s")},
                          "mlups_ratio": sv["mlups_ratio"], "capacity_ratio": sv["capacity_ratio"]}
    if dist.world == 1 and a.workload == "porous4096" and not a.no_extras:
        import llalbm_cuda as L
        line["output_writer"] = output_writer(L, dist.local)
        # the shifted forms' velocity error on config 3 as stated (20 000 steps)
        nodes = L.classify(types)
        R, C = types.shape
        line["accuracy"] = shifted_accuracy(L, wl, nodes, R, C, dist.local, a.accuracy_steps)
        # config 2's drag and lift of every storage form over its 50 000 steps
        cwl = workload("cylinder1024x256")
        ctypes_ = cwl["types"]()
        line["drag_lift"] = drag_lift(L, cwl, L.classify(ctypes_), ctypes_.shape[0], ctypes_.shape[1], dist.local,
                                      a.force_steps)
        line["open_flow"] = open_flow(L, dist.local, a.steps, a.warmup)
    if dist.rank == 0:
        if dist.world == 1 and not a.no_cpu_baseline:
            cb = reference_cpu(wl, types, 1, 3 if a.workload == "porous4096" else 100)
            if cb is None or "error" in cb:
                cb = oracle_cpu(wl, types, 2 if a.workload == "porous4096" else 100)
            line["cpu_baseline"] = cb
            if a.workload == "porous4096" and not a.no_extras:
                import llalbm_cuda as L
                line["parity"] = reference_parity(L, wl, types, L.classify(types), dist.local)
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
