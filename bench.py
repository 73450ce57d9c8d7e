"""Benchmark of the ANI-2x energy+force MD step on B200.

The JSON line also carries: per-kernel rooflines (``kernels``), the FP32
form on the same workload, accuracy against the FP64 oracle, the end-to-end
public-API call with host buffers (``e2e``), the CPU oracle on the host
cores (``cpu_baseline``), a Poisson request stream through the serving loop
(``serving``), the training-loss gradient of a 256-molecule batch
(``training_256mol``), the 98,304-atom 8-model ensemble against its FP32 form
(``ensemble_98k``) and, with ``--nve-drift-steps``, the NVE energy drift.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload water12k|water98k] [--precision bf16x3|bf16x2|bf16|fp32]

A step is one MD step of the workload: BAOAB integrator (float64) ->
neighbour list (skin filter every step, cell-list rebuild when an atom moved
more than half the skin) -> AEV -> species MLPs -> energy -> force adjoint,
replayed from a CUDA graph.  Inputs live in HBM; every timed step is
bracketed by CUDA events on the launching stream and preceded by an L2 flush
(a 512 MB write) outside the events.  Multi-GPU runs (torchrun) are
independent replicas (weak scaling); the time is the max over ranks.
Prints one JSON line on rank 0.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "E+F atom-steps/s (1 B200, BF16 vs FP32 form) at stated force RMSE; p50/p99 latency"
HARTREE_TO_KCALMOL = 627.5096080305927
MLP_FLOP_PER_ATOM = 2 * (1008 * 256 + 256 * 192 + 192 * 160 + 160 * 1) * 2  # fwd + input grad

WORKLOADS = {
    "water12k": dict(n_side=16, n_models=1, thermostat="LGV", desc=(
        "water box 12,288 atoms (4096 H2O, 49.7 A cube), Langevin 300 K gamma 1/ps, dt 0.5 fs, "
        "skin 1.0 A, list rebuilt every nblist_stride steps (FeNNol's rule gives 40 at 0.5 fs) with "
        "every step checked on the device (an atom moved > skin/2 since the rebuild: roll back and "
        "shorten the stride; the value used is in neighbour_list), "
        "ANI-2x 7-species random-init model "
        "(MD: last layer x0.02)")),
    "water98k": dict(n_side=32, n_models=8, thermostat="NVE", desc=(
        "water box 98,304 atoms (32768 H2O, 99.4 A cube), NVE dt 0.5 fs, skin 1.0 A (checked stride), "
        "8-model ANI-2x ensemble (random-init, MD: last layer x0.02)")),
}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx = float(f[2].split()[0])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], d["bf16_tflops"], d.get("bf16_tflops_sustained"), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, 1400.0, "fallback"


def make_engine(workload, precision, device, seed=0, bf16_weights=True, output_scale=None):
    from fennol_b200.md import MDEngine
    from fennol_b200.potential import ANIPotential
    from fennol_b200.systems import water_box

    from fennol_b200.params import MD_OUTPUT_SCALE

    w = WORKLOADS[workload]
    box = water_box(w["n_side"], seed=seed)
    pot = ANIPotential(precision=precision, device=device, seed=0, n_models=w["n_models"],
                       output_scale=MD_OUTPUT_SCALE if output_scale is None else output_scale,
                       bf16_weights=bf16_weights)
    eng = MDEngine(pot, box.coordinates, box.species, box.cell, dt_fs=0.5, thermostat=w["thermostat"],
                   temperature=300.0, gamma_ps=1.0, skin=1.0, trigger="stride", seed=seed)
    return box, pot, eng


def time_steps(eng, steps, warmup, flush):
    """Per-step device times (ms) of graph-replayed MD steps, L2 flushed
    between steps, and the number of list rebuilds inside the timed steps."""
    import torch

    eng.run(warmup)  # also regrows lists (and shortens the stride) if needed
    if eng.trigger == "stride":
        # start the timed steps with a rebuild: a window shorter than the
        # stride then counts a full rebuild (pessimistic, never optimistic)
        pad = (-eng.step_count) % eng.nblist_stride
        if pad:
            eng.run(pad)
    graphs = [eng.graph_for_step(k) for k in range(steps)]
    rebuilds0 = eng.rebuild_count()
    stream = torch.cuda.current_stream()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    eng.snapshot()
    torch.cuda.synchronize()
    for k in range(steps):
        flush.zero_()
        starts[k].record(stream)
        graphs[k].replay()
        ends[k].record(stream)
    torch.cuda.synchronize()
    if eng._regrow():  # an overflow during timing: lists regrown, time again
        return time_steps(eng, steps, 0, flush)
    if eng.displaced_beyond_skin():  # a stale list during timing: shorter stride, time again
        eng.shorten_stride()
        return time_steps(eng, steps, 0, flush)
    eng.step_count += steps
    return np.array([s.elapsed_time(e) for s, e in zip(starts, ends)]), eng.rebuild_count() - rebuilds0


def time_mlp(pot, eng, reps):
    """Average duration (ms) of the species-MLP launch on the current state."""
    import torch
    from fennol_b200._lib import call
    from fennol_b200.potential import C_ptr, _ptr

    lay, ws = eng.layout, eng.ws
    st = torch.cuda.current_stream().cuda_stream
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def launch():
        call("fennol_mlp_energy_grad", pot.precision, lay.rows, lay.ntiles, lay.t_tile_species.data_ptr(),
             lay.t_tile_row.data_ptr(), C_ptr(pot.mlp.struct), ws.x.data_ptr(), _ptr(ws.x_lo),
             ws.e_rows.data_ptr(), ws.dx.data_ptr(), ws.mlp_ws.data_ptr(), ws.mlp_ws.numel(), st)

    for _ in range(3):
        launch()
    torch.cuda.synchronize()
    ev0.record()
    for _ in range(reps):
        launch()
    ev1.record()
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / reps


def time_launch(fn, reps):
    """Average device time (ms) of ``fn``'s launches, after 3 warm-up calls."""
    import torch

    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(reps):
        fn()
    ev1.record()
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / reps


def kernel_times(pot, eng, reps=20):
    """Device time per launch (ms) of the three large kernels of a step, on
    the current MD state: AEV forward, species MLP, AEV adjoint."""
    import torch
    from fennol_b200._lib import call
    from fennol_b200.potential import C_ptr, _ptr

    lay, ws, g = eng.layout, eng.ws, eng.graph_buf
    st = torch.cuda.current_stream().cuda_stream
    lp = C_ptr(pot.params)

    # the staged pair, as the MD step launches it
    def aev_fwd():
        call("fennol_aev_forward_staged", ws.xyzs.data_ptr(), lay.n, lay.t_atom_sys.data_ptr(),
             lay.t_cell.data_ptr(), g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(), g.cap_r, lp,
             lay.t_atom_row.data_ptr(), ws.aev_kind, ws.x.data_ptr(), _ptr(ws.x_lo), ws.x.shape[1],
             g.aev_stage.data_ptr(), g.aev_stage.numel(), ws.status.data_ptr(), st)

    def aev_bwd():
        call("fennol_aev_backward_staged", ws.xyzs.data_ptr(), lay.n, lay.t_atom_sys.data_ptr(),
             lay.t_cell.data_ptr(), g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(), g.cap_r, lp,
             lay.t_atom_row.data_ptr(), ws.dx.data_ptr(), ws.dx.shape[1], ws.forces4.data_ptr(),
             g.aev_stage.data_ptr(), ws.status.data_ptr(), st)

    out = {"aev_forward": time_launch(aev_fwd, reps), "mlp": time_mlp(pot, eng, reps),
           "aev_backward": time_launch(aev_bwd, reps)}
    ws.forces4.zero_()
    eng._initial_forces_from_current()
    mean_nbr = float(g.rad_n[:lay.n].float().mean())
    # angular neighbours (within the angular cutoff) of the current positions, periodic cube
    from scipy.spatial import cKDTree
    box_len = float(np.asarray(eng.cell).reshape(-1, 3, 3)[0, 0, 0])
    xyz = np.mod(eng.x.cpu().numpy(), box_len)
    tree = cKDTree(xyz, boxsize=box_len)
    mean_ang = float(np.mean(tree.query_ball_point(xyz, r=pot.aev_cfg.angular_cutoff, return_length=True)) - 1.0)
    return out, mean_nbr, mean_ang


def profile_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of ``kernel`` on ``workload`` recorded by an ncu
    capture in profiles/ (a line ``traffic_bytes_per_launch <kernel> <workload> <bytes>``)."""
    d = os.path.join(ROOT, "profiles")
    try:
        names = sorted(os.listdir(d))
    except OSError:
        return None
    for name in names:
        try:
            with open(os.path.join(d, name)) as f:
                for line in f:
                    parts = line.strip().strip("`").split()
                    if len(parts) == 4 and parts[0] == "traffic_bytes_per_launch" and \
                            parts[1] == kernel and parts[2] == workload:
                        return float(parts[3])
        except OSError:
            continue
    return None


def accuracy(pot, box):
    """Single-point error of this precision vs the FP64 oracle."""
    from oracle import ani_ref

    e, f = pot.energy_and_forces(box.coordinates, box.species, [box.natoms], box.cell[None])
    ref = ani_ref.energy_and_forces(box.coordinates, box.species, [box.natoms], pot.weights,
                                    pot.aev_cfg, pot.mlp_cfg, cells=box.cell[None])
    de = abs(float(e[0]) - ref["energy"][0]) * HARTREE_TO_KCALMOL / box.natoms
    rmse = float(np.sqrt(np.mean((f.cpu().numpy() - ref["forces"]) ** 2)) * HARTREE_TO_KCALMOL)
    return {"force_rmse_kcalmol_A": rmse, "energy_err_kcalmol_atom": de,
            "force_rmse_tol": 0.05, "energy_tol": 1e-4}


def e2e(pot, box, steps, warmup):
    """Public API call per step with pinned host coordinates in and host
    forces/energy out (single point: the neighbour list is rebuilt each call)."""
    import torch

    x_host = torch.tensor(box.coordinates, dtype=torch.float32).pin_memory()
    f_host = torch.empty((box.natoms, 3), dtype=torch.float32).pin_memory()
    e_host = torch.empty(1, dtype=torch.float64).pin_memory()
    dev = pot.device
    x_dev = torch.empty_like(x_host, device=dev)
    for _ in range(warmup):
        x_dev.copy_(x_host, non_blocking=True)
        e, f = pot.energy_and_forces(x_dev, box.species, [box.natoms], box.cell[None])
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        x_dev.copy_(x_host, non_blocking=True)
        e, f = pot.energy_and_forces(x_dev, box.species, [box.natoms], box.cell[None])
        f_host.copy_(f, non_blocking=True)
        e_host.copy_(e[:1], non_blocking=True)
        torch.cuda.current_stream().synchronize()
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    return {"value": box.natoms / (ms * 1e-3), "unit": "atom-steps/s", "ms_per_step": ms,
            "h2d_bytes_per_step": int(x_host.numel() * 4),
            "d2h_bytes_per_step": int(f_host.numel() * 4 + 8),
            "api": "ANIPotential.energy_and_forces (single point, list rebuilt every call)"}


def cpu_baseline(box, n_models, samples=1):
    """The CPU oracle (float32 torch restatement of the reference formulas,
    numpy float32 pair search) timed on this host's cores."""
    import torch
    from fennol_b200.params import AEVConfig, MLPConfig, init_weights
    from oracle import ani_ref

    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    cfg, mcfg = AEVConfig(), MLPConfig()
    W = init_weights(cfg, mcfg, seed=0, n_models=n_models)
    ts = []
    for _ in range(samples):
        t = time.perf_counter()
        ani_ref.energy_and_forces(box.coordinates, box.species, [box.natoms], W, cfg, mcfg,
                                  cells=box.cell[None], dtype=torch.float32)
        ts.append(time.perf_counter() - t)
    sec = float(np.median(ts))
    return {"value": box.natoms / sec, "unit": "atom-steps/s", "cores": cores, "kind": "port",
            "sample": (f"{samples} single-point E+F of the {box.natoms}-atom box "
                       f"(pair search + AEV + {n_models}-model MLP + autodiff forces), "
                       f"float32, {sec:.2f} s each")}


def ensemble_98k(device, steps, warmup, flush):
    """The 98,304-atom water box with the 8-model ensemble: BF16 tensor-core
    form against the float32 CUDA-core form, same MD step, same timing rules."""
    import torch

    w = WORKLOADS["water98k"]
    hbm, tf_burst, tf_sust, src = measured_peaks()
    out = {"workload": w["desc"], "atoms": 0, "models": w["n_models"]}
    for precision in ("bf16x2", "fp32"):
        box, pot, eng = make_engine("water98k", precision, device)
        ms, _ = time_steps(eng, steps, warmup, flush)
        mlp_ms = time_mlp(pot, eng, 5)
        flops = MLP_FLOP_PER_ATOM * box.natoms * w["n_models"]
        out["atoms"] = box.natoms
        out[precision] = {"value": box.natoms / (float(ms.mean()) * 1e-3), "unit": "atom-steps/s",
                          "ms_per_step": float(ms.mean()), "mlp_ms_per_launch": mlp_ms,
                          "mlp_tflops": flops / (mlp_ms * 1e-3) / 1e12,
                          "mlp_frac_of_peak": flops / (mlp_ms * 1e-3) / 1e12 / tf_sust,
                          "peak": f"{src} bf16 sustained {tf_sust} TFLOP/s"}
        del eng, pot
        torch.cuda.empty_cache()
    out["speedup_vs_fp32_form"] = out["bf16x2"]["value"] / out["fp32"]["value"]
    return out


DRIFT_OUTPUT_SCALE = 0.002


def nve_drift(device, steps, workload="water98k", every=100):
    """Total-energy record of an NVE run of the workload (BF16 MLP form,
    float64 integrator): linear drift and largest excursion per atom.

    The random-weight network has no repulsive core: over thousands of steps
    its wells gather atoms until one centre has more angular neighbours than
    the kernels hold.  The drift run therefore scales the last layer by
    ``DRIFT_OUTPUT_SCALE`` (atomic energies well below kT), and stops early,
    saying so, if a list limit is hit."""
    box, pot, eng = make_engine(workload, "bf16x2", device, output_scale=DRIFT_OUTPUT_SCALE)
    n = box.natoms
    t_ps, etot = [], []
    done = 0
    stopped = None
    t0 = time.perf_counter()
    while True:
        etot.append(eng.potential_energy() + eng.kinetic_energy())
        t_ps.append(done * eng.dt)
        if done >= steps:
            break
        k = min(every, steps - done)
        try:
            eng.run(k, graph_steps=1)
        except RuntimeError as err:
            stopped = f"stopped after {done} steps: {err}"
            break
        done += k
    wall = time.perf_counter() - t0
    e = np.array(etot) / n
    slope = float(np.polyfit(np.array(t_ps), e, 1)[0]) if len(e) > 2 else 0.0
    return {"workload": WORKLOADS[workload]["desc"] + f"; last layer x{DRIFT_OUTPUT_SCALE} for this run",
            "steps": done, "stopped": stopped, "dt_fs": eng.dt * 1000.0,
            "samples": len(e), "drift_kcalmol_atom_per_ns": slope * 1000.0,
            "max_abs_dev_kcalmol_atom": float(np.abs(e - e[0]).max()),
            "e0_kcalmol_atom": float(e[0]), "temperature_end_K": eng.temperature(),
            "rebuilds": eng.rebuild_count(), "wall_s": wall}


def training_256(device, reps=5):
    """Energy + force loss gradient (the training step's gradient) for a batch
    of 256 organic molecules of 10-40 atoms, targets from a teacher network:
    device time per gradient, through the public LossGradient call."""
    import torch
    from fennol_b200.params import AEVConfig, MLPConfig, init_weights
    from fennol_b200.potential import ANIPotential
    from fennol_b200.systems import molecule_batch
    from fennol_b200.training import LossGradient

    mols = molecule_batch(256, seed=4)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    nat = np.array([m.natoms for m in mols])
    cfg, mcfg = AEVConfig(), MLPConfig()
    teacher = ANIPotential(precision="fp32", device=device, weights=init_weights(cfg, mcfg, seed=77))
    e_ref, f_ref = teacher.energy_and_forces(xyz, sp, nat)
    e_ref, f_ref = e_ref.cpu().numpy(), f_ref.cpu().numpy()
    pot = ANIPotential(precision="fp32", device=device, weights=init_weights(cfg, mcfg, seed=5, bias_std=0.05))
    lg = LossGradient(pot, w_e=1.0, w_f=10.0)
    for _ in range(3):
        terms, _ = lg(xyz, sp, nat, e_ref, f_ref)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        terms, _ = lg(xyz, sp, nat, e_ref, f_ref)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) / reps * 1e3
    return {"batch": "256 molecules, 10-40 atoms (random-walk chains, H50/C30/N7/O8/S2/F2/Cl1)",
            "atoms": int(nat.sum()), "ms_per_gradient": ms, "atoms_per_s": float(nat.sum()) / (ms * 1e-3),
            "loss": terms.loss, "loss_terms": "mean (E - E_teacher)^2 + 10 mean (F - F_teacher)^2",
            "path": "CUDA E/F + AEV tangent kernel + float32 network sweep (cuBLAS GEMMs), host time per call"}


def serving_run(device, n_requests=1000, rate_hz=2000.0, seed=0):
    """Poisson stream through the continuous-batching loop (real time):
    throughput of the energy/force work done and p50/p99 request latency."""
    from fennol_b200.params import MD_OUTPUT_SCALE
    from fennol_b200.potential import ANIPotential
    from fennol_b200.serving import (ServingEngine, atom_steps, latency_percentiles,
                                     serve_requests_from_stream)
    from fennol_b200.systems import request_stream

    pot = ANIPotential(precision="bf16x2", device=device, seed=0, output_scale=MD_OUTPUT_SCALE,
                       bf16_weights=True)
    stream = request_stream(n_requests, rate_hz=rate_hz, seed=seed, md_steps=100, pool_size=48)
    warm = serve_requests_from_stream(request_stream(24, rate_hz=rate_hz, seed=seed + 1, md_steps=10,
                                                     pool_size=8))
    eng = ServingEngine(pot, hbm_budget_gb=120.0, segment_steps=10)
    eng.run(warm, realtime=False)
    reqs = serve_requests_from_stream(stream)
    t0 = time.perf_counter()
    res = eng.run(reqs, realtime=True)
    wall = time.perf_counter() - t0
    work = atom_steps(res, {q.rid: q for q in reqs})
    lat = latency_percentiles(res)
    n_md = sum(q.kind == "md" for q in reqs)
    return {"value": work / wall, "unit": "atom-steps/s", "wall_s": wall,
            "requests": len(reqs), "md_requests": n_md,
            "atoms_mean": float(np.mean([q.natoms for q in reqs])),
            "latency_ms": {"p50": lat["p50_ms"], "p99": lat["p99_ms"], "mean": lat["mean_ms"]},
            "stream": (f"Poisson {rate_hz:.0f} req/s, atoms log-uniform 8-5000 (chains and water "
                       "boxes, 48 pre-generated systems), 70% single-point E+F, 30% 100-step "
                       "Langevin MD continuations at dt 0.5 fs; HBM budget 120 GB"),
            "captures": eng.md.captures}


def run_reference(args):
    """Reference arm: the CPU restatement of the reference algorithm, one
    bounded MD-step sample per timed step, rank 0 only."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from fennol_b200.systems import water_box
    w = WORKLOADS[args.workload]
    box = water_box(w["n_side"], seed=0)
    steps = max(1, min(args.steps, 3))
    base = cpu_baseline(box, w["n_models"], samples=steps)
    line = {"metric": METRIC, "value": base["value"], "unit": "atom-steps/s", "n_gpus": world,
            "steps": steps, "warmup": 0, "ms_per_step": box.natoms / base["value"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": w["desc"]},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": ("the reference (JAX/Flax) is not installed in this image; its CPU path is "
                     "restated by the oracle and timed on the host cores")}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="water12k", choices=list(WORKLOADS))
    ap.add_argument("--precision", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-98k", action="store_true", help="skip the 98k-atom 8-model comparison")
    ap.add_argument("--skip-serving", action="store_true", help="skip the request-stream run")
    ap.add_argument("--skip-training", action="store_true", help="skip the training-gradient timing")
    ap.add_argument("--nve-drift-steps", type=int, default=0,
                    help="also record NVE energy drift of the 98k-atom ensemble over this many steps")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device(f"cuda:{local}"),
                                timeout=__import__("datetime").timedelta(seconds=300))
    device = torch.device(f"cuda:{local}")
    torch.cuda.set_device(device)

    from fennol_b200 import _lib
    precision = args.precision
    if precision is None:
        precision = "bf16x2" if os.environ.get("FENNOL_BENCH_FP32_ONLY") is None else "fp32"
    w = WORKLOADS[args.workload]
    try:
        box, pot, eng = make_engine(args.workload, precision, device, seed=rank)
    except _lib.FennolError as err:
        if err.code != _lib.ERR_UNSUPPORTED:
            raise
        precision = "fp32"
        box, pot, eng = make_engine(args.workload, precision, device, seed=rank)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ms, rebuilds = time_steps(eng, args.steps, args.warmup, flush)
    total_ms = float(ms.sum())
    if world > 1:
        from fennol_b200.replicas import max_over_ranks
        total_ms = max_over_ranks(total_ms, device)
        dist.barrier()
    value = world * box.natoms * args.steps / (total_ms * 1e-3)

    res = {"metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "bf16" if precision.startswith("bf16") else "f32", "data": "synthetic",
           "config": {"workload": w["desc"], "atoms_per_gpu": box.natoms, "precision": precision,
                      "weights": "BF16-representable (seeded N(0, 1/fan_in) rounded to BF16)",
                      "mlp_precision": {"fp32": "float32 CUDA cores",
                                        "bf16": "tcgen05 BF16, FP32 accumulate",
                                        "bf16x2": "tcgen05 BF16 hi+lo activations (2 MMAs)",
                                        "bf16x3": "tcgen05 BF16 hi+lo activations and weights (3 MMAs)"}[precision],
                      "aev": "float32", "integrator": "float64",
                      "l2": "flushed between timed steps (512 MB write outside the events)",
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
           "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
           "clocks": clocks.summary(),
           "gpu_launches": eng.launches_per_step() * args.steps + eng.rebuild_launches() * rebuilds,
           "rebuilds_in_run": rebuilds,
           "neighbour_list": {"trigger": eng.trigger, "nblist_stride": eng.nblist_stride,
                              "stride_shortenings": eng.stride_reductions}}
    # end-to-end public-API calls on every rank; the job rate uses the slowest rank
    e2e_res = e2e(pot, box, max(5, args.steps // 3), 3)
    if world > 1:
        from fennol_b200.replicas import max_over_ranks
        ms_e2e = max_over_ranks(e2e_res["ms_per_step"], device)
        e2e_res.update(value=world * box.natoms / (ms_e2e * 1e-3), ms_per_step=ms_e2e,
                       h2d_bytes_per_step=world * e2e_res["h2d_bytes_per_step"],
                       d2h_bytes_per_step=world * e2e_res["d2h_bytes_per_step"])
    # the comparisons below are single-GPU measurements, made at N = 1 only
    extras = world == 1
    if rank == 0:
        hbm, tf_burst, tf_sust, src = measured_peaks()
        kt, mean_nbr, mean_ang = kernel_times(pot, eng)
        mlp_ms = kt["mlp"]
        flops = MLP_FLOP_PER_ATOM * box.natoms * w["n_models"]
        mlp_tf = flops / (mlp_ms * 1e-3) / 1e12
        # the per-centre staging record the forward writes and the adjoint reads:
        # 20 B per radial edge, 28 B per angular neighbour, 4 S counters (S = 7)
        rec = 20 * mean_nbr + 28 * mean_ang + 4 * 4 * 7
        # algorithmic bytes per atom of the adjoint: its dE/dAEV row (float32),
        # its staging record, the neighbour indices of its row and its force out
        bwd_bytes = box.natoms * (1008 * 4 + rec + mean_nbr * 4 + 16)
        # forward: neighbour row and position in, AEV row out (BF16 hi + lo or
        # float32), staging record out
        fwd_bytes = box.natoms * (mean_nbr * 8 + 16 + 1008 * (2 if precision == "bf16" else 4) + rec)
        kernels = {
            "aev_backward": {"ms_per_launch": kt["aev_backward"], "bound": "hbm",
                             "algorithmic_bytes_per_launch": bwd_bytes,
                             "achieved": bwd_bytes / (kt["aev_backward"] * 1e-3) / 1e9, "unit": "GB/s",
                             "peak": hbm},
            "aev_forward": {"ms_per_launch": kt["aev_forward"], "bound": "hbm",
                            "algorithmic_bytes_per_launch": fwd_bytes,
                            "achieved": fwd_bytes / (kt["aev_forward"] * 1e-3) / 1e9, "unit": "GB/s",
                            "peak": hbm},
            "mlp": {"ms_per_launch": mlp_ms, "bound": "tensor", "algorithmic_flop_per_launch": flops,
                    "achieved": mlp_tf, "unit": "TFLOP/s", "peak": tf_burst},
        }
        for k in kernels.values():
            k["frac"] = k["achieved"] / k["peak"]
        res["kernels"] = kernels
        res["kernels"]["mean_radial_neighbors"] = mean_nbr
        res["kernels"]["mean_angular_neighbors"] = mean_ang
        top = max(("aev_backward", "aev_forward", "mlp"), key=lambda k: kernels[k]["ms_per_launch"])
        kd = kernels[top]
        names = {"aev_backward": "k_aev_backward", "aev_forward": "k_aev_forward", "mlp": "k_mlp_fused"}
        traffic = profile_traffic(names[top], args.workload)
        res["roofline"] = {"bound": kd["bound"], "kernel": names[top], "achieved": kd["achieved"],
                           "peak": kd["peak"], "unit": kd["unit"], "frac": kd["frac"],
                           "traffic": traffic,
                           "peak_source": f"{src} {'HBM copy' if kd['bound'] == 'hbm' else 'bf16 burst'}",
                           "ms_per_launch": kd["ms_per_launch"],
                           "algorithmic_per_launch": kd.get("algorithmic_bytes_per_launch",
                                                            kd.get("algorithmic_flop_per_launch"))}
        if precision != "fp32" and extras:
            _, pot32, eng32 = make_engine(args.workload, "fp32", device, seed=rank)
            ms32, _ = time_steps(eng32, max(5, args.steps // 3), 3, flush)
            v32 = box.natoms / (float(ms32.mean()) * 1e-3)
            res["fp32_form"] = {"value": v32, "ms_per_step": float(ms32.mean()),
                                "mlp_ms_per_launch": time_mlp(pot32, eng32, 10)}
            res["speedup_vs_fp32_form"] = value / world / v32
            del eng32, pot32
        if extras:
            from fennol_b200.potential import ANIPotential
            spec = ANIPotential(precision=precision, device=device, seed=0, n_models=w["n_models"],
                                bf16_weights=True)
            res["accuracy_vs_fp64_oracle"] = accuracy(spec, box)
            res["accuracy_vs_fp64_oracle"]["model"] = ("unscaled N(0, 1/fan_in) random-init weights "
                                                       "rounded to BF16 (same weights in the oracle)")
            del spec
        res["e2e"] = e2e_res
        if not args.skip_serving and extras:
            res["serving"] = serving_run(device)
        if not args.skip_training and extras:
            res["training_256mol"] = training_256(device)
        if not args.skip_98k and args.workload != "water98k" and extras:
            # last: the 98k-atom engines hold several GB that later parts would work around
            del eng, pot
            torch.cuda.empty_cache()
            res["ensemble_98k"] = ensemble_98k(device, 5, 3, flush)
        if args.nve_drift_steps > 0 and extras:
            res["nve_drift"] = nve_drift(device, args.nve_drift_steps)
        if not args.no_cpu_baseline and extras:
            res["cpu_baseline"] = cpu_baseline(box, w["n_models"])
        print(json.dumps(res), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
