"""Benchmark of the ANI-2x energy+force MD step on B200.

Default workload (the configuration the metric is quoted on): the
98,304-atom water box (32,768 H2O, 99.4 A cube) with an 8-model ensemble,
NVE at dt 0.5 fs, species MLPs in the fused tcgen05 FP16 split form
(``f16x3x1``) on float32 weights (seeded N(0, 1/fan_in), not rounded), AEV in
float32, energy sum and integrator in float64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload water98k|water12k] [--precision f16x3x1|f16x3x2|bf16x2|fp32]

A step is one MD step of the workload: float64 integrator -> neighbour list
(FeNNol's rebuild stride with every step's displacement checked on the
device) -> AEV -> species MLPs -> energy -> force adjoint, replayed from a
CUDA graph.  Inputs live in HBM; every timed step is bracketed by CUDA events
on the launching stream and preceded by an L2 flush (a 512 MB write) outside
the events.  Multi-GPU runs (torchrun) are independent replicas (weak
scaling); the time is the max over ranks.  Prints one JSON line on rank 0.

Besides the headline the line carries: ``e2e`` (the FeNNol-API call
``FENNIX.energy_and_forces`` with pinned host buffers in and out), the FP32
form of the same workload, the other MLP forms, accuracy against the FP64
oracle (12,288-atom box, and its 2x2x2 tiling for the 98,304-atom size),
per-kernel rooflines, the 12,288-atom box as a secondary line, the request
stream through the serving loop, the training-loss gradient, the NVE drift
(``--nve-drift-steps``) and the CPU port on the host cores (``cpu_baseline``).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from collections import OrderedDict

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "E+F atom-steps/s (1 B200, BF16 vs FP32 form) at stated force RMSE; p50/p99 latency"
HARTREE_TO_KCALMOL = 627.5096080305927
MLP_FLOP_PER_ATOM = 2 * (1008 * 256 + 256 * 192 + 192 * 160 + 160 * 1) * 2  # fwd + input grad
DEFAULT_PRECISION = "f16x3x1"
SMS = 148

WORKLOADS = {
    "water98k": dict(n_side=32, n_models=8, thermostat="NVE", desc=(
        "water box 98,304 atoms (32768 H2O, 99.4 A cube), 8-model ANI-2x ensemble (independent seeds, "
        "seeded N(0, 1/fan_in) float32 weights; MD: last layer x0.02), NVE dt 0.5 fs, skin 1.0 A, "
        "list rebuilt every nblist_stride steps with every step's displacement checked on the device")),
    "water12k": dict(n_side=16, n_models=1, thermostat="LGV", desc=(
        "water box 12,288 atoms (4096 H2O, 49.7 A cube), one ANI-2x model (seeded N(0, 1/fan_in) "
        "float32 weights; MD: last layer x0.02), Langevin 300 K gamma 1/ps, dt 0.5 fs, skin 1.0 A, "
        "checked rebuild stride")),
}

MLP_FORMS = {"fp32": "float32 CUDA cores",
             "bf16": "tcgen05 BF16, FP32 accumulate",
             "bf16x2": "tcgen05 BF16 hi+lo activations, BF16 weights (2 MMAs per product)",
             "bf16x3": "tcgen05 BF16 hi+lo activations and weights (3 MMAs, unfused)",
             "f16x3x1": ("tcgen05 FP16 hi+lo activations and power-of-two-scaled float32 weights: "
                         "3 MMAs forward, 1 MMA input gradient, FP32 accumulate"),
             "f16x3x2": ("tcgen05 FP16 hi+lo activations and power-of-two-scaled float32 weights: "
                         "3 MMAs forward, 2 MMAs input gradient, FP32 accumulate")}


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


def md_weights(workload, output_scale=None, bf16_weights=False):
    from fennol_b200.params import MD_OUTPUT_SCALE, AEVConfig, MLPConfig, init_weights
    from fennol_b200.potential import round_weights_bf16

    w = WORKLOADS[workload]
    W = init_weights(AEVConfig(), MLPConfig(), seed=0, n_models=w["n_models"],
                     output_scale=MD_OUTPUT_SCALE if output_scale is None else output_scale)
    return round_weights_bf16(W) if bf16_weights else W


def make_engine(workload, precision, device, seed=0, bf16_weights=False, output_scale=None):
    """MD engine of a workload.  ``bf16_weights`` rounds the model to BF16
    (the BF16-model form, reported separately)."""
    from fennol_b200.md import MDEngine
    from fennol_b200.potential import ANIPotential
    from fennol_b200.systems import water_box

    w = WORKLOADS[workload]
    box = water_box(w["n_side"], seed=seed)
    pot = ANIPotential(precision=precision, device=device,
                       weights=md_weights(workload, output_scale, bf16_weights))
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

    def launch():
        call("fennol_mlp_energy_grad_active", pot.precision, lay.rows, lay.ntiles, lay.t_tile_species.data_ptr(),
             lay.t_tile_row.data_ptr(), C_ptr(pot.mlp.struct), ws.x.data_ptr(), _ptr(ws.x_lo),
             pot.active_chunks(lay.species_mask), ws.e_rows.data_ptr(), ws.dx.data_ptr(), ws.mlp_ws.data_ptr(),
             ws.mlp_ws.numel(), st)

    return time_launch(launch, reps)


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
    the current MD state: AEV forward, species MLP, AEV adjoint; and the mean
    radial and angular neighbour counts."""
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
    from scipy.spatial import cKDTree
    box_len = float(np.asarray(eng.cell).reshape(-1, 3, 3)[0, 0, 0])
    xyz = np.mod(eng.x.cpu().numpy(), box_len)
    tree = cKDTree(xyz, boxsize=box_len)
    mean_ang = float(np.mean(tree.query_ball_point(xyz, r=pot.aev_cfg.angular_cutoff, return_length=True)) - 1.0)
    return out, mean_nbr, mean_ang


def profile_value(key: str, kernel: str, workload: str):
    """A per-launch figure recorded from an ncu capture in profiles/: a line
    ``<key> <kernel> <workload> <value>`` (keys ``traffic_bytes_per_launch``,
    ``inst_per_launch``)."""
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
                    if len(parts) == 4 and parts[0] == key and parts[1] == kernel and parts[2] == workload:
                        return float(parts[3])
        except OSError:
            continue
    return None


def present_aev_columns(species, cfg) -> int:
    """Columns of the AEV that a system with these species can make non-zero:
    the radial blocks of its species and the angular blocks of its species
    pairs (the adjoint reads only those)."""
    present = sorted(set(cfg.species_index(np.asarray(species)).tolist()))
    s = len(present)
    return s * cfg.radial_dist_divisions + s * (s + 1) // 2 * cfg.angular_sublength


# products per GEMM of each tensor-core form: (forward, input gradient)
PRODUCTS = {"bf16": (1, 1), "bf16x2": (2, 2), "bf16x3": (3, 3), "f16x3x1": (3, 1), "f16x3x2": (3, 2)}


def mlp_work(pot, species, precision):
    """FLOPs per atom and model: the dense count over all 1008 AEV inputs
    (2 FLOPs per multiply-add of every layer), the count on the AEV columns that can be non-zero for
    these species, and the MMA work the fused kernel issues (padded widths,
    active 64-column input chunks, split products)."""
    cols = present_aev_columns(species, pot.aev_cfg)
    present = 2 * (cols * 256 + 256 * 192 + 192 * 160 + 160) * 2
    out = {"dense_flop": MLP_FLOP_PER_ATOM, "present_column_flop": present, "present_columns": cols}
    if precision in PRODUCTS:
        pf, pb = PRODUCTS[precision]
        mask = pot.active_chunks(int(np.bitwise_or.reduce(1 << np.unique(pot.aev_cfg.species_index(species)))))
        k1 = 64 * bin(mask & 0xFFFF).count("1")
        d1, d2, d3 = pot.mlp.dims[1:4]
        out["mma_flop"] = 2 * (pf * (k1 * d1 + d1 * d2 + d2 * d3) + pb * (d3 * d2 + d2 * d1 + d1 * k1))
        out["active_input_columns"] = k1
    return out


def rooflines(pot, eng, box, workload, precision, sm_mhz):
    """Per-kernel rooflines of the step's three large kernels.  The MLP is
    bound by the tensor pipe (algorithmic FLOPs against the sustained bf16
    GEMM peak); the AEV kernels by instruction issue (warp instructions per
    launch from an ncu capture against 148 SMs x 4 schedulers x the sampled
    SM clock), with their HBM fraction over the algorithmic bytes beside it."""
    hbm, tf_burst, tf_sust, src = measured_peaks()
    kt, mean_nbr, mean_ang = kernel_times(pot, eng)
    w = WORKLOADS[workload]
    n = box.natoms
    flops = MLP_FLOP_PER_ATOM * n * w["n_models"]
    cols = present_aev_columns(box.species, pot.aev_cfg)
    # algorithmic bytes per atom: adjoint = the present dE/dAEV columns (float32)
    # + the row's neighbour indices + position in + force out; forward = indices
    # + position in, the present AEV columns out (two 16-bit parts, or float32)
    bwd_bytes = n * (cols * 4 + mean_nbr * 4 + 16 + 16)
    aev_out = 2 if precision == "bf16" else 4
    fwd_bytes = n * (mean_nbr * 4 + 16 + cols * aev_out)
    clock_hz = (sm_mhz or 1965.0) * 1e6
    work = mlp_work(pot, box.species, precision)
    units = n * w["n_models"]
    kernels = {
        "mlp": {"kernel": "k_mlp_fused", "ms_per_launch": kt["mlp"], "bound": "tensor",
                "algorithmic_flop_per_launch": flops, "achieved": flops / (kt["mlp"] * 1e-3) / 1e12,
                "unit": "TFLOP/s", "peak": tf_sust, "peak_source": f"{src} bf16 sustained",
                "flop_accounting": ("achieved = dense 1.352 MFLOP per atom and model (1008 inputs); "
                                    "present_column_tflops counts only the AEV columns these species can "
                                    "make non-zero; mma_tflops is the tensor-core work issued (padded "
                                    "widths, active input chunks, split products)"),
                "present_column_tflops": work["present_column_flop"] * units / (kt["mlp"] * 1e-3) / 1e12},
    }
    if "mma_flop" in work:
        mma = work["mma_flop"] * units / (kt["mlp"] * 1e-3) / 1e12
        kernels["mlp"].update(mma_tflops=mma, mma_frac=mma / tf_sust,
                              active_input_columns=work["active_input_columns"])
    for name, kname, b in (("aev_backward", "k_aev_backward", bwd_bytes), ("aev_forward", "k_aev_forward", fwd_bytes)):
        ms = kt[name]
        inst = profile_value("inst_per_launch", kname, workload)
        k = {"kernel": kname, "ms_per_launch": ms, "bound": "issue",
             "algorithmic_bytes_per_launch": b, "hbm_achieved_gbs": b / (ms * 1e-3) / 1e9,
             "hbm_frac": b / (ms * 1e-3) / 1e9 / hbm, "hbm_peak": hbm,
             "warp_inst_per_launch": inst}
        if inst is not None:
            k.update(achieved=inst / (ms * 1e-3) / 1e9, unit="Gwarp-inst/s",
                     peak=SMS * 4 * clock_hz / 1e9,
                     peak_source=f"{SMS} SMs x 4 issue/clk x {clock_hz / 1e6:.0f} MHz (sampled)")
        else:
            k.update(achieved=k["hbm_achieved_gbs"], unit="GB/s", peak=hbm, peak_source=f"{src} HBM copy")
        kernels[name] = k
    for k in kernels.values():
        k["frac"] = k["achieved"] / k["peak"]
    kernels["mean_radial_neighbors"] = mean_nbr
    kernels["mean_angular_neighbors"] = mean_ang
    kernels["aev_columns_present"] = cols
    return kernels


def supercell(box, k):
    L = box.cell[0, 0]
    shifts = np.array([[a, b, c] for a in range(k) for b in range(k) for c in range(k)], dtype=np.float64) * L
    xyz = (box.coordinates[None, :, :] + shifts[:, None, :]).reshape(-1, 3)
    return xyz, np.tile(box.species, k ** 3), box.cell * k


def accuracy(device, precision, n_models):
    """Error of the form against the FP64 oracle for the spec's model (seeded
    N(0, 1/fan_in) float32 weights, unscaled, not rounded): on the 12,288-atom
    box directly, and on its 2x2x2 tiling (98,304 atoms), whose exact energy
    is 8x the box's and whose every copy carries the box's forces."""
    import torch
    from fennol_b200.params import AEVConfig, MLPConfig, init_weights
    from fennol_b200.potential import ANIPotential
    from fennol_b200.systems import water_box
    from oracle import ani_ref

    torch.set_num_threads(os.cpu_count() or 1)
    cfg, mcfg = AEVConfig(), MLPConfig()
    W = init_weights(cfg, mcfg, seed=0, n_models=n_models)
    box = water_box(16, seed=0)
    t = time.perf_counter()
    ref = ani_ref.energy_and_forces(box.coordinates, box.species, [box.natoms], W, cfg, mcfg,
                                    cells=box.cell[None])
    t_oracle = time.perf_counter() - t
    pot = ANIPotential(cfg, mcfg, weights=W, precision=precision, device=device)
    out = {"model": f"{n_models}-model ensemble, seeded N(0, 1/fan_in) float32 weights (not rounded, "
                    "not scaled)", "oracle": "FP64 torch-CPU restatement, autograd forces",
           "force_rmse_tol_kcalmol_A": 0.05, "energy_tol_kcalmol_atom": 1e-4,
           "oracle_seconds": t_oracle}
    e, f = pot.energy_and_forces(box.coordinates, box.species, [box.natoms], box.cell[None])
    out["box_12288"] = {
        "energy_err_kcalmol_atom": abs(float(e[0]) - ref["energy"][0]) * HARTREE_TO_KCALMOL / box.natoms,
        "force_rmse_kcalmol_A": float(np.sqrt(np.mean((f.cpu().numpy() - ref["forces"]) ** 2))
                                      * HARTREE_TO_KCALMOL)}
    xyz, sp, cell = supercell(box, 2)
    e, f = pot.energy_and_forces(xyz, sp, [xyz.shape[0]], cell[None])
    fr = np.tile(ref["forces"], (8, 1))
    out["tiled_98304"] = {
        "energy_err_kcalmol_atom": abs(float(e[0]) - 8 * ref["energy"][0]) * HARTREE_TO_KCALMOL / xyz.shape[0],
        "force_rmse_kcalmol_A": float(np.sqrt(np.mean((f.cpu().numpy() - fr) ** 2)) * HARTREE_TO_KCALMOL),
        "note": "2x2x2 tiling of the 12,288-atom box: exact reference = 8 x its energy, tiled forces"}
    out["within_budget"] = all(v["energy_err_kcalmol_atom"] <= 1e-4 and v["force_rmse_kcalmol_A"] <= 0.05
                               for v in (out["box_12288"], out["tiled_98304"]))
    return out


def ani2x_fennix(precision, n_models, device, output_scale):
    """A FeNNol model description of the ANI-2x network (the ``ANI_AEV`` and
    ``SPECIES_INDEX_NET`` modules with FeNNol's graph preprocessing) built
    through the FeNNol-compatible API, with the workload's ensemble."""
    from fennol_b200.fennix import FENNIX
    from fennol_b200.params import ANI2X_SPECIES, AEVConfig, MLPConfig, init_weights, weights_to_variables

    sp = list(ANI2X_SPECIES)
    modules = OrderedDict(
        embedding=dict(module_name="ANI_AEV", species_order=sp, graph_angle_key="graph_angle", radial_eta=19.7,
                       angular_eta=12.5, radial_dist_divisions=16, angular_dist_divisions=8, zeta=14.1,
                       angle_sections=4, radial_start=0.9, angular_start=0.9),
        energy=dict(module_name="SPECIES_INDEX_NET", species_order=sp, activation="partial(celu,alpha=0.1)",
                    output_dim=1, hidden_neurons=[256, 192, 160], input_key="embedding", squeeze=True))
    prep = OrderedDict(
        graph_filter_angle=dict(module_name="GRAPH_FILTER", cutoff=3.5, graph_key="graph_angle",
                                parent_graph="graph"),
        angle_extension=dict(module_name="GRAPH_ANGULAR_EXTENSION", graph_key="graph_angle"),
        species_indexer=dict(output_key="species_index"))
    W = init_weights(AEVConfig(), MLPConfig(), seed=0, n_models=n_models, output_scale=output_scale)
    return FENNIX(5.2, modules, prep, energy_terms=["energy"], precision=precision, device=device,
                  variables=weights_to_variables(W, "energy"))


def e2e(precision, box, n_models, device, steps, warmup):
    """FeNNol-API single point per step: ``FENNIX.energy_and_forces`` with
    pinned host coordinates in and host forces and energy out (the neighbour
    list is built on every call, with FeNNol's capacity protocol)."""
    import torch
    from fennol_b200.params import MD_OUTPUT_SCALE

    model = ani2x_fennix(precision, n_models, device, MD_OUTPUT_SCALE)
    x_host = torch.tensor(box.coordinates, dtype=torch.float32).pin_memory()
    f_host = torch.empty((box.natoms, 3), dtype=torch.float32).pin_memory()
    e_host = torch.empty(1, dtype=torch.float64).pin_memory()
    args = dict(species=box.species, natoms=np.array([box.natoms]), cells=box.cell[None],
                flags={"minimum_image": True})

    def call():
        e, f, _ = model.energy_and_forces(coordinates=x_host, **args)
        f_host.copy_(f, non_blocking=True)
        e_host.copy_(e[:1], non_blocking=True)
        torch.cuda.current_stream().synchronize()

    for _ in range(warmup):
        call()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        call()
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    return {"value": box.natoms / (ms * 1e-3), "unit": "atom-steps/s", "ms_per_step": ms,
            "h2d_bytes_per_step": int(x_host.numel() * 4),
            "d2h_bytes_per_step": int(f_host.numel() * 4 + 8),
            "api": ("fennix.FENNIX.energy_and_forces (FeNNol API: preprocessing chain with capacity "
                    "checks, list rebuilt every call), host buffers in and out")}


def cpu_baseline(box, n_models, samples=1, warmup=0):
    """The CPU port of the reference algorithm (float32 torch restatement of
    the formulas with autograd forces, numpy float32 all-pairs search) timed
    on this host's cores, on one box per sample."""
    import torch
    from fennol_b200.params import AEVConfig, MLPConfig, init_weights
    from oracle import ani_ref

    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    cfg, mcfg = AEVConfig(), MLPConfig()
    W = init_weights(cfg, mcfg, seed=0, n_models=n_models)
    ts = []
    for k in range(warmup + samples):
        t = time.perf_counter()
        ani_ref.energy_and_forces(box.coordinates, box.species, [box.natoms], W, cfg, mcfg,
                                  cells=box.cell[None], dtype=torch.float32)
        if k >= warmup:
            ts.append(time.perf_counter() - t)
    sec = float(np.mean(ts))
    return {"value": box.natoms / sec, "unit": "atom-steps/s", "cores": cores, "kind": "port",
            "seconds_per_sample": sec, "samples": samples,
            "sample": (f"single-point E+F of the {box.natoms}-atom water box with the {n_models}-model "
                       f"ensemble (all-pairs search + AEV + MLPs + autodiff forces), float32, "
                       f"{sec:.2f} s each; a bounded sample of the 98,304-atom workload, whose per-atom "
                       f"cost on the CPU is higher (the all-pairs search grows as N^2)")}


def step_line(workload, precision, device, steps, warmup, flush, bf16_weights=False):
    """Throughput of one workload in one MLP form (single GPU)."""
    import torch

    box, pot, eng = make_engine(workload, precision, device, bf16_weights=bf16_weights)
    ms, _ = time_steps(eng, steps, warmup, flush)
    res = {"value": box.natoms / (float(ms.mean()) * 1e-3), "unit": "atom-steps/s",
           "ms_per_step": float(ms.mean()), "mlp_ms_per_launch": time_mlp(pot, eng, 5),
           "mlp": MLP_FORMS[precision]}
    del eng, pot
    torch.cuda.empty_cache()
    return res


def nve_trace(eng, steps, every):
    """Total energy per atom, temperature and largest angular-neighbour count
    every ``every`` steps of an NVE run; stops early (saying so) at a list limit."""
    from fennol_b200 import _lib

    n = eng.n
    t_ps, etot, temp, angmax = [], [], [], []
    done, stopped = 0, None
    while True:
        etot.append((eng.potential_energy() + eng.kinetic_energy()) / n)
        temp.append(eng.temperature())
        angmax.append(int(eng.ws.status[_lib.ST_ANG_MAXCOUNT]))
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
    return np.array(t_ps), np.array(etot), np.array(temp), angmax, done, stopped


def _drift(t_ps, e):
    return float(np.polyfit(t_ps, e, 1)[0]) * 1000.0 if len(e) > 2 else 0.0   # per ns


def nve_drift(device, steps, workload="water98k", every=100, precision=DEFAULT_PRECISION, compare_steps=1000):
    """NVE runs of the workload with the model the throughput is timed on
    (last layer x0.02; float64 integrator).

    The random-weight network has no repulsive core: its wells gather atoms,
    so the box heats as it collapses (about 300 -> 600 K over the first ps)
    and close contacts eventually limit energy conservation at dt 0.5 fs.
    Reported: the drift over the whole run and over its first picosecond, the
    temperature trace, and the energy of the same start integrated with the
    float32 MLP form for ``compare_steps`` steps beside this form (the
    precision's own effect on conservation)."""
    import torch
    from fennol_b200.params import MD_OUTPUT_SCALE

    t0 = time.perf_counter()
    box, pot, eng = make_engine(workload, precision, device, output_scale=MD_OUTPUT_SCALE)
    t_ps, e, temp, angmax, done, stopped = nve_trace(eng, steps, every)
    del eng, pot
    torch.cuda.empty_cache()
    first = t_ps <= 1.0 + 1e-9
    out = {"workload": WORKLOADS[workload]["desc"], "precision": precision, "steps": done, "stopped": stopped,
           "dt_fs": 0.5, "samples": len(e), "e0_kcalmol_atom": float(e[0]),
           "drift_kcalmol_atom_per_ns": _drift(t_ps, e),
           "max_abs_dev_kcalmol_atom": float(np.abs(e - e[0]).max()),
           "first_ps": {"drift_kcalmol_atom_per_ns": _drift(t_ps[first], e[first]),
                        "max_abs_dev_kcalmol_atom": float(np.abs(e[first] - e[0]).max()),
                        "temperature_end_K": float(temp[first][-1])},
           "temperature_K": {f"{tp:.1f} ps": round(float(tk), 1) for tp, tk in zip(t_ps[::10], temp[::10])},
           "max_angular_neighbours_end": angmax[-1],
           "note": ("random-init model without a repulsive core: the box heats as atoms gather in its wells; "
                    "conservation is limited by close contacts once T rises, not by the MLP form")}
    if compare_steps > 0 and precision != "fp32":
        traces = {}
        for p in (precision, "fp32"):
            _, pp, ee = make_engine(workload, p, device, output_scale=MD_OUTPUT_SCALE)
            tp, ep, _, _, dn, _ = nve_trace(ee, compare_steps, every)
            traces[p] = (tp[:len(ep)], ep)
            del ee, pp
            torch.cuda.empty_cache()
        (ta, ea), (tb, eb) = traces[precision], traces["fp32"]
        m = min(len(ea), len(eb))
        out["vs_fp32_form"] = {"steps": compare_steps,
                               "drift_kcalmol_atom_per_ns": {precision: _drift(ta[:m], ea[:m]),
                                                             "fp32": _drift(tb[:m], eb[:m])},
                               "max_abs_etot_difference_kcalmol_atom": float(np.abs(ea[:m] - eb[:m]).max())}
    out["wall_s"] = time.perf_counter() - t0
    return out


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
            "path": getattr(lg, "path_description", "CUDA E/F + AEV tangent kernel + network sweep")}


def serving_run(device, n_requests=1000, rate_hz=2000.0, seed=0, precision=DEFAULT_PRECISION):
    """Poisson stream through the continuous-batching loop (real time):
    throughput of the energy/force work done and p50/p99 request latency."""
    from fennol_b200.params import MD_OUTPUT_SCALE
    from fennol_b200.potential import ANIPotential
    from fennol_b200.serving import (ServingEngine, atom_steps, latency_percentiles,
                                     serve_requests_from_stream)
    from fennol_b200.systems import request_stream

    pot = ANIPotential(precision=precision, device=device, seed=0, output_scale=MD_OUTPUT_SCALE)
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
    return {"value": work / wall, "unit": "atom-steps/s", "wall_s": wall, "precision": precision,
            "requests": len(reqs), "md_requests": n_md,
            "atoms_mean": float(np.mean([q.natoms for q in reqs])),
            "latency_ms": {"p50": lat["p50_ms"], "p99": lat["p99_ms"], "mean": lat["mean_ms"]},
            "stream": (f"Poisson {rate_hz:.0f} req/s, atoms log-uniform 8-5000 (chains and water "
                       "boxes, 48 pre-generated systems), 70% single-point E+F, 30% 100-step "
                       "Langevin MD continuations at dt 0.5 fs; HBM budget 120 GB"),
            "captures": eng.md.captures}


def run_reference(args):
    """Reference arm: the CPU port of the reference algorithm on the host
    cores, one bounded sample of the workload per step, rank 0 only."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from fennol_b200.systems import water_box
    w = WORKLOADS[args.workload]
    # the 98,304-atom box needs 4.8e9 all-pairs candidates per step on the CPU;
    # a step of this arm is the 12,288-atom box with the workload's ensemble
    box = water_box(min(w["n_side"], 16), seed=0)
    base = cpu_baseline(box, w["n_models"], samples=args.steps, warmup=args.warmup)
    line = {"metric": METRIC, "value": base["value"], "unit": "atom-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": base["seconds_per_sample"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": w["desc"], "sample": base["sample"]},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": ("the reference (JAX/Flax) is not installed in this image; its CPU path is "
                     "restated by the oracle and timed on the host cores")}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="water98k", choices=list(WORKLOADS))
    ap.add_argument("--precision", default=DEFAULT_PRECISION, choices=list(MLP_FORMS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true",
                    help="headline, e2e and rooflines only (no comparisons, accuracy or side runs)")
    ap.add_argument("--skip-serving", action="store_true", help="skip the request-stream run")
    ap.add_argument("--skip-training", action="store_true", help="skip the training-gradient timing")
    ap.add_argument("--nve-drift-steps", type=int, default=10000,
                    help="NVE energy-drift run of the 98k-atom ensemble on the MD model (0: skip)")
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

    precision = args.precision
    w = WORKLOADS[args.workload]
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
    clk = clocks.summary()

    res = {"metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": {"fp32": "f32", "f16x3x1": "f16", "f16x3x2": "f16"}.get(precision, "bf16"),
           "data": "synthetic",
           "config": {"workload": w["desc"], "atoms_per_gpu": box.natoms, "models": w["n_models"],
                      "precision": precision, "mlp_precision": MLP_FORMS[precision],
                      "weights": ("seeded N(0, 1/fan_in) float32 weights, not rounded (MD runs scale the "
                                  "last layer by 0.02; accuracy uses the unscaled model)"),
                      "aev": "float32", "energy_sum_and_integrator": "float64",
                      "l2": "flushed between timed steps (512 MB write outside the events)",
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
           "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
           "clocks": clk,
           "gpu_launches": eng.launches_per_step() * args.steps + eng.rebuild_launches() * rebuilds,
           "rebuilds_in_run": rebuilds,
           "neighbour_list": {"trigger": eng.trigger, "nblist_stride": eng.nblist_stride,
                              "stride_shortenings": eng.stride_reductions}}
    if rank == 0:
        kernels = rooflines(pot, eng, box, args.workload, precision, clk.get("sm_mhz"))
        res["kernels"] = kernels
        top = max(("aev_backward", "aev_forward", "mlp"), key=lambda k: kernels[k]["ms_per_launch"])
        kd = kernels[top]
        res["roofline"] = {"bound": kd["bound"], "kernel": kd["kernel"], "achieved": kd["achieved"],
                           "peak": kd["peak"], "unit": kd["unit"], "frac": kd["frac"],
                           "traffic": profile_value("traffic_bytes_per_launch", kd["kernel"], args.workload),
                           "peak_source": kd["peak_source"], "ms_per_launch": kd["ms_per_launch"],
                           "algorithmic_per_launch": kd.get("algorithmic_flop_per_launch",
                                                            kd.get("algorithmic_bytes_per_launch"))}
    del eng, pot
    torch.cuda.empty_cache()
    # end-to-end FeNNol-API calls on every rank; the job rate uses the slowest rank
    e2e_res = e2e(precision, box, w["n_models"], device, max(5, args.steps // 4), max(3, args.warmup))
    if world > 1:
        from fennol_b200.replicas import max_over_ranks
        ms_e2e = max_over_ranks(e2e_res["ms_per_step"], device)
        e2e_res.update(value=world * box.natoms / (ms_e2e * 1e-3), ms_per_step=ms_e2e,
                       h2d_bytes_per_step=world * e2e_res["h2d_bytes_per_step"],
                       d2h_bytes_per_step=world * e2e_res["d2h_bytes_per_step"])
    res["e2e"] = e2e_res
    # the comparisons below are single-GPU measurements, made at N = 1 only
    extras = world == 1 and rank == 0 and not args.quick
    if extras:
        if precision != "fp32":
            res["fp32_form"] = step_line(args.workload, "fp32", device, max(5, args.steps // 4), 3, flush)
            res["speedup_vs_fp32_form"] = value / world / res["fp32_form"]["value"]
        forms = {}
        for p, rounded in (("f16x3x2", False), ("bf16x2", True)):
            if p != precision:
                r = step_line(args.workload, p, device, max(5, args.steps // 4), 3, flush, bf16_weights=rounded)
                if rounded:
                    r["weights"] = "the same model rounded to BF16 (a different model: exact only for BF16 weights)"
                forms[p if not rounded else "bf16x2_bf16_model"] = r
        res["other_forms"] = forms
        res["accuracy_vs_fp64_oracle"] = accuracy(device, precision, w["n_models"])
        if args.workload != "water12k":
            c2 = step_line("water12k", precision, device, args.steps, 3, flush)
            c2["fp32_form"] = step_line("water12k", "fp32", device, max(5, args.steps // 4), 3, flush)
            c2["speedup_vs_fp32_form"] = c2["value"] / c2["fp32_form"]["value"]
            c2["workload"] = WORKLOADS["water12k"]["desc"]
            res["water12k"] = c2
        if not args.skip_serving:
            res["serving"] = serving_run(device)
            # below saturation the latencies measure service, not queueing
            res["serving_500rps"] = serving_run(device, rate_hz=500.0)
        if not args.skip_training:
            res["training_256mol"] = training_256(device)
        if args.nve_drift_steps > 0:
            res["nve_drift"] = nve_drift(device, args.nve_drift_steps)
        if not args.no_cpu_baseline:
            from fennol_b200.systems import water_box
            res["cpu_baseline"] = cpu_baseline(water_box(min(w["n_side"], 16), seed=0), w["n_models"])
    if rank == 0:
        print(json.dumps(res), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
