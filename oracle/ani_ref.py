"""Torch-CPU restatement of the ANI-2x energy and forces (oracle; test-only).

Forward formulas follow the reference line by line (paths within
thomasple/FeNNol):

* edge geometry ``vec = x[dst] - x[src] + shift @ cell``,
  ``d = sqrt(max(sum(vec**2), 1e-5))`` (``GraphProcessor``,
  ``src/fennol/models/preprocessing.py:719-740``; ``safe_sqrt``
  ``src/fennol/utils/activations.py:173-174``);
* cosine switch ``0.5*cos(pi d / rc) + 0.5`` masked by ``d < rc``
  (``SwitchFunction``, ``src/fennol/models/misc/misc.py:674-708``);
* angular sub-graph gathered through ``filter_indices``
  (``GraphFilterProcessor``, ``preprocessing.py:979-1043``);
* ``theta = arccos(0.95 * dir_j . dir_k)`` with ``dir = vec / max(d, 1e-5)``
  (``GraphAngleProcessor``, ``preprocessing.py:1294-1317``);
* radial and angular AEV (``ANIAEV.__call__``,
  ``src/fennol/models/embeddings/ani.py:64-139``);
* per-species MLP with CELU (``SpeciesIndexNet``/``FullyConnectedNet``,
  ``src/fennol/models/misc/nets.py:82-102, 397-417``);
* per-system energy ``segment_sum`` (``src/fennol/models/fennix.py:218-258``)
  and forces ``-dE/dx`` by reverse-mode autodiff (``fennix.py:260-272``).

Float64 by default (the FP64 oracle the error budgets are quoted against).
"""

from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import graph_fp32


def triu_pair_index(num_species: int) -> np.ndarray:
    """``triu_index[s1, s2]`` from ``np.triu_indices(S, 0)`` order (ani.py:123-129)."""
    s1, s2 = np.triu_indices(num_species, 0)
    t = np.zeros((num_species, num_species), dtype=np.int64)
    t[s1, s2] = np.arange(s1.shape[0])
    t[s2, s1] = np.arange(s1.shape[0])
    return t


def celu(x: torch.Tensor, alpha: float) -> torch.Tensor:
    """``jax.nn.celu``: ``x if x > 0 else alpha*expm1(x/alpha)``, evaluated as
    ``max(x, 0) + alpha*expm1(min(x, 0)/alpha)`` so that the exponential never
    sees a large positive argument (a ``where`` over both branches would give
    NaN gradients through the untaken branch for inputs above ~71)."""
    return torch.clamp(x, min=0) + alpha * torch.expm1(torch.clamp(x, max=0) / alpha)


class Graph:
    """Directed radial graph + angular sub-graph + triplets for one batch."""

    def __init__(self, coordinates, natoms, cells=None, reciprocal_cells=None,
                 radial_cutoff=5.2, angular_cutoff=3.5, minimum_image=True,
                 pairs: Optional[dict] = None):
        coordinates = np.asarray(coordinates)
        self.nat = coordinates.shape[0]
        natoms = np.asarray(natoms).reshape(-1)
        self.batch_index = np.repeat(np.arange(natoms.shape[0]), natoms)
        if pairs is None:
            pairs = graph_fp32.pair_list(coordinates, natoms, cells, reciprocal_cells,
                                         radial_cutoff, minimum_image)
        self.pairs = pairs
        src, dst, sh, d12 = graph_fp32.symmetrize(pairs)
        self.src, self.dst, self.shift, self.d12 = src, dst, sh, d12
        # angular sub-graph: filter on the parent's d12 (preprocessing.py:854-866)
        self.filter_indices = np.nonzero(d12 < np.float32(angular_cutoff ** 2))[0]
        a_src = src[self.filter_indices]
        self.angle_src, self.angle_dst, self.central_atom = \
            graph_fp32.angular_triplets(a_src, self.nat)
        self.cells = None if cells is None else np.asarray(cells, dtype=np.float64).reshape(-1, 3, 3)
        self.radial_cutoff = radial_cutoff
        self.angular_cutoff = angular_cutoff


def _switch(d, mask, rc):
    return torch.where(mask, 0.5 * torch.cos(d * (math.pi / rc)) + 0.5, torch.zeros_like(d))


def aev(coords: torch.Tensor, species_idx: np.ndarray, g: Graph, cfg,
        strain: Optional[torch.Tensor] = None) -> torch.Tensor:
    """ANIAEV embedding ``[nat, F]`` (ani.py:47-139).  ``strain`` ([B,3,3]):
    every edge vector of system b becomes ``vec @ strain[b]`` (the homogeneous
    deformation the reference differentiates for the virial, fennix.py:320-347)."""
    dt = coords.dtype
    nat = coords.shape[0]
    S = cfg.num_species
    P = S * (S + 1) // 2
    src = torch.as_tensor(g.src)
    dst = torch.as_tensor(g.dst)
    vec = coords[dst] - coords[src]
    if g.cells is not None:
        sh = torch.as_tensor(g.shift, dtype=dt)
        if g.cells.shape[0] == 1:
            vec = vec + sh @ torch.as_tensor(g.cells[0], dtype=dt)
        else:
            cb = torch.as_tensor(g.cells, dtype=dt)[torch.as_tensor(g.batch_index)[src]]
            vec = vec + torch.einsum("ej,eji->ei", sh, cb)
    if strain is not None:
        vec = torch.einsum("ej,ejk->ek", vec, strain[torch.as_tensor(g.batch_index)[src]])
    d2 = (vec ** 2).sum(-1)
    dist = torch.sqrt(torch.clamp(d2, min=1e-5))
    rc = g.radial_cutoff
    sw = _switch(dist, dist < rc, rc)
    spec = torch.as_tensor(species_idx, dtype=torch.long)

    # radial (ani.py:71-86)
    shiftR = torch.as_tensor(-cfg.radial_shifts()[None, :], dtype=dt)
    x2 = cfg.radial_eta * (dist[:, None] + shiftR) ** 2
    rterms = torch.exp(-x2) * (0.25 * sw)[:, None]
    ridx = src * S + spec[dst]
    rad = torch.zeros(nat * S, cfg.radial_dist_divisions, dtype=dt)
    rad = rad.index_add(0, ridx, rterms).reshape(nat, S * cfg.radial_dist_divisions)

    # angular sub-graph (preprocessing.py:1000-1043)
    fi = torch.as_tensor(g.filter_indices)
    vec_a = vec[fi]
    dist_a = dist[fi]
    rca = g.angular_cutoff
    sw_a = _switch(dist_a, dist_a < rca, rca)
    # angles (preprocessing.py:1294-1317)
    asrc = torch.as_tensor(g.angle_src)
    adst = torch.as_tensor(g.angle_dst)
    # angle_src/dst index the *filtered* edge list
    direc = vec_a / torch.clamp(dist_a[:, None], min=1e-5)
    cosang = (direc[asrc] * direc[adst]).sum(-1)
    angles = torch.arccos(0.95 * cosang)
    # angular AEV (ani.py:88-137)
    sq = cfg.angular_eta ** 0.5
    dsc = (0.5 * sq) * dist_a
    d12 = (dsc[asrc] + dsc[adst])[:, None]
    shiftZ = torch.as_tensor(-cfg.angle_shifts()[None, :], dtype=dt)
    shiftA = torch.as_tensor((-sq) * cfg.angular_shifts()[None, :], dtype=dt)
    swz = sw_a * (2.0 * (0.5 ** cfg.zeta)) ** 0.5
    f1 = (swz[asrc] * swz[adst])[:, None] * (1 + torch.cos(angles[:, None] + shiftZ)) ** cfg.zeta
    f2 = torch.exp(-(d12 + shiftA) ** 2)
    aterms = (f1[:, None, :] * f2[:, :, None]).reshape(-1, cfg.angle_sections * cfg.angular_dist_divisions)
    a_dst_atoms = torch.as_tensor(g.dst)[fi]
    sp_d = spec[a_dst_atoms]
    triu = torch.as_tensor(triu_pair_index(S))
    central = torch.as_tensor(g.central_atom)
    aidx = central * P + triu[sp_d[asrc], sp_d[adst]]
    ang = torch.zeros(nat * P, aterms.shape[1], dtype=dt)
    ang = ang.index_add(0, aidx, aterms).reshape(nat, P * aterms.shape[1])
    return torch.cat([rad, ang], dim=-1)


def species_net(x: torch.Tensor, species_idx: np.ndarray, model: Dict, species_order: Sequence[str],
                alpha: float) -> torch.Tensor:
    """``SpeciesIndexNet``: one FullyConnectedNet per species (nets.py:397-417)."""
    out = torch.zeros(x.shape[0], dtype=x.dtype)
    for k, sym in enumerate(species_order):
        idx = np.nonzero(species_idx == k)[0]
        if idx.size == 0:
            continue
        h = x[torch.as_tensor(idx)]
        layers = model[sym]
        for li, (w, b) in enumerate(layers):
            h = h @ torch.as_tensor(w, dtype=x.dtype) + torch.as_tensor(b, dtype=x.dtype)
            if li < len(layers) - 1:
                h = celu(h, alpha)
        out = out.index_put((torch.as_tensor(idx),), h[:, 0])
    return out


def energy_and_forces(coordinates, species, natoms, weights: List[Dict], aev_cfg, mlp_cfg,
                      cells=None, reciprocal_cells=None, minimum_image=True,
                      dtype=torch.float64, graph: Optional[Graph] = None,
                      need_forces: bool = True, return_aev: bool = False):
    """Energies [B] (Ha, ensemble mean), forces [N,3] (Ha/A), atomic energies [N].

    ``species`` are atomic numbers.  The pair list comes from the float32
    builder, as in the reference (coordinates are cast to float32 there even
    in double precision runs, ``preprocessing.py:81``).
    """
    coordinates = np.asarray(coordinates, dtype=np.float64)
    natoms = np.asarray(natoms).reshape(-1)
    if graph is None:
        graph = Graph(coordinates, natoms, cells, reciprocal_cells,
                      aev_cfg.radial_cutoff, aev_cfg.angular_cutoff, minimum_image)
    sidx = aev_cfg.species_index(species)
    x = torch.tensor(coordinates, dtype=dtype, requires_grad=need_forces)
    emb = aev(x, sidx, graph, aev_cfg)
    eat = None
    for model in weights:
        e = species_net(emb, sidx, model, aev_cfg.species_order, mlp_cfg.celu_alpha)
        eat = e if eat is None else eat + e
    eat = eat / len(weights)
    bidx = torch.as_tensor(graph.batch_index)
    etot = torch.zeros(natoms.shape[0], dtype=dtype).index_add(0, bidx, eat)
    forces = None
    if need_forces:
        (g,) = torch.autograd.grad(etot.sum(), x)
        forces = (-g).detach().numpy()
    res = {"energy": etot.detach().numpy(), "forces": forces,
           "atomic_energies": eat.detach().numpy(), "graph": graph}
    if return_aev:
        res["aev"] = emb.detach().numpy()
    return res


def loss_and_grads(coordinates, species, natoms, model: Dict, aev_cfg, mlp_cfg, e_ref, f_ref,
                   w_e: float = 1.0, w_f: float = 10.0, cells=None, minimum_image=True,
                   dtype=torch.float64, graph: Optional[Graph] = None):
    """Energy + force loss of one model and its gradient with respect to every
    kernel and bias, by second-order autograd (what ``jax.value_and_grad``
    over the loss of ``training/utils.py:140-525`` computes).

    ``L = w_e * mean_b (E_b - e_ref_b)^2 + w_f * mean (F - f_ref)^2``.
    Returns (loss, {symbol: [(dW, db), ...]}) as float64 numpy."""
    coordinates = np.asarray(coordinates, dtype=np.float64)
    natoms = np.asarray(natoms).reshape(-1)
    if graph is None:
        graph = Graph(coordinates, natoms, cells, None, aev_cfg.radial_cutoff, aev_cfg.angular_cutoff,
                      minimum_image)
    sidx = aev_cfg.species_index(species)
    params = {sym: [(torch.tensor(np.asarray(w), dtype=dtype, requires_grad=True),
                     torch.tensor(np.asarray(b), dtype=dtype, requires_grad=True)) for w, b in layers]
              for sym, layers in model.items()}
    x = torch.tensor(coordinates, dtype=dtype, requires_grad=True)
    emb = aev(x, sidx, graph, aev_cfg)
    eat = species_net(emb, sidx, params, aev_cfg.species_order, mlp_cfg.celu_alpha)
    bidx = torch.as_tensor(graph.batch_index)
    etot = torch.zeros(natoms.shape[0], dtype=dtype).index_add(0, bidx, eat)
    (g,) = torch.autograd.grad(etot.sum(), x, create_graph=True)
    forces = -g
    e_ref = torch.as_tensor(np.asarray(e_ref, np.float64), dtype=dtype)
    f_ref = torch.as_tensor(np.asarray(f_ref, np.float64), dtype=dtype).reshape(forces.shape)
    loss = w_e * ((etot - e_ref) ** 2).mean() + w_f * ((forces - f_ref) ** 2).mean()
    flat = [p for sym in aev_cfg.species_order for wb in params[sym] for p in wb]
    gl = torch.autograd.grad(loss, flat, allow_unused=True)
    out, k = {}, 0
    for sym in aev_cfg.species_order:
        layers = []
        for w, b in params[sym]:
            gw = gl[k] if gl[k] is not None else torch.zeros_like(w)
            gb = gl[k + 1] if gl[k + 1] is not None else torch.zeros_like(b)
            layers.append((gw.detach().numpy(), gb.detach().numpy()))
            k += 2
        out[sym] = layers
    return float(loss.detach()), out


def loss_value(coordinates, species, natoms, model: Dict, aev_cfg, mlp_cfg, e_ref, f_ref,
               w_e: float = 1.0, w_f: float = 10.0, cells=None, graph: Optional[Graph] = None):
    """The loss of :func:`loss_and_grads` alone (float64), for finite differences."""
    r = energy_and_forces(coordinates, species, natoms, [model], aev_cfg, mlp_cfg, cells=cells,
                          graph=graph)
    e = np.asarray(r["energy"]) - np.asarray(e_ref, np.float64)
    f = np.asarray(r["forces"]) - np.asarray(f_ref, np.float64).reshape(r["forces"].shape)
    return float(w_e * np.mean(e ** 2) + w_f * np.mean(f ** 2))


def energy_forces_virial(coordinates, species, natoms, weights: List[Dict], aev_cfg, mlp_cfg,
                         cells=None, minimum_image=True, dtype=torch.float64):
    """Energies, forces and the reference's ``virial_tensor`` = dE/dS at S = 1
    for x -> x S, cell -> cell S per system (fennix.py:320-347), FP64 autograd."""
    coordinates = np.asarray(coordinates, dtype=np.float64)
    natoms = np.asarray(natoms).reshape(-1)
    graph = Graph(coordinates, natoms, cells, None, aev_cfg.radial_cutoff, aev_cfg.angular_cutoff,
                  minimum_image)
    sidx = aev_cfg.species_index(species)
    x = torch.tensor(coordinates, dtype=dtype, requires_grad=True)
    S = torch.eye(3, dtype=dtype).repeat(natoms.shape[0], 1, 1).requires_grad_(True)
    emb = aev(x, sidx, graph, aev_cfg, strain=S)
    eat = None
    for model in weights:
        e = species_net(emb, sidx, model, aev_cfg.species_order, mlp_cfg.celu_alpha)
        eat = e if eat is None else eat + e
    eat = eat / len(weights)
    etot = torch.zeros(natoms.shape[0], dtype=dtype).index_add(0, torch.as_tensor(graph.batch_index), eat)
    gx, gs = torch.autograd.grad(etot.sum(), (x, S))
    return {"energy": etot.detach().numpy(), "forces": (-gx).numpy(), "virial": gs.numpy()}
