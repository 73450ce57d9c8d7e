"""Parameter gradients of an energy + force training loss through the
hand-written adjoints.

FeNNol trains with ``jax.value_and_grad`` over a loss that holds forces
(``src/fennol/training/utils.py:140-525``; ``train_step`` at ``:508``), i.e.
second-order automatic differentiation through the whole model.  Here the
same gradient is assembled from explicit pieces:

* energies and forces from the CUDA path (pair search, AEV, species MLPs,
  energy sum, force adjoint);
* the loss ``L = w_e * mean_b (E_b - E_ref_b)^2 + w_f * mean (F - F_ref)^2``
  and its seeds ``dL/dE_b`` and ``u = dL/dF``;
* the AEV tangent ``t = dAEV/dx . u`` (``fennol_aev_tangent``), because
  ``sum_k u_k . dF_k/dtheta = -d/dtheta sum_i <dE/dAEV_i, t_i>`` with ``t``
  independent of the network parameters;
* per species, the network activations recomputed from the AEV rows, their
  tangents along ``t``, and one reverse sweep that returns the gradient of
  ``sum_rows (dL/dE * E_row - <dE_row/dAEV_row, t_row>)`` with respect to
  every kernel and bias (CELU first and second derivatives included).

The network part runs as plain GEMMs on the device (torch/cuBLAS), in
float32 by default or float64.
"""

from __future__ import annotations

import dataclasses
from typing import Dict, List, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import call
from .potential import ANIPotential, C_ptr, _stream


@dataclasses.dataclass
class LossTerms:
    loss: float
    energy_loss: float
    force_loss: float
    energy: np.ndarray   # [B] model unit
    forces: np.ndarray   # [N, 3]


def _celu_parts(z: torch.Tensor, alpha: float):
    """celu(z), celu'(z), celu''(z) as jax.nn.celu defines them (x > 0 branch)."""
    pos = z > 0
    ez = torch.exp(torch.clamp(z, max=0.0) / alpha)
    h = torch.where(pos, z, alpha * (ez - 1.0))
    d1 = torch.where(pos, torch.ones_like(z), ez)
    d2 = torch.where(pos, torch.zeros_like(z), ez / alpha)
    return h, d1, d2


def network_loss_gradient(a: torch.Tensor, t: torch.Tensor, c_e: torch.Tensor, layers, alpha: float):
    """Gradient with respect to ``layers`` [(W, b), ...] (torch, on device) of
    ``sum_rows c_e[row] * f(a_row) - <grad_a f(a_row), t_row>`` for the
    network ``f`` (CELU hidden layers, linear output of width 1)."""
    n_hidden = len(layers) - 1
    d1s, d2s, hs, zds, hds = [], [], [a], [], [t]
    h, hd = a, t
    for W, b in layers[:-1]:
        z = h @ W + b
        zd = hd @ W
        h, d1, d2 = _celu_parts(z, alpha)
        hd = d1 * zd
        d1s.append(d1), d2s.append(d2), zds.append(zd)
        hs.append(h), hds.append(hd)
    W4, _ = layers[-1]
    # seeds: energy output f -> c_e; tangent output s = hd_last . w4 -> -1
    grads: List[Tuple[torch.Tensor, torch.Tensor]] = [None] * len(layers)
    grads[-1] = (hs[-1].t() @ c_e[:, None] - hds[-1].sum(0)[:, None], c_e.sum().reshape(1))
    hbar = c_e[:, None] * W4[:, 0][None, :]          # d/dh of the energy term
    hdbar = -W4[:, 0][None, :].expand_as(hds[-1])    # d/dh-dot of the tangent term
    for l in range(n_hidden - 1, -1, -1):
        d1, d2, zd = d1s[l], d2s[l], zds[l]
        zdbar = d1 * hdbar
        zbar = d1 * hbar + d2 * zd * hdbar
        W, _ = layers[l]
        grads[l] = (hs[l].t() @ zbar + hds[l].t() @ zdbar, zbar.sum(0))
        if l > 0:
            hbar = zbar @ W.t()
            hdbar = zdbar @ W.t()
    return grads


class LossGradient:
    """Energy + force loss and its parameter gradient for a batch of systems.

    ``pot`` holds the (single-model) network; ``w_e`` / ``w_f`` weight the
    mean squared energy and force-component errors.  Energies are in the
    potential's unit, forces per Angstrom.
    """

    def __init__(self, pot: ANIPotential, w_e: float = 1.0, w_f: float = 10.0,
                 dtype: torch.dtype = torch.float32):
        if pot.mlp.n_models != 1:
            raise ValueError("training gradients are computed for one model")
        self.pot, self.w_e, self.w_f, self.dtype = pot, w_e, w_f, dtype
        dev = pot.device
        self.layers = {sym: [(torch.tensor(w, dtype=dtype, device=dev), torch.tensor(b, dtype=dtype, device=dev))
                             for w, b in layers]
                       for sym, layers in pot.weights[0].items()}

    def __call__(self, coordinates, species, natoms, e_ref, f_ref, cells=None):
        pot, dev = self.pot, self.pot.device
        natoms = np.asarray(natoms).reshape(-1)
        energy, forces = pot.energy_and_forces(coordinates, species, natoms, cells)
        layout, g, ws = next(iter(pot._cache.values()))
        B, N = int(natoms.shape[0]), int(layout.n)
        e_ref_t = torch.as_tensor(np.asarray(e_ref, np.float64), device=dev)
        f_ref_t = torch.as_tensor(np.asarray(f_ref, np.float64), device=dev).reshape(N, 3)
        de = energy - e_ref_t
        df = forces.double() - f_ref_t
        losses = torch.stack([(de ** 2).mean(), (df ** 2).mean()])
        c_sys = (2.0 * self.w_e / B) * de                      # dL/dE_b
        u = (2.0 * self.w_f / (3 * N)) * df                    # dL/dF
        du4 = torch.zeros((N, 4), dtype=torch.float32, device=dev)
        du4[:, :3] = u.float()
        d0 = ws.x.shape[1]
        t = torch.zeros((layout.rows, d0), dtype=torch.float32, device=dev)
        status = torch.zeros(_lib.STATUS_WORDS, dtype=torch.int32, device=dev)
        call("fennol_aev_tangent", ws.xyzs.data_ptr(), N, layout.t_atom_sys.data_ptr(), layout.t_cell.data_ptr(),
             g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(), g.cap_r, C_ptr(pot.params),
             layout.t_atom_row.data_ptr(), du4.data_ptr(), t.data_ptr(), d0, status.data_ptr(), _stream(dev))
        F = pot.aev_cfg.aev_length
        x = ws.x.float()
        if ws.x_lo is not None:
            x = x + ws.x_lo.float()
        # per-row energy seeds in the species-sorted row order of the AEV
        c_row = torch.zeros(layout.rows, dtype=self.dtype, device=dev)
        c_row[layout.t_atom_row.long()] = c_sys[layout.t_atom_sys.long()].to(self.dtype)
        dev_grads: Dict[str, list] = {}
        for k, row0, count in layout.species_segments:
            sym = pot.aev_cfg.species_order[k]
            sl = slice(row0, row0 + count)
            dev_grads[sym] = network_loss_gradient(x[sl, :F].to(self.dtype), t[sl, :F].to(self.dtype),
                                                   c_row[sl], self.layers[sym], pot.mlp_cfg.celu_alpha)
        # one transfer for the whole gradient
        parts, shapes = [], []
        for sym in pot.aev_cfg.species_order:
            for l, (W, b) in enumerate(self.layers[sym]):
                if sym in dev_grads:
                    gW, gb = dev_grads[sym][l]
                else:
                    gW, gb = torch.zeros_like(W), torch.zeros_like(b)
                parts += [gW.reshape(-1), gb.reshape(-1)]
                shapes += [tuple(W.shape), tuple(b.shape)]
        flat = torch.cat([p_.double() for p_ in parts]).cpu().numpy()
        grads: Dict[str, List[Tuple[np.ndarray, np.ndarray]]] = {}
        pos, i = 0, 0
        for sym in pot.aev_cfg.species_order:
            layers = []
            for _ in self.layers[sym]:
                arrs = []
                for _k in range(2):
                    size = int(np.prod(shapes[i]))
                    arrs.append(flat[pos:pos + size].reshape(shapes[i]))
                    pos += size
                    i += 1
                layers.append(tuple(arrs))
            grads[sym] = layers
        l_e, l_f = (float(v) for v in (losses * torch.tensor([self.w_e, self.w_f], dtype=losses.dtype,
                                                              device=dev)).cpu())
        if int(status[_lib.ST_ANG_OVERFLOW]):
            raise RuntimeError(f"more than {_lib.MAX_ANGULAR_NEIGHBORS} angular neighbours around one atom")
        terms = LossTerms(l_e + l_f, l_e, l_f, energy.cpu().numpy(), forces.cpu().numpy())
        return terms, grads


def flatten(grads: Dict[str, List[Tuple[np.ndarray, np.ndarray]]], species_order) -> np.ndarray:
    """Concatenate a gradient (or weight) dictionary in a fixed order."""
    parts = []
    for sym in species_order:
        for W, b in grads[sym]:
            parts.append(np.asarray(W).ravel())
            parts.append(np.asarray(b).ravel())
    return np.concatenate(parts)
