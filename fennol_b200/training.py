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

The network part is ``fennol_net_loss_grad`` (``csrc/train.cu``): grouped
CUDA-core GEMMs and CELU kernels over all species of the batch, in float32
by default or float64.
"""

from __future__ import annotations

import ctypes
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


class LossGradient:
    """Energy + force loss and its parameter gradient for a batch of systems.

    ``pot`` holds the (single-model) network; ``w_e`` / ``w_f`` weight the
    mean squared energy and force-component errors.  Energies are in the
    potential's unit, forces per Angstrom.
    """

    def __init__(self, pot: ANIPotential, w_e: float = 1.0, w_f: float = 10.0,
                 dtype: torch.dtype = torch.float32, use_graphs: bool = True):
        if pot.mlp.n_models != 1:
            raise ValueError("training gradients are computed for one model")
        self.pot, self.w_e, self.w_f, self.dtype = pot, w_e, w_f, dtype
        dev = pot.device
        self.layers = {sym: [(torch.tensor(w, dtype=dtype, device=dev), torch.tensor(b, dtype=dtype, device=dev))
                             for w, b in layers]
                       for sym, layers in pot.weights[0].items()}
        self.shapes = [tuple(t_.shape) for sym in pot.aev_cfg.species_order for wb in self.layers[sym]
                       for t_ in wb]
        # the networks as fennol_net_loss_grad reads them; output pointers per call
        order = pot.aev_cfg.species_order
        net = _lib.NetTrain()
        net.n_species = len(order)
        dims = [self.layers[order[0]][0][0].shape[0]] + [w.shape[1] for w, _ in self.layers[order[0]]]
        for k in range(5):
            net.dims[k] = int(dims[k])
        net.celu_alpha = pot.mlp_cfg.celu_alpha
        net.is_double = int(dtype == torch.float64)
        for s, sym in enumerate(order):
            for l, (W, b) in enumerate(self.layers[sym]):
                net.w[l][s] = W.data_ptr()
                net.b[l][s] = b.data_ptr()
        self.net = net
        self.offsets = {}   # (species, layer) -> (kernel offset, bias offset) in the flat gradient
        pos = 0
        for s, sym in enumerate(order):
            for l, (W, b) in enumerate(self.layers[sym]):
                self.offsets[(s, l)] = (pos, pos + W.numel())
                pos += W.numel() + b.numel()
        self._ws = {}
        self.path_description = ("CUDA E/F + AEV tangent kernel + fennol_net_loss_grad (grouped CUDA-core "
                                 f"GEMMs and CELU kernels, {'float64' if net.is_double else 'float32'}), "
                                 "one CUDA-graph replay per call from the third call on a batch")
        self.use_graphs = use_graphs
        self._rec = None      # captured pass of the current batch
        self._seen = None     # batch key of the previous call

    # ------------------------------------------------------------ device pass
    def _device_pass(self, layout, g, ws, coords, e_ref, f_ref, out):
        """Every launch of one loss + gradient evaluation, from device inputs
        to the flat device output [status words, E loss, F loss, gradient].
        No host synchronisation, so it can be captured in a CUDA graph."""
        pot, dev = self.pot, self.pot.device
        st = _stream(dev)
        B, N = layout.nsys, layout.n
        pot._launch_all(layout, g, ws, coords, st, True)
        energy, forces = ws.energy, ws.forces[:N]
        de = energy - e_ref
        df = forces.double() - f_ref
        c_sys = (2.0 * self.w_e / B) * de                      # dL/dE_b
        u = (2.0 * self.w_f / (3 * N)) * df                    # dL/dF
        du4 = torch.zeros((N, 4), dtype=torch.float32, device=dev)
        du4[:, :3] = u.float()
        d0 = ws.x.shape[1]
        t = torch.zeros((layout.rows, d0), dtype=torch.float32, device=dev)
        call("fennol_aev_tangent", ws.xyzs.data_ptr(), N, layout.t_atom_sys.data_ptr(), layout.t_cell.data_ptr(),
             g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(), g.cap_r, C_ptr(pot.params),
             layout.t_atom_row.data_ptr(), du4.data_ptr(), t.data_ptr(), d0, ws.status.data_ptr(), st)
        x = ws.x
        if ws.x_lo is not None:
            x = x.float() + ws.x_lo.float()
        x = x.to(self.dtype).contiguous()
        t = t.to(self.dtype).contiguous()
        # per-row energy seeds in the species-sorted row order of the AEV
        c_row = torch.zeros(layout.rows, dtype=self.dtype, device=dev)
        c_row[layout.t_atom_row.long()] = c_sys[layout.t_atom_sys.long()].to(self.dtype)
        out_small, out_grad = out
        torch.cat([ws.status.double(), torch.stack([self.w_e * (de ** 2).mean(), self.w_f * (df ** 2).mean()])],
                  out=out_small)
        # the network sweep of every species present, straight into the flat gradient
        S = self.net.n_species
        row0 = np.zeros(S, np.int32)
        rows = np.zeros(S, np.int32)
        for k, r0, count in layout.species_segments:
            row0[k], rows[k] = r0, count
        net = self.net
        base, esz = out_grad.data_ptr(), out_grad.element_size()
        for (s, l), (ow, ob) in self.offsets.items():
            net.gw[l][s] = base + ow * esz
            net.gb[l][s] = base + ob * esz
        out_grad.zero_()
        key = rows.tobytes()
        if key not in self._ws:
            nb = _lib.load().fennol_net_loss_grad_workspace_bytes(ctypes.byref(net), rows.ctypes.data)
            self._ws = {key: torch.empty(max(int(nb), 256), dtype=torch.uint8, device=dev)}
        wsb = self._ws[key]
        call("fennol_net_loss_grad", ctypes.byref(net), row0.ctypes.data, rows.ctypes.data, x.data_ptr(),
             t.data_ptr(), d0, c_row.data_ptr(), wsb.data_ptr(), wsb.numel(), st)

    def __call__(self, coordinates, species, natoms, e_ref, f_ref, cells=None):
        pot, dev = self.pot, self.pot.device
        natoms = np.asarray(natoms).reshape(-1)
        species = np.asarray(species)
        key = (species.tobytes(), natoms.tobytes(),
               None if cells is None else np.asarray(cells, np.float32).tobytes())
        coords = torch.as_tensor(coordinates, dtype=torch.float32).to(dev).reshape(-1, 3).contiguous()
        e_ref_t = torch.as_tensor(np.asarray(e_ref, np.float64), device=dev).reshape(-1)
        f_ref_t = torch.as_tensor(np.asarray(f_ref, np.float64), device=dev).reshape(-1, 3)
        rec = self._rec if (self.use_graphs and self._rec is not None and self._rec["key"] == key) else None
        if rec is not None:
            rec["coords"].copy_(coords)
            rec["e_ref"].copy_(e_ref_t)
            rec["f_ref"].copy_(f_ref_t)
            rec["graph"].replay()
            small = rec["out"][0].cpu().numpy()
            if not self._overflowed(small):
                return self._unpack(small, rec["out"][1], rec["layout"], rec["ws"])
            self._rec = None  # lists too short for these positions: rebuild eagerly
        # eager pass: sizes the lists (regrowing on overflow) and checks them
        pot.energy_and_forces(coords, species, natoms, cells)
        layout, g, ws = next(iter(pot._cache.values()))
        out = self._outputs()
        self._device_pass(layout, g, ws, coords, e_ref_t, f_ref_t, out)
        small = out[0].cpu().numpy()
        if self._overflowed(small):
            raise RuntimeError("neighbour or angular capacity exceeded during the gradient pass")
        result = self._unpack(small, out[1], layout, ws)
        if self.use_graphs and self._seen == key:
            self._capture(key, layout, g, ws, coords, e_ref_t, f_ref_t)
        self._seen = key
        return result

    def _outputs(self):
        """(status words + the two loss terms in float64, flat gradient in the sweep's dtype)."""
        dev = self.pot.device
        return (torch.empty(_lib.STATUS_WORDS + 2, dtype=torch.float64, device=dev),
                torch.empty(sum(int(np.prod(s_)) for s_ in self.shapes), dtype=self.dtype, device=dev))

    def _capture(self, key, layout, g, ws, coords, e_ref, f_ref):
        rec = {"key": key, "layout": layout, "ws": ws, "coords": coords.clone(), "e_ref": e_ref.clone(),
               "f_ref": f_ref.clone(), "out": self._outputs()}
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self._device_pass(layout, g, ws, rec["coords"], rec["e_ref"], rec["f_ref"], rec["out"])
        rec["graph"] = graph
        self._rec = rec

    @staticmethod
    def _overflowed(host: np.ndarray) -> bool:
        st = host[:_lib.STATUS_WORDS]
        return bool(st[_lib.ST_NBR_OVERFLOW] or st[_lib.ST_FILTER_OVERFLOW] or st[_lib.ST_ANG_OVERFLOW])

    def _unpack(self, small: np.ndarray, grad_dev: torch.Tensor, layout, ws):
        """Loss terms and the gradient as views into one host copy of the flat
        device gradient (float64 arrays for float64 sweeps, else float32)."""
        l_e, l_f = float(small[_lib.STATUS_WORDS]), float(small[_lib.STATUS_WORDS + 1])
        # one copy into a pinned buffer; the arrays returned are copies of it
        if getattr(self, "_host", None) is None or self._host.shape != grad_dev.shape or \
                self._host.dtype != grad_dev.dtype:
            self._host = torch.empty(grad_dev.shape, dtype=grad_dev.dtype, pin_memory=True)
        self._host.copy_(grad_dev)
        host = self._host.numpy().copy()
        grads: Dict[str, List[Tuple[np.ndarray, np.ndarray]]] = {}
        pos, i = 0, 0
        for sym in self.pot.aev_cfg.species_order:
            layers = []
            for _ in self.layers[sym]:
                arrs = []
                for _k in range(2):
                    size = int(np.prod(self.shapes[i]))
                    arrs.append(host[pos:pos + size].reshape(self.shapes[i]))
                    pos += size
                    i += 1
                layers.append(tuple(arrs))
            grads[sym] = layers
        terms = LossTerms(l_e + l_f, l_e, l_f, ws.energy.cpu().numpy(), ws.forces[:layout.n].cpu().numpy())
        return terms, grads


def flatten(grads: Dict[str, List[Tuple[np.ndarray, np.ndarray]]], species_order) -> np.ndarray:
    """Concatenate a gradient (or weight) dictionary in a fixed order."""
    parts = []
    for sym in species_order:
        for W, b in grads[sym]:
            parts.append(np.asarray(W).ravel())
            parts.append(np.asarray(b).ravel())
    return np.concatenate(parts)
