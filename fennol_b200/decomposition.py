"""Spatial decomposition of one large periodic box over several GPUs.

FeNNol evaluates a system on one device (``md/dynamic.py:116``); a box too
large for one GPU is cut here into P slabs along x, one per rank:

* rank r owns the atoms whose wrapped x lies in [r w, (r + 1) w), w = L_x / P;
* it also holds ghost copies of the atoms within ``halo`` (at least the
  radial cutoff, plus the skin for MD lists) of its slab's two faces, shifted
  across the periodic boundary where needed, in a local cell that is the
  slab plus both halos plus one more halo of empty space along x (so no
  periodic image along x comes within the cutoff) and the box itself along
  y and z;
* it evaluates the potential for owned + ghost atoms with only the owned
  atoms as centres (``ANIPotential.energy_and_forces(..., centres=n_owned)``
  clears the ghost centres' energies and dE/dAEV before the sum and the
  adjoint), so its energy is the sum of its owned atomic energies and its
  forces are -d/dx of that sum on owned and ghost atoms;
* the exchange step is a halo exchange: every rank sends the forces that
  landed on its ghosts to the ranks that own them (point-to-point messages
  over ``torch.distributed``: NCCL on GPUs, gloo on CPUs), so each rank
  ends with the complete forces of its owned atoms; message sizes follow
  from the plan, which every rank can evaluate for every other rank, so no
  size exchange is needed.  The energy is a one-element all-reduce.  The
  traffic per rank is the halo (a few atom layers), not the box.

Positions stay replicated on every rank (N x 3 floats: 24 MB for 10^6
atoms); the neighbour lists, AEVs, MLP and adjoint, which carry the memory
and the time, are split.  The slab width must be at least the halo, and the
cell orthorhombic.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np
import torch


@dataclass
class LocalSystem:
    ids: np.ndarray        # global atom index of each local atom: owned first, then ghosts
    coordinates: np.ndarray  # [m, 3] float64, in the local cell
    n_owned: int
    cell: np.ndarray       # [3, 3] local cell (rows are lattice vectors)


class SlabPlan:
    """Cut an orthorhombic box into ``n_ranks`` slabs along x."""

    def __init__(self, cell, n_ranks: int, halo: float):
        cell = np.asarray(cell, dtype=np.float64).reshape(3, 3)
        if np.abs(cell - np.diag(np.diag(cell))).max() > 0:
            raise ValueError("slab decomposition needs an orthorhombic cell")
        if n_ranks < 1:
            raise ValueError("n_ranks must be >= 1")
        self.cell = cell
        self.lengths = np.diag(cell).copy()
        self.n_ranks = int(n_ranks)
        self.halo = float(halo)
        self.width = self.lengths[0] / self.n_ranks
        if self.n_ranks > 1 and self.width < self.halo:
            raise ValueError(f"slab width {self.width:.3f} A is below the halo {self.halo:.3f} A: "
                             "use fewer ranks")

    def wrapped_x(self, coordinates) -> np.ndarray:
        """x wrapped once into [0, L_x) (np.mod of a tiny negative x can round
        to L_x itself; that value is mapped to 0)."""
        lx = self.lengths[0]
        xw = np.mod(np.asarray(coordinates, dtype=np.float64)[:, 0], lx)
        xw[xw >= lx] = 0.0
        return xw

    def owners(self, coordinates) -> np.ndarray:
        """Owning rank of every atom: floor(x_wrapped / w), clamped to the last rank."""
        return np.minimum((self.wrapped_x(coordinates) / self.width).astype(np.int64), self.n_ranks - 1)

    def local(self, coordinates, rank: int) -> LocalSystem:
        """The atoms rank ``rank`` evaluates and where they sit in its cell.

        Ownership is decided by :meth:`owners` alone, so every atom is owned by
        exactly one rank; ghosts are chosen only among the atoms other ranks
        own, so no atom is both owned and a ghost on one rank (which would put
        a pair at zero distance).  Near a face, rounding may call an atom of
        the rank below an "above" ghost at offset ~0 (or the reverse): both
        place it at the face, within rounding."""
        x = np.asarray(coordinates, dtype=np.float64)
        n = x.shape[0]
        if self.n_ranks == 1:
            return LocalSystem(np.arange(n), x.copy(), n, self.cell.copy())
        lx, w, h = self.lengths[0], self.width, self.halo
        xw = self.wrapped_x(x)
        own = self.owners(x)
        # offset from the slab's lower face: owned atoms as is (a rounding
        # residue may make it a tiny negative), others wrapped into [0, L_x]
        d = xw - rank * w
        u = np.where(d < 0.0, d + lx, d)
        other = own != rank
        owned = np.nonzero(~other)[0]
        above = np.nonzero(other & (u < w + h))[0]             # beyond the upper face
        below = np.nonzero(other & (u >= lx - h))[0]           # beyond the lower face (shifted by -L_x)
        ids = np.concatenate([owned, above, below])
        ux = np.concatenate([d[owned], u[above], u[below] - lx]) + h
        yz = np.mod(x[ids, 1:], self.lengths[1:])
        local_x = np.concatenate([ux[:, None], yz], axis=1)
        cell = np.diag([w + 3.0 * h, self.lengths[1], self.lengths[2]])
        return LocalSystem(ids, local_x, owned.size, cell)


def rank_contribution(pot, plan: SlabPlan, rank: int, coordinates, species) -> Tuple[torch.Tensor, torch.Tensor]:
    """Energy of the owned atoms of ``rank`` (float64 scalar) and its forces
    on all atoms (float64 [N, 3], zero away from its owned and ghost atoms),
    both on the potential's device.  Summed over the ranks they are the energy
    and forces of the whole box."""
    loc = plan.local(coordinates, rank)
    sp = np.asarray(species)[loc.ids]
    e, f = pot.energy_and_forces(loc.coordinates, sp, [loc.ids.size], loc.cell[None], centres=loc.n_owned)
    n = np.asarray(coordinates).shape[0]
    forces = torch.zeros((n, 3), dtype=torch.float64, device=f.device)
    forces.index_add_(0, torch.as_tensor(loc.ids, device=f.device), f.to(torch.float64))
    return e.to(torch.float64).sum(), forces


def ghost_routes(plan: SlabPlan, coordinates, rank: int):
    """For rank ``rank``: ``send[q]`` = positions (in its local atom list) of
    the ghosts that rank q owns, and ``recv[q]`` = global ids of rank q's
    ghosts that ``rank`` owns, in the order rank q sends them.  Both come from
    the replicated positions, so sender and receiver agree without a message."""
    own = plan.owners(coordinates)
    loc = plan.local(coordinates, rank)
    ghost_owner = own[loc.ids[loc.n_owned:]]
    send = {}
    for q in range(plan.n_ranks):
        if q == rank:
            continue
        pos = loc.n_owned + np.nonzero(ghost_owner == q)[0]
        if pos.size:
            send[q] = pos
    recv = {}
    for q in range(plan.n_ranks):
        if q == rank:
            continue
        lq = plan.local(coordinates, q)
        g = lq.ids[lq.n_owned:]
        mine = g[own[g] == rank]
        if mine.size:
            recv[q] = mine
    return loc, send, recv


class SlabEnergyForces:
    """Energy and forces of one periodic box evaluated by all ranks of a
    process group, each on its slab.

    A call returns the total energy (every rank) and the forces of the
    atoms this rank owns, as an [N, 3] float64 array that is zero on the
    other atoms (``owned_ids()`` lists them): the ghost forces reach their
    owners through one halo exchange of point-to-point messages."""

    def __init__(self, pot, cell, halo: Optional[float] = None, group=None):
        import torch.distributed as dist

        self.pot, self.group = pot, group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.plan = SlabPlan(cell, self.world, pot.aev_cfg.radial_cutoff if halo is None else halo)
        self.last_exchange_rows = 0

    def owned_ids(self, coordinates) -> np.ndarray:
        return np.nonzero(self.plan.owners(coordinates) == self.rank)[0]

    def __call__(self, coordinates, species) -> Tuple[torch.Tensor, torch.Tensor]:
        import torch.distributed as dist

        x = np.asarray(coordinates, dtype=np.float64)
        n = x.shape[0]
        loc, send, recv = ghost_routes(self.plan, x, self.rank)
        sp = np.asarray(species)[loc.ids]
        e, f_loc = self.pot.energy_and_forces(loc.coordinates, sp, [loc.ids.size], loc.cell[None],
                                              centres=loc.n_owned)
        f_loc = f_loc.to(torch.float64)
        dev = f_loc.device
        e = e.to(torch.float64).sum().reshape(1)
        forces = torch.zeros((n, 3), dtype=torch.float64, device=dev)
        forces.index_add_(0, torch.as_tensor(loc.ids[:loc.n_owned], device=dev), f_loc[:loc.n_owned])
        if self.world > 1:
            ops, bufs = [], {}
            for q, pos in send.items():
                ops.append(dist.P2POp(dist.isend, f_loc[torch.as_tensor(pos, device=dev)].contiguous(), q,
                                      group=self.group))
            for q, ids in recv.items():
                bufs[q] = torch.empty((ids.size, 3), dtype=torch.float64, device=dev)
                ops.append(dist.P2POp(dist.irecv, bufs[q], q, group=self.group))
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()
            for q, ids in recv.items():
                forces.index_add_(0, torch.as_tensor(ids, device=dev), bufs[q])
            self.last_exchange_rows = int(sum(p.size for p in send.values()))
            dist.all_reduce(e, group=self.group)
        return e[0], forces
