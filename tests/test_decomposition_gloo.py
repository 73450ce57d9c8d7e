"""Slab decomposition with two and three gloo ranks on CPU.

Each rank evaluates its owned + ghost atoms with the FP64 oracle (standing in
for the CUDA potential, which these CPU ranks cannot run), keeps only its
owned centres, and the halo exchange sends ghost forces to their owners.
Every rank's energy and its owned atoms' forces must equal the oracle on the
undecomposed box; together the ranks cover every atom once."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fennol_b200.decomposition import SlabEnergyForces, SlabPlan, rank_contribution
from fennol_b200.params import AEVConfig, MLPConfig, init_weights
from fennol_b200.systems import water_box
from oracle import ani_ref


class OraclePot:
    """The ANIPotential.energy_and_forces signature over the FP64 oracle,
    with ``centres`` (only the first centres atoms' energies count)."""

    def __init__(self, seed=0):
        self.aev_cfg, self.mlp_cfg = AEVConfig(), MLPConfig()
        self.weights = init_weights(self.aev_cfg, self.mlp_cfg, seed=seed)

    def energy_and_forces(self, coordinates, species, natoms=None, cells=None, want_forces=True,
                          centres=None):
        x0 = np.asarray(coordinates, dtype=np.float64)
        n = x0.shape[0]
        g = ani_ref.Graph(x0, [n], cells, None, self.aev_cfg.radial_cutoff, self.aev_cfg.angular_cutoff,
                          minimum_image=True)
        sidx = self.aev_cfg.species_index(np.asarray(species))
        x = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
        emb = ani_ref.aev(x, sidx, g, self.aev_cfg)
        eat = sum(ani_ref.species_net(emb, sidx, m, self.aev_cfg.species_order, self.mlp_cfg.celu_alpha)
                  for m in self.weights) / len(self.weights)
        k = n if centres is None else centres
        e = eat[:k].sum()
        (grad,) = torch.autograd.grad(e, x)
        return e.detach().reshape(1), (-grad).detach()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _box(faces=False, world=3):
    s = water_box(6, seed=41)  # 648 atoms, 18.6 A cube
    x = s.coordinates.copy()
    if faces:
        # oxygens moved onto the slab faces and one ulp either side of them,
        # and one to x = -1e-17 (np.mod rounds it to L_x)
        L = float(s.cell[0, 0])
        w = L / world
        shift = np.zeros(3)
        picks = [(0, -1e-17)]
        for k in range(world):
            f = k * w
            picks += [(3 + 9 * k, f), (6 + 9 * k, np.nextafter(f, -np.inf)), (9 + 9 * k, np.nextafter(f, np.inf))]
        for i, xv in picks:
            shift[:] = 0.0
            shift[0] = xv - x[i, 0]
            x[i:i + 3] += shift  # the whole molecule (O, H, H) moves with its oxygen
    return x, s.species, s.cell


def _worker(rank, world, port, faces, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        x, sp, cell = _box(faces, world)
        ef = SlabEnergyForces(OraclePot(), cell)
        e, f = ef(x, sp)
        out[rank] = (float(e), f.numpy(), ef.owned_ids(x), ef.last_exchange_rows)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,faces", [(2, False), (3, False), (3, True), (2, True)])
def test_slab_ranks_reproduce_the_whole_box(world, faces):
    x, sp, cell = _box(faces, world)
    pot = OraclePot()
    e_ref, f_ref = pot.energy_and_forces(x, sp, [len(sp)], cell[None])
    f_ref = f_ref.numpy()
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, faces, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    covered = np.zeros(len(sp), dtype=int)
    for r in range(world):
        e, f, owned, rows = res[r]
        assert abs(e - float(e_ref)) < 1e-9 * len(sp)
        np.testing.assert_allclose(f[owned], f_ref[owned], atol=1e-9, rtol=0)
        mask = np.ones(len(sp), dtype=bool)
        mask[owned] = False
        assert not f[mask].any()          # only owned atoms carry forces on this rank
        covered[owned] += 1
        assert 0 < rows < len(sp)          # the ghost rows (both halos), not the box
    assert (covered == 1).all()


def test_plan_owns_every_atom_once_and_ghosts_cover_the_halo():
    x, sp, cell = _box()
    plan = SlabPlan(cell, 3, 5.2)
    owners = plan.owners(x)
    assert set(np.unique(owners)) == {0, 1, 2}
    seen = np.zeros(len(sp), dtype=int)
    L = np.diag(np.asarray(cell).reshape(3, 3))
    for r in range(3):
        loc = plan.local(x, r)
        seen[loc.ids[:loc.n_owned]] += 1
        # every atom within 5.2 A (minimum image) of an owned atom is present locally
        own = x[loc.ids[:loc.n_owned]]
        d = x[None, :, :] - own[:, None, :]
        d -= L * np.round(d / L)
        near = np.unique(np.nonzero((d ** 2).sum(-1) < 5.2 ** 2)[1])
        assert set(near) <= set(loc.ids)
    assert (seen == 1).all()


def test_single_rank_is_the_plain_box():
    x, sp, cell = _box()
    pot = OraclePot()
    e, f = rank_contribution(pot, SlabPlan(cell, 1, 5.2), 0, x, sp)
    e_ref, f_ref = pot.energy_and_forces(x, sp, [len(sp)], cell[None])
    assert abs(float(e) - float(e_ref)) < 1e-12 * len(sp)
    np.testing.assert_allclose(f.numpy(), f_ref.numpy(), atol=1e-12)


def test_narrow_slabs_are_rejected():
    with pytest.raises(ValueError):
        SlabPlan(np.diag([18.0, 18.0, 18.0]), 4, 5.2)


def test_plan_wraps_coordinates_and_faces():
    cell = np.diag([30.0, 20.0, 20.0])
    plan = SlabPlan(cell, 3, 5.2)  # slabs of 10 A
    x = np.array([[-1.0, 0.0, 0.0],    # wraps to 29: rank 2
                  [10.0, 0.0, 0.0],    # on the 0|1 face: rank 1
                  [29.999, 5.0, -3.0],  # rank 2
                  [31.0, 25.0, 0.0],   # wraps to 1: rank 0
                  [0.0, 0.0, 0.0]])
    np.testing.assert_array_equal(plan.owners(x), [2, 1, 2, 0, 0])
    loc = plan.local(x, 0)
    owned = set(loc.ids[:loc.n_owned].tolist())
    assert owned == {3, 4}
    # rank 0's local x: owned atoms in [halo, halo + width), everything inside the local cell
    assert np.all(loc.coordinates[:loc.n_owned, 0] >= 5.2) and np.all(loc.coordinates[:loc.n_owned, 0] < 15.2)
    assert np.all(loc.coordinates[:, 0] >= 0.0) and np.all(loc.coordinates[:, 0] < loc.cell[0, 0])
    assert np.all(loc.coordinates[:, 1:] >= 0.0) and np.all(loc.coordinates[:, 1:] < 20.0)
    # atoms 0 and 2 (x = 29, 29.999) sit within the halo below rank 0's lower face
    assert {0, 2} <= set(loc.ids[loc.n_owned:].tolist())


def test_plan_rejects_triclinic_cells():
    cell = np.array([[20.0, 0.0, 0.0], [3.0, 20.0, 0.0], [0.0, 0.0, 20.0]])
    with pytest.raises(ValueError):
        SlabPlan(cell, 2, 5.2)


@pytest.mark.parametrize("world", [2, 3, 4])
def test_faces_and_ulps_owned_once_and_in_both_neighbours(world):
    """Atoms on every slab face, one ulp either side, and at x = -1e-17: each
    is owned by exactly one rank, the ranks on both sides of its face hold it
    (owned or ghost), no rank lists an atom twice at the same place, and every
    owned atom sees exactly its minimum-image neighbours at the right distance."""
    L = 24.0
    cell = np.diag([L, 13.0, 13.0])
    plan = SlabPlan(cell, world, 3.0)
    w = plan.width
    xs = [-1e-17, 0.0, np.nextafter(L, 0.0)]
    for k in range(world):
        f = k * w
        xs += [f, np.nextafter(f, -np.inf), np.nextafter(f, np.inf)]
    rng = np.random.default_rng(0)
    bulk = rng.uniform(0, 1, (200, 3)) * [L, 13.0, 13.0]
    face = np.stack([np.array(xs), rng.uniform(0, 13.0, len(xs)), rng.uniform(0, 13.0, len(xs))], 1)
    x = np.concatenate([face, bulk])
    own = plan.owners(x)
    assert own.min() >= 0 and own.max() < world
    count = np.zeros(len(x), dtype=int)
    Lv = np.diag(cell)
    for r in range(world):
        loc = plan.local(x, r)
        count[loc.ids[:loc.n_owned]] += 1
        # no two local entries of the same atom at the same place
        key = {}
        for i, gid in enumerate(loc.ids):
            for j in key.get(gid, []):
                assert np.abs(loc.coordinates[i] - loc.coordinates[j]).max() > 1.0
            key.setdefault(gid, []).append(i)
        # owned atoms see their true neighbours within the halo
        lx = loc.coordinates
        ll = np.diag(loc.cell)
        for i in range(loc.n_owned):
            d = lx - lx[i]
            d -= ll * np.round(d / ll)
            r2 = (d ** 2).sum(-1)
            near_loc = sorted((int(loc.ids[j]), round(float(r2[j]), 9)) for j in np.nonzero(r2 < 9.0)[0]
                              if j != i)
            g = x - x[loc.ids[i]]
            g -= Lv * np.round(g / Lv)
            g2 = (g ** 2).sum(-1)
            near_true = sorted((int(j), round(float(g2[j]), 9)) for j in np.nonzero(g2 < 9.0)[0]
                               if j != loc.ids[i])
            assert near_loc == near_true, (r, int(loc.ids[i]))
    assert (count == 1).all()
    # atoms on a face are held by the ranks on both sides of it
    for k in range(world):
        lower, upper = (k - 1) % world, k
        for i in range(1 + 2 + 3 * k, 1 + 2 + 3 * k + 3):
            for r in (lower, upper):
                assert i in set(plan.local(x, r).ids.tolist()), (i, r)
