"""Generate the golden fixtures of this directory from the CPU oracle.

The reference (thomasple/FeNNol) ships no golden vectors for this path and
cannot be imported here (JAX is absent), so the fixtures are produced by the
oracle restatement and pinned by the oracle's own checks (finite
differences, invariances) in ``tests/test_oracle.py``.

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from fennol_b200.params import AEVConfig, MLPConfig, init_weights  # noqa: E402
from fennol_b200.systems import molecule_batch, water_box  # noqa: E402
from oracle import ani_ref, graph_fp32  # noqa: E402

WEIGHT_SEED = 0
N_AEV_ROWS = 8


def weights_checksum(weights) -> float:
    return float(sum(np.sum(w) + np.sum(b) for m in weights for L in m.values() for w, b in L))


def water64():
    cfg, mcfg = AEVConfig(), MLPConfig()
    W = init_weights(cfg, mcfg, seed=WEIGHT_SEED)
    s = water_box(4, seed=0)
    cells = s.cell[None]
    r = ani_ref.energy_and_forces(s.coordinates, s.species, [s.natoms], W, cfg, mcfg, cells=cells,
                                  return_aev=True)
    g = r["graph"]
    gen = graph_fp32.pair_list(s.coordinates, [s.natoms], cells, None, 5.2, minimum_image=False)
    skin = graph_fp32.pair_list(s.coordinates, [s.natoms], cells, None, 6.2, minimum_image=True)
    return dict(coordinates=s.coordinates, species=s.species, cell=s.cell, weight_seed=WEIGHT_SEED,
                weight_checksum=weights_checksum(W),
                p1=g.pairs["p1"].astype(np.int32), p2=g.pairs["p2"].astype(np.int32),
                shift=g.pairs["shift"].astype(np.int8), d12=g.pairs["d12"],
                gen_p1=gen["p1"].astype(np.int32), gen_p2=gen["p2"].astype(np.int32),
                gen_shift=gen["shift"].astype(np.int8),
                skin_npairs=np.int64(len(skin["p1"])),
                n_angular_edges=np.int64(len(g.filter_indices)), n_triplets=np.int64(len(g.angle_src)),
                energy=r["energy"], forces=r["forces"], atomic_energies=r["atomic_energies"],
                aev_rows=r["aev"][:N_AEV_ROWS])


def molecules():
    cfg, mcfg = AEVConfig(), MLPConfig()
    W = init_weights(cfg, mcfg, seed=WEIGHT_SEED)
    mols = molecule_batch(6, seed=3)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    nat = np.array([m.natoms for m in mols])
    r = ani_ref.energy_and_forces(xyz, sp, nat, W, cfg, mcfg)
    g = r["graph"]
    return dict(coordinates=xyz, species=sp, natoms=nat, weight_seed=WEIGHT_SEED,
                weight_checksum=weights_checksum(W),
                p1=g.pairs["p1"].astype(np.int32), p2=g.pairs["p2"].astype(np.int32),
                energy=r["energy"], forces=r["forces"])


def main():
    np.savez_compressed(HERE / "water64.npz", **water64())
    np.savez_compressed(HERE / "molecules6.npz", **molecules())
    for f in ("water64.npz", "molecules6.npz"):
        print(f, os.path.getsize(HERE / f), "bytes")


if __name__ == "__main__":
    main()
