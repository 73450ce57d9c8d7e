"""A small energy+force workload to run under a profiler.

    python -m fennol_b200.profile_case [--n-side 16] [--precision f16x3x1] [--models 1] [--calls 3]

Builds the seeded water box with ``n_side**3`` molecules (12,288 atoms for
16), an ANI-2x-style potential with seeded random weights (rounded to BF16
for the BF16 forms), and
calls ``ANIPotential.energy_and_forces`` ``calls`` times: each call launches
the neighbour search, the AEV, the species MLPs, the energy reduction and the
force adjoint once.
"""

import argparse

import torch

from .potential import ANIPotential
from .systems import water_box


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-side", type=int, default=16)
    ap.add_argument("--precision", default="f16x3x1")
    ap.add_argument("--models", type=int, default=1)
    ap.add_argument("--calls", type=int, default=3)
    args = ap.parse_args()
    dev = torch.device("cuda:0")
    box = water_box(args.n_side, seed=0)
    pot = ANIPotential(precision=args.precision, device=dev, seed=0, n_models=args.models,
                       bf16_weights=args.precision.startswith("bf16"))
    x = torch.tensor(box.coordinates, dtype=torch.float32, device=dev)
    for _ in range(args.calls):
        e, f = pot.energy_and_forces(x, box.species, [box.natoms], box.cell[None])
    torch.cuda.synchronize()
    print(f"atoms {box.natoms} models {args.models} {args.precision} "
          f"energy {float(e[0]):.6f} Ha |F|max {float(f.abs().max()):.4f} Ha/A")


if __name__ == "__main__":
    main()
