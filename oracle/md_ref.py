"""Float64 restatement of FeNNol's MD step (oracle; test-only).

``integrate`` of ``src/fennol/md/integrate.py:286-294``:
``v += dt/m F; x += dt/2 v; thermostat(v); x += dt/2 v`` with NVE
(``md/thermostats.py:172-190``: no O step).  Forces from :mod:`oracle.ani_ref`
with the graph rebuilt every step (the reference's no-skin mode).
"""

from __future__ import annotations

import numpy as np

from . import ani_ref

HARTREE_TO_KCALMOL = 627.5096080305927


def nve_trajectory(x0, v0, species, natoms, mass_md, weights, aev_cfg, mlp_cfg, dt_ps, nsteps,
                   cells=None):
    """Positions after each step (list of [N,3] float64) and potential energies (kcal/mol)."""
    x = np.array(x0, dtype=np.float64)
    v = np.array(v0, dtype=np.float64)
    m = np.asarray(mass_md, dtype=np.float64)[:, None]
    r = ani_ref.energy_and_forces(x, species, natoms, weights, aev_cfg, mlp_cfg, cells=cells)
    f = r["forces"] * HARTREE_TO_KCALMOL
    xs, es = [], []
    for _ in range(nsteps):
        v = v + dt_ps * f / m
        x = x + 0.5 * dt_ps * v
        x = x + 0.5 * dt_ps * v
        r = ani_ref.energy_and_forces(x, species, natoms, weights, aev_cfg, mlp_cfg, cells=cells)
        f = r["forces"] * HARTREE_TO_KCALMOL
        xs.append(x.copy())
        es.append(float(r["energy"].sum()) * HARTREE_TO_KCALMOL)
    return xs, es, v
