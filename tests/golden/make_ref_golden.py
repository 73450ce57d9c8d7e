"""Golden pair sets, angular sub-graphs and triplets produced by the
reference's own host graph builders (thomasple/FeNNol).

``GraphGenerator.__call__`` (``src/fennol/models/preprocessing.py:74-355``),
``GraphFilter.__call__`` (``:834-894``) and ``GraphAngularExtension.__call__``
(``:1085-1181``) are plain numpy.  The module they live in also imports jax,
flax, numba and ase at module level, none of which is installed here; this
script gives those names stand-ins (a jit or njit decorator returns the
function unchanged, ``flax.linen.Module`` is a plain class, ``FrozenDict`` a
dict) and loads ``preprocessing.py`` from the reference checkout without
running the package's ``__init__`` files, so every line that builds a graph
below is the reference's own code.  Its outputs go to ``ref_<case>.npz``:

* ``p1, p2, shift``: the half pair list (p1 < p2, periodic shift of p2) of the
  radial graph, sorted by (p1, p2, shift);
* ``a_src, a_dst, a_shift``: the directed angular sub-graph (GraphFilter at
  3.5 A, shifts taken from the parent graph through ``filter_indices``), sorted;
* ``t_c, t_j, t_sj, t_k, t_sk``: the triplets (centre, the two neighbours with
  their shifts, the pair ordered), sorted -- small cases only; every case
  keeps ``t_count`` (triplets per centre atom);
* for the skin case, ``skin_p1, skin_p2, skin_shift``: the cutoff + skin list.

Cells are passed in float64 and the reciprocal cells are left to the
reference's convention (the inverse of the float64 cell, cast to float32 in
the builder).  Run in a checkout with the reference next to it:

    python tests/golden/make_ref_golden.py [path/to/FeNNol/src]
"""

from __future__ import annotations

import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from fennol_b200.systems import molecule_batch, water_box  # noqa: E402

ANGULAR_CUTOFF = 3.5
RADIAL_CUTOFF = 5.2
# the boundary geometry of tests/test_gpu_graph.py: 6 bins of 5.2 A, atoms on
# bin faces, at exactly 5.2f and one float32 ulp beyond, at the box edge
BOUNDARY_L = 31.2


class _Placeholder:
    """Stand-in for any attribute of a missing module.  Called with a single
    function (a decorator use such as ``jax.jit(f)`` or ``numba.njit(f)``) it
    returns that function; otherwise another placeholder (a decorator factory
    such as ``numba.njit(cache=True)``)."""

    def __init__(self, name: str):
        self._name = name

    def __getattr__(self, k):
        if k.startswith("__") and k.endswith("__"):
            raise AttributeError(k)
        return _Placeholder(f"{self._name}.{k}")

    def __call__(self, *args, **kwargs):
        if len(args) == 1 and callable(args[0]) and not isinstance(args[0], _Placeholder):
            return args[0]
        return _Placeholder(self._name + "()")

    def __getitem__(self, k):
        return _Placeholder(self._name + "[]")

    def __iter__(self):
        return iter(())

    def __mro_entries__(self, bases):
        return (object,)


class FrozenDict(dict):
    """``flax.core.frozen_dict.FrozenDict`` as a plain dict."""


class _Module(types.ModuleType):
    def __init__(self, name):
        super().__init__(name)
        self.__path__ = []

    def __getattr__(self, k):
        if k.startswith("__") and k.endswith("__"):
            raise AttributeError(k)
        if k == "Module":
            return type("Module", (), {})
        if k == "FrozenDict":
            return FrozenDict
        return _Placeholder(f"{self.__name__}.{k}")


class _MissingModules:
    """Meta-path finder that supplies the packages absent from this image."""

    roots = ("jax", "jaxlib", "flax", "numba", "ase", "optax")

    def find_spec(self, name, path, target=None):
        if name.split(".")[0] in self.roots:
            return importlib.util.spec_from_loader(name, self)
        return None

    def create_module(self, spec):
        return _Module(spec.name)

    def exec_module(self, module):
        pass


def load_reference_preprocessing(src: str):
    sys.dont_write_bytecode = True
    sys.meta_path.insert(0, _MissingModules())
    for pkg, sub in (("fennol", "fennol"), ("fennol.models", "fennol/models")):
        m = types.ModuleType(pkg)
        m.__path__ = [os.path.join(src, sub)]
        sys.modules[pkg] = m
    import fennol.models.preprocessing as pp  # noqa: E402
    return pp


def _sorted_rows(*cols):
    if cols[0].size == 0:
        return cols
    keys = []
    for c in reversed(cols):
        c2 = c.reshape(c.shape[0], -1)
        keys.extend(c2[:, k] for k in reversed(range(c2.shape[1])))
    o = np.lexsort(keys)
    return tuple(c[o] for c in cols)


def run_reference(pp, coordinates, species, natoms, cells=None, minimum_image=True, skin=0.0):
    """The reference's GraphGenerator -> GraphFilter -> GraphAngularExtension
    on one batch; returns the canonical arrays described above."""
    natoms = np.asarray(natoms, dtype=np.int32)
    inputs = {"coordinates": np.asarray(coordinates, dtype=np.float64),
              "species": np.asarray(species, dtype=np.int32), "natoms": natoms,
              "batch_index": np.repeat(np.arange(natoms.shape[0], dtype=np.int32), natoms)}
    if cells is not None:
        cells = np.asarray(cells, dtype=np.float64).reshape(-1, 3, 3)
        inputs["cells"] = cells
        inputs["reciprocal_cells"] = np.linalg.inv(cells)
        inputs["flags"] = {"minimum_image": None} if minimum_image else {}
    gen = pp.GraphGenerator(cutoff=RADIAL_CUTOFF)
    state = dict(gen.init())
    if skin > 0:
        state["nblist_skin"] = skin
    state, out = gen(state, inputs)
    g = out["graph"]
    nat = int(natoms.sum())
    half = g["edge_src"].shape[0] // 2
    src, dst = g["edge_src"][:half], g["edge_dst"][:half]
    ok = src < nat
    sh = (np.asarray(g["pbc_shifts"])[:half] if g.get("pbc_shifts") is not None
          else np.zeros((half, 3)))
    p1, p2, shift = _sorted_rows(src[ok].astype(np.int32), dst[ok].astype(np.int32),
                                 np.rint(sh[ok]).astype(np.int8))
    res = {"p1": p1, "p2": p2, "shift": shift}
    if skin > 0:
        ss, sd = g["edge_src_skin"], g["edge_dst_skin"]
        ok = ss < nat
        shs = (np.asarray(g["pbc_shifts_skin"]) if cells is not None else np.zeros((ss.shape[0], 3)))
        a, b, c = _sorted_rows(ss[ok].astype(np.int32), sd[ok].astype(np.int32), np.rint(shs[ok]).astype(np.int8))
        res.update(skin_p1=a, skin_p2=b, skin_shift=c)
    # angular sub-graph and triplets
    filt = pp.GraphFilter(cutoff=ANGULAR_CUTOFF, parent_graph="graph", graph_key="graph_angle")
    _, out = filt(dict(filt.init()), out)
    ga = out["graph_angle"]
    fi = ga["filter_indices"]
    nedge_parent = g["edge_src"].shape[0]
    valid = fi < nedge_parent
    full_sh = (np.concatenate([sh, -sh]) if cells is not None else np.zeros((nedge_parent, 3)))
    a_src = ga["edge_src"][valid].astype(np.int32)
    a_dst = ga["edge_dst"][valid].astype(np.int32)
    a_shift = np.rint(full_sh[fi[valid]]).astype(np.int8)
    ang = pp.GraphAngularExtension(graph_key="graph_angle")
    _, out = ang(dict(ang.init()), out)
    gt = out["graph_angle"]
    na = ga["edge_src"].shape[0]
    t_ok = gt["angle_src"] < na
    js, ks = gt["angle_src"][t_ok], gt["angle_dst"][t_ok]
    cen = gt["central_atom"][t_ok].astype(np.int32)
    e_dst = ga["edge_dst"]
    e_sh = np.zeros((na, 3), np.int8)
    e_sh[valid] = a_shift
    tj, tk = e_dst[js].astype(np.int32), e_dst[ks].astype(np.int32)
    sj, sk = e_sh[js], e_sh[ks]
    # order the unordered pair (j, sj) <= (k, sk)
    kj = np.column_stack([tj, sj.astype(np.int32)])
    kk = np.column_stack([tk, sk.astype(np.int32)])
    swap = np.zeros(kj.shape[0], bool)
    for c in range(4):
        undecided = ~swap & np.all(kj[:, :c] == kk[:, :c], axis=1) if c else np.ones(kj.shape[0], bool)
        swap |= undecided & (kj[:, c] > kk[:, c])
    kj[swap], kk[swap] = kk[swap].copy(), kj[swap].copy()
    res["t_count"] = np.bincount(cen, minlength=nat).astype(np.int32)
    a_src, a_dst, a_shift = _sorted_rows(a_src, a_dst, a_shift)
    res.update(a_src=a_src, a_dst=a_dst, a_shift=a_shift)
    if cen.size <= 200_000:
        t = _sorted_rows(cen, kj[:, 0], kj[:, 1:].astype(np.int8), kk[:, 0], kk[:, 1:].astype(np.int8))
        res.update(t_c=t[0], t_j=t[1], t_sj=t[2], t_k=t[3], t_sk=t[4])
    return res


def boundary_points():
    f = np.float32
    pts = []
    for k in range(6):
        base = f(k * 5.2)
        pts.append([base, 1.0, 1.0])
        pts.append([f(base + f(5.2)), 1.0, 1.0])
        pts.append([f(base + np.nextafter(f(5.2), f(10))), 3.0, 1.0])
        pts.append([base, 3.0, 1.0])
    pts.append([f(BOUNDARY_L), 7.0, 7.0])
    pts.append([f(0.0), 7.0, 7.0])
    pts.append([f(-1e-7), 12.0, 12.0])
    pts.append([f(BOUNDARY_L - 5.2), 12.0, 12.0])
    return np.array(pts, dtype=np.float64)


def cases():
    """(name, coordinates, species, natoms, cells or None, minimum_image, skin)."""
    out = []
    s = water_box(4, seed=0)
    out.append(("water64_mi", s.coordinates, s.species, [s.natoms], s.cell[None], True, 0.0))
    out.append(("water64_general", s.coordinates, s.species, [s.natoms], s.cell[None], False, 0.0))
    s = water_box(11, seed=2)
    out.append(("water4k_mi", s.coordinates, s.species, [s.natoms], s.cell[None], True, 0.0))
    mols = molecule_batch(6, seed=3)
    out.append(("molecules6", np.concatenate([m.coordinates for m in mols]),
                np.concatenate([m.species for m in mols]), [m.natoms for m in mols], None, True, 0.0))
    a, b = water_box(4, seed=11), water_box(5, seed=12)
    out.append(("two_boxes_mi", np.concatenate([a.coordinates, b.coordinates]),
                np.concatenate([a.species, b.species]), [a.natoms, b.natoms],
                np.stack([a.cell, b.cell]), True, 0.0))
    s = water_box(2, seed=13)  # 6.21 A box: images beyond the nearest are within the cutoff
    out.append(("water8_general", s.coordinates, s.species, [s.natoms], s.cell[None], False, 0.0))
    x = boundary_points()
    sp = np.full(x.shape[0], 6, dtype=np.int32)
    cell = (np.eye(3) * BOUNDARY_L)[None]
    out.append(("boundary_mi", x, sp, [x.shape[0]], cell, True, 0.0))
    out.append(("boundary_general", x, sp, [x.shape[0]], cell, False, 0.0))
    out.append(("boundary_nopbc", x, sp, [x.shape[0]], None, True, 0.0))
    s = water_box(6, seed=14)
    out.append(("water648_skin", s.coordinates, s.species, [s.natoms], s.cell[None], True, 1.0))
    return out


def main(src: str):
    pp = load_reference_preprocessing(src)
    for name, x, sp, nat, cells, mi, skin in cases():
        res = run_reference(pp, x, sp, nat, cells, mi, skin)
        meta = dict(coordinates=np.asarray(x, np.float64), species=np.asarray(sp, np.int32),
                    natoms=np.asarray(nat, np.int32), minimum_image=np.bool_(mi), skin=np.float64(skin))
        if cells is not None:
            meta["cells"] = np.asarray(cells, np.float64)
        np.savez_compressed(HERE / f"ref_{name}.npz", **meta, **res)
        print(f"{name}: {len(res['p1'])} pairs, {len(res['a_src'])} angular edges, "
              f"{int(res['t_count'].sum())} triplets")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")
