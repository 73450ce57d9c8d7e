"""CPU oracle for the ANI-2x energy/force path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker (or the timed
CPU baseline), never as part of the product path.

What it restates (reference paths are within thomasple/FeNNol):

* :mod:`oracle.graph_fp32` -- the numpy host graph builder
  ``GraphGenerator.__call__`` (``src/fennol/models/preprocessing.py:74-355``),
  ``GraphFilter.__call__`` (``:834-894``) and
  ``GraphAngularExtension.__call__`` (``:1085-1181``), in the same float32
  numpy arithmetic, so its pair sets are the reference's pair sets bit for bit.
* :mod:`oracle.ani_ref` -- the graph processors (``preprocessing.py:719-777,
  979-1043, 1294-1317``), ``SwitchFunction`` (``misc/misc.py:617-716``),
  ``ANIAEV`` (``embeddings/ani.py:47-142``), ``SpeciesIndexNet`` /
  ``FullyConnectedNet`` (``misc/nets.py:13-102, 301-426``) and the energy sum
  (``fennix.py:218-258``) written with torch CPU tensors in float64 (or
  float32); forces come from ``torch.autograd`` exactly as the reference takes
  them from ``jax.grad`` (``fennix.py:260-272``).
* :mod:`oracle.md_ref` -- the velocity-Verlet/BAOAB step
  (``src/fennol/md/integrate.py:286-294``, ``md/thermostats.py:56-120, 172-190``).

PARITY UNPINNED: the reference ships no golden vectors or known-answer tests
for this path (its tests cover electric field, polarisation and the unit
parser), and the reference itself (JAX/Flax) cannot be imported here.  The
oracle is therefore checked against finite differences, symmetry/invariance
properties and the fixtures under ``tests/golden`` that it generated itself;
the pair set follows the reference's own numpy calls and is exact.
"""
