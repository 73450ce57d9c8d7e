"""Index arithmetic the kernels rely on, checked on the CPU.

* ``k_energy_sum`` (csrc/reduce_md.cu) puts chunk c of system b into slot
  b + floor(start_b / 1024) + c, with max(1, ceil(n_b / 1024)) chunks per
  system, and sizes its partial array as natoms // 1024 + nsys + 1 slots:
  the slots must be distinct and inside that bound for any batch.
* ``div_small`` (csrc/aev.cu) forms q = floor(v / n) from a float32
  reciprocal, (v + 1/2) * float32(1/n), for the triplet indices of the
  adjoint (v < 256 * 256 + 256 * 2, n <= 256, the largest angular staging);
  it must be exact there without its correction step (which stays in the
  kernel as a guard).
"""

import numpy as np
import pytest

CHUNK = 1024


def slots_of(sys_start):
    out = []
    for b in range(len(sys_start) - 1):
        n = sys_start[b + 1] - sys_start[b]
        base = b + sys_start[b] // CHUNK
        for c in range(max(1, -(-n // CHUNK))):
            out.append(base + c)
    return out


@pytest.mark.parametrize("seed", range(20))
def test_energy_slots_distinct_and_bounded(seed):
    rng = np.random.default_rng(seed)
    nsys = int(rng.integers(1, 60))
    # sizes from empty to several chunks, with chunk-boundary cases mixed in
    sizes = rng.choice([0, 1, 7, 1023, 1024, 1025, 2048, 3000, 5000], size=nsys)
    sizes = np.where(rng.random(nsys) < 0.5, rng.integers(0, 4000, nsys), sizes)
    start = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    slots = slots_of(start)
    natoms = int(start[-1])
    assert len(set(slots)) == len(slots)
    assert max(slots) < natoms // CHUNK + nsys + 1


def test_energy_slots_single_large_system():
    start = np.array([0, 98_304])
    assert slots_of(start) == list(range(96))


def test_div_small_exact_without_correction():
    n = np.arange(1, 257, dtype=np.int64)
    rn = (np.float32(1.0) / n.astype(np.float32)).astype(np.float32)
    v = np.arange(0, 256 * 256 + 2 * 256, dtype=np.int64)
    for k in range(n.size):
        q = ((v.astype(np.float32) + np.float32(0.5)) * rn[k]).astype(np.int64)  # float32 product, truncation
        np.testing.assert_array_equal(q, v // n[k])
