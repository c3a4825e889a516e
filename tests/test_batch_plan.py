"""Block sizes of the batched form (host logic, no GPU): every grid gets threads in proportion to
its cells, a multiple of 32 from 32 to the largest grid's cap, with the fewest cells per thread
for which all blocks fit in the device's thread slots, so that the blocks finish together."""
from __future__ import annotations

import numpy as np
import pytest

from diffusionimex_b200 import cases
from diffusionimex_b200.solver import SolverError, batch_block_sizes


def restated(cells, threads, slots):
    cells = np.asarray(cells, dtype=np.int64)
    nmax = int(cells.max())

    def blocks(per):
        t = (cells + 32 * per - 1) // (32 * per) * 32
        return np.minimum(np.maximum(t, 32), threads)

    per = (nmax + threads - 1) // threads
    if slots > 0:
        while per < nmax and blocks(per).sum() > slots:
            per += 1
    return blocks(per), per


def test_plan_of_the_512_riemann_problems():
    """The batched workload (cell counts uniform in [256, 4096]) on a B200's 148 SMs x 256 threads of
    the kernel, 15/16 of them: 42 cells per thread, blocks of 32 to 128 threads."""
    cells = [c["nx"] for c in cases.riemann_batch(count=512, seed=0)]
    slots = 148 * 256 * 15 // 16
    b, per = batch_block_sizes(cells, 256, slots)
    assert per == 42 and b.sum() <= slots
    sizes, counts = np.unique(b, return_counts=True)
    assert dict(zip(sizes.tolist(), counts.tolist())) == {32: 143, 64: 165, 96: 191, 128: 13}
    # without a thread limit the largest grid gets the cap
    b, per = batch_block_sizes(cells, 256, 0)
    assert per == 16 and b.max() == 256


@pytest.mark.parametrize("seed", range(6))
def test_plan_matches_its_restatement(seed):
    rng = np.random.default_rng(seed)
    cells = rng.integers(1, 20000, size=int(rng.integers(1, 700)))
    threads = int(rng.choice([32, 64, 96, 128, 256]))
    slots = int(rng.choice([0, 4096, 35520, 10 ** 6]))
    b, per = batch_block_sizes(cells, threads, slots)
    rb, rper = restated(cells, threads, slots)
    assert per == rper and np.array_equal(b, rb)
    assert np.all(b % 32 == 0) and b.min() >= 32 and b.max() <= threads


def test_equal_grids_get_the_cap():
    b, _ = batch_block_sizes([1000] * 10, 128, 0)
    assert np.all(b == 128)


@pytest.mark.parametrize("args", [([], 64, 0), ([10, 0], 64, 0), ([10], 48, 0), ([10], 512, 0), ([10], 64, -1)])
def test_bad_arguments(args):
    with pytest.raises(SolverError):
        batch_block_sizes(*args)
