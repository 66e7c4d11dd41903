"""Every spin-wait in the device code is bounded: when the flag it waits on is
never set, the kernel gives up after its limit, reports an error status the
host reads, and the context stays usable. luc_debug_waits makes the next
call wait on a flag nothing sets (a sort tile that never runs; an mbarrier
nothing commits to) with a short limit; nothing faults, traps or hangs, and
no tensor-core work is left in flight (the hook issues no MMA at all).
"""
import numpy as np
import pytest

import oracle as O
import lucida_b200 as lb
from lucida_b200.native import LUC_DEBUG_SORT_ORPHAN_TILE, LUC_DEBUG_TC_NO_COMMIT, check, lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


@pytest.mark.parametrize("n", [4097, 1 << 20])
def test_sort_lookback_wait_runs_out(gpu, n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    b = lb.LbvhBuilder(gpu)
    check(gpu.handle, lib().luc_debug_waits(gpu.handle, LUC_DEBUG_SORT_ORPHAN_TILE, 4096))
    with pytest.raises(lb.GpuError) as e:
        b.sort(keys, vals)
    assert e.value.kind == "Validation" and "look-back wait gave up" in str(e.value)
    # The hook was one-shot and the context is intact: the next sort is right.
    ko, vo = b.sort(keys, vals)
    rk, rv = O.sort_pairs(keys, vals)
    assert np.array_equal(ko, rk) and np.array_equal(vo, rv)


def test_tensor_core_wait_runs_out(gpu):
    from lucida_b200 import Guide
    rng = np.random.default_rng(5)
    n = 3000
    x = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3)).astype(np.float32)
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    guide = Guide(gpu, seed=3, lo=(-5, -5, -5), hi=(5, 5, 5))
    ref = guide.forward(x, nrm, wo)
    check(gpu.handle, lib().luc_debug_waits(gpu.handle, LUC_DEBUG_TC_NO_COMMIT, 1024))
    with pytest.raises(lb.GpuError) as e:
        guide.forward(x, nrm, wo)
    assert "tensor-core wait ran out" in str(e.value)
    # TMEM was freed and the next launch allocates it again: same outputs.
    assert np.array_equal(guide.forward(x, nrm, wo), ref)
    # and a guided render (tcgen05 inference per bounce) still runs clean.
    from lucida_b200 import scenes
    s = scenes.cornell_analytic()
    acc = lb.render_accum(gpu, s, lb.RenderParams(width=32, height=32, samples=2, max_depth=4), guided=True)
    assert np.all(np.isfinite(acc["radiance"]))
    assert guide.stats().tc_error == 0


def test_unknown_debug_mode_is_rejected(gpu):
    assert lib().luc_debug_waits(gpu.handle, 99, 1) == -4
