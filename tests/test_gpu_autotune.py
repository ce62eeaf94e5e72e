"""The schedule autotuner (hbx_autotune; no counterpart in the reference,
whose size-class batching is fixed): it times the real kernel for a grid of
CTA schedules on the device and returns the fastest; the engine built with
those options computes the same product (FP64 oracle, 1e-13)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_returns_a_schedule_no_slower_than_the_default(gpu, build_libs):
    import oracle
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(4)
    kw, best_us, def_us = Engine.autotune(H.st, H.nd, reps=10)
    print(f"L4 FP64 autotune: {kw}, {best_us:.1f} us (default {def_us:.1f} us)")
    assert 0.0 < best_us <= def_us
    E = Engine(H.st, H.nd, **kw)
    if kw["block_cost"]:
        assert E.info["block_cost"] == kw["block_cost"]
    if kw["merge"]:
        assert E.info["merge_keep"] == (kw["merge"] - 1 if kw["merge"] > 0 else -1)
    if kw["l2_keep_mb"]:
        assert E.info["l2_keep_mb"] == max(0, kw["l2_keep_mb"])
    x = np.random.default_rng(4).standard_normal(H.nd)
    y, _, _ = E.matvec_host(x)
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()


def test_autotune_multi_rhs(gpu, build_libs):
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(4)
    kw, best_us, def_us = Engine.autotune(H.st, H.nd, precision=abi.HBX_FP32, nrhs=abi.HBX_NRHS, reps=5)
    print(f"L4 64-RHS autotune: {kw}, {best_us:.1f} us (default {def_us:.1f} us)")
    assert 0.0 < best_us <= def_us
    Engine(H.st, H.nd, precision=abi.HBX_FP32, nrhs=abi.HBX_NRHS, **kw).close()


@pytest.mark.parametrize("merge,l2", [(-1, -1), (1, 12), (9, 48)])
def test_layout_options_keep_the_product(gpu, build_libs, merge, l2):
    """The layout options the autotuner searches (merged D+U runs: merge =
    k + 1 keeps each CTA's first k atoms split, -1 none; the L2 budget of the
    stream, -1 no cache hints) change the packing and the cache policy, not
    the product: 1e-13 of the oracle, and the kernel-order replay of the same
    layout bit for bit."""
    import oracle
    from conftest import kernel_order_matvec
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(4)
    E = Engine(H.st, H.nd, merge=merge, l2_keep_mb=l2)
    mk = merge - 1 if merge > 0 else -1
    assert E.info["merge_keep"] == mk and E.info["l2_keep_mb"] == max(0, l2)
    x = np.random.default_rng(5).standard_normal(H.nd)
    y, _, _ = E.matvec_host(x)
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.array_equal(y, kernel_order_matvec(H, E.info["num_ctas"], merge_keep=mk)(x))
