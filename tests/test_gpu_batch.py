"""The uneven-batch form on the GPU (no counterpart in the reference, which
solves one body per run): hbx_create_batch packs independent H-matrices of
different sizes as one block-diagonal engine, hbx_matvec multiplies all of
them in one persistent launch, and hbx_bicgstab_batch runs BiCGSTAB on every
instance with its own scalars and convergence mask.  Parity: each instance's
product against the FP64 oracle (1e-13); each instance's solve reaches the
tolerance in the FP64 residual recomputed by the oracle, in a step count
within 3 of the oracle's restated solve of that instance alone.  (The packed
layout of the batch assigns panels to warps in another order than the
instance packed alone, so the products differ in the last bits and
BiCGSTAB can cross 1e-8 a step or two apart; measured differences are
printed.)"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _instances(count=6, max_level=3):
    from hacapk_b200 import configs
    return configs.c5(count=count, seed=5, max_level=max_level)


def test_batch_matvec_is_block_diagonal(gpu, build_libs):
    import oracle
    from hacapk_b200.engine import Engine
    inst = _instances(6, 3)
    Hs = [H for H, _ in inst]
    E = Engine.batch(Hs)
    assert E.info["instances"] == len(Hs)
    x = np.random.default_rng(1).standard_normal(E.nd)
    y, _, _ = E.matvec_host(x)
    off = E.offsets
    for k, H in enumerate(Hs):
        ref = oracle.matvec(H.st, x[off[k]:off[k + 1]])
        assert np.abs(y[off[k]:off[k + 1]] - ref).max() <= 1e-13 * np.abs(ref).max()


def test_batch_solve_matches_single_solves(gpu, build_libs):
    import oracle
    from hacapk_b200.engine import Engine
    inst = _instances(8, 4)
    Hs = [H for H, _ in inst]
    E = Engine.batch(Hs)
    b = np.concatenate([bk for _, bk in inst])
    u, infos = E.bicgstab_batch_host(b, tol=1e-8, max_iter=500)
    off = E.offsets
    diffs = []
    for k, (H, bk) in enumerate(inst):
        _, n_ref, _, _ = oracle.bicgstab(H.st, bk, tol=1e-8, max_iter=500, kind="restated")
        assert infos[k]["status"] == 0, (k, infos[k])
        diffs.append(infos[k]["iterations"] - n_ref)
        assert abs(diffs[-1]) <= 3, (k, infos[k]["iterations"], n_ref)
        uk = u[off[k]:off[k + 1]]
        rel = np.linalg.norm(bk - oracle.matvec(H.st, uk)) / np.linalg.norm(bk)
        assert rel < 1.05e-8, (k, rel)
        assert abs(rel - infos[k]["true_relres"]) <= 1e-3 * rel + 1e-16
    print(f"batch of {len(inst)}: steps minus the oracle's per instance {diffs}")


def test_batch_masks_converged_instances(gpu, build_libs):
    """An instance whose rhs is zero is converged before the first step: its
    u stays zero while the others iterate."""
    from hacapk_b200.engine import Engine
    inst = _instances(4, 3)
    E = Engine.batch([H for H, _ in inst])
    bs = [bk.copy() for _, bk in inst]
    bs[2][:] = 0.0
    u, infos = E.bicgstab_batch_host(np.concatenate(bs), tol=1e-8)
    off = E.offsets
    assert infos[2]["iterations"] == 0 and np.all(u[off[2]:off[3]] == 0.0)
    assert all(i["status"] == 0 for i in infos)
    assert min(i["iterations"] for k, i in enumerate(infos) if k != 2) > 0


def test_skipping_finished_instances_changes_no_bit(gpu, build_libs, monkeypatch):
    """Inside the batched steps the products stream only the chunks of
    instances still running (a per-CTA chunk -> instance-range table built at
    hbx_create_batch, prefix counts of the active flags before each product).
    The running instances' arithmetic is untouched, so the solve equals the
    one that streams every chunk (HBX_STREAM_ALL=1) bit for bit, in every
    instance's steps and solution."""
    from hacapk_b200.engine import Engine
    inst = _instances(24, 4)
    E = Engine.batch([H for H, _ in inst])
    b = np.concatenate([bk for _, bk in inst])
    u1, i1 = E.bicgstab_batch_host(b, tol=1e-8, max_iter=400)
    monkeypatch.setenv("HBX_STREAM_ALL", "1")
    u2, i2 = E.bicgstab_batch_host(b, tol=1e-8, max_iter=400)
    monkeypatch.delenv("HBX_STREAM_ALL")
    assert [i["iterations"] for i in i1] == [i["iterations"] for i in i2]
    assert len(set(i["iterations"] for i in i1)) > 3  # instances finish at different steps
    assert np.array_equal(u1, u2)
    assert all(i["status"] == 0 and i["true_relres"] < 1.05e-8 for i in i1)


@pytest.mark.parametrize("precision,inner_tol", [(1, 0.0), (2, 1e-2)])
def test_refined_batch_meets_the_fp64_tolerance(gpu, build_libs, precision, inner_tol):
    """The mixed-precision batched solve (FP32 or BF16 factors for the
    corrections, FP64 residuals): every instance reaches 1e-8 in the FP64
    residual recomputed by the oracle, in a few refinement steps."""
    import oracle
    from hacapk_b200.engine import Engine
    inst = _instances(16, 4)
    Hs = [H for H, _ in inst]
    E = Engine.batch(Hs)
    El = Engine.batch(Hs, precision=precision)
    b = np.concatenate([bk for _, bk in inst])
    u, infos = E.bicgstab_batch_refined_host(El, b, tol=1e-8, max_iter=1000, inner_tol=inner_tol)
    off = E.offsets
    for k, (H, bk) in enumerate(inst):
        uk = u[off[k]:off[k + 1]]
        rel = np.linalg.norm(bk - oracle.matvec(H.st, uk)) / np.linalg.norm(bk)
        assert infos[k]["status"] == 0 and rel < 1.05e-8, (k, infos[k], rel)
        assert infos[k]["true_relres"] == pytest.approx(rel, rel=1e-3, abs=1e-12)
        assert 1 <= infos[k]["outer"] <= 8
