"""CPU tests of the engine's host planner and packer (hbx_plan.cpp): a
test-only interpreter (tests/emu/plan_emu.cpp) walks the packed per-CTA
streams exactly as the kernel does, checks the layout invariants the kernel
relies on, and its result is compared with the oracle."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, sphere

EMU_SRC = os.path.join(ROOT, "tests", "emu", "plan_emu.cpp")
EMU_LIB = os.path.join(ROOT, "tests", "emu", "_build", "libplanemu.so")


@pytest.fixture(scope="module")
def emu(build_libs):
    os.makedirs(os.path.dirname(EMU_LIB), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", EMU_LIB, EMU_SRC,
                    os.path.join(ROOT, "hacapk-magma_b200", "csrc", "hbx_plan.cpp")], check=True)
    lib = C.CDLL(EMU_LIB)
    lib.emu_matvec.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_longlong), C.c_char_p, C.c_int]
    lib.emu_matvec_transposed.argtypes = lib.emu_matvec.argtypes
    lib.emu_matvec_prec.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_char_p, C.c_int]
    lib.emu_matvec_pairs.argtypes = lib.emu_matvec.argtypes
    lib.emu_matvec_batch.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_int, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_char_p, C.c_int]
    lib.emu_matvec_costs.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_char_p, C.c_int]
    lib.emu_matvec_merged.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_char_p, C.c_int]
    lib.emu_bf16_from_double.argtypes = [C.c_double]
    lib.emu_bf16_from_double.restype = C.c_uint
    return lib


def run_emu(lib, st_ptr, nd, nc, x, transposed=False):
    y = np.zeros(nd)
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    fn = lib.emu_matvec_transposed if transposed else lib.emu_matvec
    rc = fn(st_ptr, nd, nc, x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)),
            stats, msg, 512)
    return rc, msg.value.decode(), y, list(stats)


@pytest.mark.parametrize("level,leaf,nc", [(2, 32, 148), (3, 32, 148), (3, 32, 1), (3, 15, 7), (4, 32, 148),
                                           (4, 32, 300)])
def test_packed_layout_reproduces_oracle(emu, level, leaf, nc):
    import oracle
    H = sphere(level, leaf_size=leaf)
    x = np.random.default_rng(level * 100 + nc).standard_normal(H.nd)
    rc, msg, y, stats = run_emu(emu, C.cast(H.st, C.c_void_p), H.nd, nc, x)
    assert rc == 0, msg
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()
    d, lr = H.storage_words()
    assert stats[6] == 8 * (d + lr) + stats[7]  # every factor byte packed once, plus the zero columns
    assert stats[7] <= 0.02 * 8 * (d + lr)       # of odd-width blocks (a few percent at most)


def _fortran_like(H, stride):
    """A copy of the container whose leaves sit `stride` bytes apart (Fortran
    derived types carry pointer descriptors between the fields the C side
    reads), to check that st_lf_stride is honoured."""
    from hacapk_b200 import abi
    n = H.nlf
    buf = (C.c_char * (stride * n))()
    src = H.st.contents.st_lf
    for ip in range(n):
        C.memmove(C.addressof(buf) + ip * stride, C.addressof(src[ip]), C.sizeof(abi.LeafMtx))
    P = abi.LeafMtxP()
    C.memmove(C.byref(P), H.st, C.sizeof(abi.LeafMtxP))
    P.st_lf_stride = stride
    P.st_lf = C.cast(buf, C.POINTER(abi.LeafMtx))
    return P, buf


def test_leaf_stride_is_honoured(emu):
    import oracle
    H = sphere(3)
    P, keep = _fortran_like(H, 160)
    x = np.random.default_rng(7).standard_normal(H.nd)
    rc, msg, y, _ = run_emu(emu, C.cast(C.pointer(P), C.c_void_p), H.nd, 148, x)
    assert rc == 0, msg
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()


def _custom(leaves, nd):
    """Container over hand-made leaves: (ltmtx, kt, nstrtl, ndl, nstrtt, ndt, a1 array)."""
    from hacapk_b200 import abi
    arr = (abi.LeafMtx * max(1, len(leaves)))()
    keep = []
    for i, (lt, kt, l0, ndl, t0, ndt, data) in enumerate(leaves):
        data = np.ascontiguousarray(data, np.float64)
        keep.append(data)
        arr[i].ltmtx, arr[i].kt, arr[i].nstrtl, arr[i].ndl = lt, kt, l0, ndl
        arr[i].nstrtt, arr[i].ndt = t0, ndt
        arr[i].a1 = data.ctypes.data_as(C.POINTER(C.c_double)) if data.size else None
        arr[i].a1size = 8 * (ndt * kt if lt == 1 else ndt * ndl)
    P = abi.LeafMtxP()
    P.nd, P.nlf = nd, len(leaves)
    P.st_lf_stride = C.sizeof(abi.LeafMtx)
    P.st_lf = arr
    return P, (arr, keep)


def _dense_of(leaves, nd):
    A = np.zeros((nd, nd))
    for lt, kt, l0, ndl, t0, ndt, data in leaves:
        if lt == 2:
            A[l0 - 1:l0 - 1 + ndl, t0 - 1:t0 - 1 + ndt] += np.asarray(data).reshape(ndl, ndt)
        elif kt:
            V = np.asarray(data[:ndt * kt]).reshape(kt, ndt).T
            U = np.asarray(data[ndt * kt:]).reshape(kt, ndl).T
            A[l0 - 1:l0 - 1 + ndl, t0 - 1:t0 - 1 + ndt] += U @ V.T
    return A


def test_edge_cases(emu):
    rng = np.random.default_rng(9)
    nd = 100
    leaves = [
        (2, 0, 1, 40, 1, 100, rng.standard_normal(40 * 100)),        # wide dense leaf (atoms split rows)
        (1, 0, 41, 30, 1, 50, np.zeros(0)),                          # kt = 0 low-rank leaf: contributes nothing
        (1, 3, 41, 30, 51, 50, rng.standard_normal(3 * (30 + 50))),  # ordinary low-rank
        (1, 70, 71, 30, 1, 100, rng.standard_normal(70 * 130)),      # kt > panel width: several panels
        (2, 0, 41, 30, 1, 50, rng.standard_normal(30 * 50)),
    ]
    P, keep = _custom(leaves, nd)
    x = rng.standard_normal(nd)
    for nc in (1, 5, 148):
        rc, msg, y, _ = run_emu(emu, C.cast(C.pointer(P), C.c_void_p), nd, nc, x)
        assert rc == 0, msg
        ref = _dense_of(leaves, nd) @ x
        assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()


def test_empty_leaf_list_gives_zero(emu):
    P, keep = _custom([], 37)
    x = np.ones(37)
    rc, msg, y, _ = run_emu(emu, C.cast(C.pointer(P), C.c_void_p), 37, 148, x)
    assert rc == 0, msg
    assert np.all(y == 0.0)


def test_malformed_leaves_are_rejected(emu):
    rng = np.random.default_rng(10)
    bad = [
        [(3, 0, 1, 10, 1, 10, rng.standard_normal(100))],           # unknown ltmtx
        [(2, 0, 95, 10, 1, 10, rng.standard_normal(100))],          # rows past nd
        [(2, 0, 0, 10, 1, 10, rng.standard_normal(100))],           # nstrtl < 1
        [(1, -1, 1, 10, 1, 10, np.zeros(0))],                       # negative kt
    ]
    for leaves in bad:
        P, keep = _custom(leaves, 100)
        rc, msg, _, _ = run_emu(emu, C.cast(C.pointer(P), C.c_void_p), 100, 4, np.ones(100))
        assert rc != 0 and "make_plan" in msg


@pytest.mark.parametrize("level,nc", [(3, 148), (4, 148), (3, 5)])
def test_transposed_layout_reproduces_oracle_transpose(emu, level, nc):
    """H^T packed from the transposed leaf list (hbx_plan.cpp:transpose_leaves)
    against the oracle's transposed product; same bytes as H."""
    import oracle
    H = sphere(level)
    x = np.random.default_rng(level + 40).standard_normal(H.nd)
    rc, msg, y, stats = run_emu(emu, C.cast(H.st, C.c_void_p), H.nd, nc, x, transposed=True)
    assert rc == 0, msg
    ref = oracle.matvec_t(H.st, x)
    assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()
    d, lr = H.storage_words()
    assert stats[6] == 8 * (d + lr) + stats[7]


def test_transposed_edge_cases(emu):
    rng = np.random.default_rng(19)
    nd = 100
    leaves = [
        (2, 0, 1, 40, 1, 100, rng.standard_normal(40 * 100)),
        (1, 0, 41, 30, 1, 50, np.zeros(0)),
        (1, 3, 41, 30, 51, 50, rng.standard_normal(3 * (30 + 50))),
        (1, 70, 71, 30, 1, 100, rng.standard_normal(70 * 130)),
        (2, 0, 41, 30, 1, 50, rng.standard_normal(30 * 50)),
    ]
    P, keep = _custom(leaves, nd)
    x = rng.standard_normal(nd)
    rc, msg, y, _ = run_emu(emu, C.cast(C.pointer(P), C.c_void_p), nd, 7, x, transposed=True)
    assert rc == 0, msg
    ref = _dense_of(leaves, nd).T @ x
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("level,nc", [(3, 148), (4, 148), (3, 7)])
def test_fp32_layout(emu, level, nc):
    """FP32 storage: 4-column float panels with the same 16-byte rows; every
    factor stored once (half the bytes), products within float rounding of
    the FP64 oracle."""
    import oracle
    H = sphere(level)
    x = np.random.default_rng(level + 70).standard_normal(H.nd)
    y = np.zeros(H.nd)
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    rc = emu.emu_matvec_prec(C.cast(H.st, C.c_void_p), H.nd, nc, 1, x.ctypes.data_as(C.POINTER(C.c_double)),
                             y.ctypes.data_as(C.POINTER(C.c_double)), stats, msg, 512)
    assert rc == 0, msg.value.decode()
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() <= 2e-6 * np.abs(ref).max()
    d, lr = H.storage_words()
    assert stats[6] == 4 * (d + lr) + stats[7]
    assert stats[7] <= 0.05 * 4 * (d + lr)


def _bf16_reference(v: np.ndarray) -> np.ndarray:
    """bfloat16 bits of v rounded to 8 significant bits, to nearest with ties
    to even, in one step from the double (frexp/rint restatement, float's
    normal range)."""
    m, e = np.frexp(v)                      # v = m 2^e, 0.5 <= |m| < 1
    r = np.ldexp(np.rint(np.ldexp(m, 8)), e - 8)
    return (r.astype(np.float32).view(np.uint32) >> 16).astype(np.uint32)


def test_bf16_rounding(emu):
    """The packer's double -> bfloat16 rounding against an independent
    restatement: random values over many magnitudes, and exact ties and
    near-ties, where rounding through float first would give another result
    (1 + 2^-8 + 2^-40 rounds up; via float it would be a tie, rounded down)."""
    rng = np.random.default_rng(11)
    v = rng.standard_normal(20000) * np.exp2(rng.integers(-60, 60, 20000))
    ties = np.array([1 + 2.0**-8, 1 + 3 * 2.0**-8, -(1 + 2.0**-8), 1 + 2.0**-8 + 2.0**-40,
                     1 + 2.0**-8 - 2.0**-40, 3.0 * (1 + 2.0**-8), 0.75 * (1 + 5 * 2.0**-9)])
    v = np.concatenate([v, ties, [0.0, 1.0, -2.5, 65504.0, 1e-30]])
    got = np.array([emu.emu_bf16_from_double(float(t)) for t in v], dtype=np.uint32)
    assert np.array_equal(got, _bf16_reference(v))
    assert emu.emu_bf16_from_double(1 + 2.0**-8 + 2.0**-40) == 0x3F81  # up: not a tie in the double
    assert emu.emu_bf16_from_double(1 + 2.0**-8) == 0x3F80             # a tie: to even
    assert emu.emu_bf16_from_double(-0.0) == 0x8000


def test_bf16_rounding_below_float_normal_range(emu):
    """Below 2^-126 bfloat16 is subnormal (multiples of 2^-133): one
    rounding from the double, against exact rational arithmetic; rounding
    through float first would round twice (2^-133 * (5/2 + 2^-30) rounds up
    to 3 units here, while a float rounding would first make it an exact
    tie, 5/2, and then round it to even, 2)."""
    from fractions import Fraction
    unit = Fraction(1, 2**133)

    def ref(v):
        q = abs(Fraction(v)) / unit
        k = int(q)
        rem = q - k
        if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and k % 2 == 1):
            k += 1
        return (0x8000 if np.signbit(v) else 0) | k

    rng = np.random.default_rng(12)
    v = list(rng.uniform(0, 2.0**-126, 300) * rng.choice([-1.0, 1.0], 300))
    v += [2.0**-133 * (2.5 + 2.0**-30), 2.0**-133 * 2.5, 2.0**-133 * 3.5, 2.0**-126 * (1 - 2.0**-40),
          2.0**-140, -2.0**-133 * 0.5, 5e-324]
    for t in v:
        assert emu.emu_bf16_from_double(float(t)) == ref(float(t)), t
    assert emu.emu_bf16_from_double(2.0**-133 * (2.5 + 2.0**-30)) == 3


@pytest.mark.parametrize("level,nc", [(3, 148), (4, 148), (3, 7), (3, 1)])
def test_bf16_layout(emu, level, nc):
    """BF16 storage: 8-column bfloat16 panels with the same 16-byte rows,
    vectors staged as float; every factor stored once (a quarter of the FP64
    bytes).  bfloat16 keeps 8 significant bits (unit roundoff 2^-9), so the
    product is compared with the FP64 oracle in the relative 2-norm against
    a bound of 2^-8 (measured values printed); run widths stay within the
    2048-float stage."""
    import oracle
    H = sphere(level)
    x = np.random.default_rng(level + 80).standard_normal(H.nd)
    y = np.zeros(H.nd)
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    rc = emu.emu_matvec_prec(C.cast(H.st, C.c_void_p), H.nd, nc, 2, x.ctypes.data_as(C.POINTER(C.c_double)),
                             y.ctypes.data_as(C.POINTER(C.c_double)), stats, msg, 512)
    assert rc == 0, msg.value.decode()
    ref = oracle.matvec(H.st, x)
    rel = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    d, lr = H.storage_words()
    print(f"L{level} nc={nc}: BF16 relative error {rel:.2e}, padding {stats[7] / (2 * (d + lr)):.3f}")
    assert rel <= 2.0**-8
    assert stats[6] == 2 * (d + lr) + stats[7]
    assert stats[7] <= 0.15 * 2 * (d + lr)


@pytest.mark.parametrize("level,nc", [(3, 148), (4, 148), (3, 7), (3, 1)])
def test_pair_panel_layout(emu, level, nc):
    """The multi-RHS engine's layout: FP32 panels, every run a whole number of
    panel pairs (the K = 8 of one TF32 tensor-core step), segments in stage
    order; one right-hand side through it matches the FP64 oracle within
    float rounding, and the pair padding stays small."""
    import oracle
    H = sphere(level)
    x = np.random.default_rng(level + 90).standard_normal(H.nd)
    y = np.zeros(H.nd)
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    rc = emu.emu_matvec_pairs(C.cast(H.st, C.c_void_p), H.nd, nc, x.ctypes.data_as(C.POINTER(C.c_double)),
                              y.ctypes.data_as(C.POINTER(C.c_double)), stats, msg, 512)
    assert rc == 0, msg.value.decode()
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() <= 2e-6 * np.abs(ref).max()
    d, lr = H.storage_words()
    assert stats[6] == 4 * (d + lr) + stats[7]
    assert stats[7] <= 0.12 * 4 * (d + lr)


@pytest.mark.parametrize("nc", [148, 5])
def test_block_diagonal_batch_layout(emu, nc):
    """Independent H-matrices of different sizes packed as one block-diagonal
    leaf list (hbx_create_batch's layout): the packed product is each
    instance's oracle product, one after the other."""
    import oracle
    from hacapk_b200 import hmatrix
    Hs = [hmatrix.HostHMatrix(hmatrix.ellipsoid(lv, ax), leaf_size=32, eta=2.0, aca_eps=1e-5)
          for lv, ax in [(2, (1.0, 0.5, 2.0)), (3, (0.4, 1.2, 0.9)), (2, (2.5, 2.5, 0.3)), (3, (1.0, 1.0, 1.0))]]
    nds = [H.nd for H in Hs]
    x = np.random.default_rng(11).standard_normal(sum(nds))
    sts = (C.c_void_p * len(Hs))(*[C.cast(H.st, C.c_void_p) for H in Hs])
    ndarr = (C.c_int * len(Hs))(*nds)
    y = np.zeros(sum(nds))
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    rc = emu.emu_matvec_batch(sts, ndarr, len(Hs), nc, x.ctypes.data_as(C.POINTER(C.c_double)),
                              y.ctypes.data_as(C.POINTER(C.c_double)), stats, msg, 512)
    assert rc == 0, msg.value.decode()
    off = np.concatenate([[0], np.cumsum(nds)])
    for k, H in enumerate(Hs):
        ref = oracle.matvec(H.st, x[off[k]:off[k + 1]])
        assert np.abs(y[off[k]:off[k + 1]] - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("block_cost,run_cost", [(1, 1), (2048, 1024), (32768, 16384), (1 << 20, 1)])
def test_cost_models_keep_the_layout_valid(emu, block_cost, run_cost):
    """Every balancing cost model the autotuner may pick gives a valid layout
    (the emulator's structural checks) with the oracle's product: the model
    only moves blocks between CTAs."""
    import oracle
    H = sphere(4)
    x = np.random.default_rng(block_cost % 97).standard_normal(H.nd)
    y = np.zeros(H.nd)
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    rc = emu.emu_matvec_costs(C.cast(H.st, C.c_void_p), H.nd, 148, block_cost, run_cost,
                              x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)),
                              stats, msg, 512)
    assert rc == 0, msg.value.decode()
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()


def test_batch_layout_rejects_bad_instances(emu):
    """combine_leaves refuses a missing container, a non-positive size and a
    leaf outside its instance's [1, nd]."""
    from hacapk_b200 import hmatrix
    H = hmatrix.HostHMatrix(hmatrix.ellipsoid(2, (1.0, 1.0, 1.0)), leaf_size=32, eta=2.0, aca_eps=1e-5)
    x = np.zeros(2 * H.nd)
    y = np.zeros(2 * H.nd)
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)

    def run(sts, nds):
        arr = (C.c_void_p * len(sts))(*sts)
        nd = (C.c_int * len(nds))(*nds)
        return emu.emu_matvec_batch(arr, nd, len(sts), 148, x.ctypes.data_as(C.POINTER(C.c_double)),
                                    y.ctypes.data_as(C.POINTER(C.c_double)), stats, msg, 512)

    st = C.cast(H.st, C.c_void_p).value
    assert run([st, st], [H.nd, H.nd]) == 0
    assert run([st, None], [H.nd, H.nd]) != 0 and b"null container" in msg.value
    assert run([st, st], [H.nd, 0]) != 0 and b"nd <= 0" in msg.value
    assert run([st, st], [H.nd, H.nd - 1]) != 0 and b"outside [1, nd]" in msg.value


def test_pair_panel_layout_edge_cases(emu):
    """The multi-RHS layout on the edge leaves of test_edge_cases plus an atom
    that only low-rank leaves touch (its D block is empty: one run of no
    panels) and an empty leaf list: runs stay whole panel pairs, the float
    product matches the dense one within float rounding."""
    rng = np.random.default_rng(19)
    nd = 100
    leaves = [
        (2, 0, 1, 40, 1, 100, rng.standard_normal(40 * 100)),
        (1, 0, 41, 30, 1, 50, np.zeros(0)),
        (1, 3, 41, 30, 51, 50, rng.standard_normal(3 * (30 + 50))),
        (1, 70, 71, 30, 1, 100, rng.standard_normal(70 * 130)),
        (2, 0, 41, 30, 1, 50, rng.standard_normal(30 * 50)),
    ]
    P, keep = _custom(leaves, nd)
    x = rng.standard_normal(nd)
    ref = _dense_of(leaves, nd) @ x
    for nc in (1, 5, 148):
        y = np.zeros(nd)
        stats = (C.c_longlong * 8)()
        msg = C.create_string_buffer(512)
        rc = emu.emu_matvec_pairs(C.cast(C.pointer(P), C.c_void_p), nd, nc, x.ctypes.data_as(C.POINTER(C.c_double)),
                                  y.ctypes.data_as(C.POINTER(C.c_double)), stats, msg, 512)
        assert rc == 0, msg.value.decode()
        assert np.abs(y - ref).max() <= 2e-6 * np.abs(ref).max()
    P0, keep0 = _custom([], 33)
    y = np.ones(33)
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    rc = emu.emu_matvec_pairs(C.cast(C.pointer(P0), C.c_void_p), 33, 148, np.ones(33).ctypes.data_as(C.POINTER(C.c_double)),
                              y.ctypes.data_as(C.POINTER(C.c_double)), stats, msg, 512)
    assert rc == 0, msg.value.decode()
    assert np.all(y == 0.0)


def _merged(emu, H, nc, keep, precision=0, seed=0):
    x = np.random.default_rng(seed).standard_normal(H.nd)
    y = np.zeros(H.nd)
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    rc = emu.emu_matvec_merged(C.cast(H.st, C.c_void_p), H.nd, nc, precision, keep,
                               x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)),
                               stats, msg, 512)
    return rc, msg.value.decode(), x, y, list(stats)


@pytest.mark.parametrize("level,nc,keep", [(3, 148, 0), (3, 148, 1), (4, 148, 0), (4, 148, 2), (3, 7, 1),
                                           (3, 1, 0), (4, 300, 0)])
def test_merged_du_layout(emu, level, nc, keep):
    """Merged D+U blocks (make_plan's merge_keep): an atom's dense and
    low-rank columns in one block in the U section, each gather segment
    marked with its source.  The layout keeps every invariant the emulator
    checks (rows written once, by the CTA that owns them; the atom list in
    the order of the blocks that first write them), reproduces the oracle,
    packs the same factor bytes and needs no more runs than the split layout
    (fewer when every atom merges: at 148 CTAs these matrices hold few
    atoms with low-rank rows per CTA, so merge_keep = 1 or 2 may leave all
    split)."""
    import oracle
    H = sphere(level)
    rc, msg, x, y, st_m = _merged(emu, H, nc, keep, seed=level + nc)
    assert rc == 0, msg
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()
    rc, msg, _, _, st_s = _merged(emu, H, nc, -1, seed=level + nc)
    assert rc == 0, msg
    d, lr = H.storage_words()
    assert st_m[6] == 8 * (d + lr) + st_m[7]   # every factor packed once
    assert st_m[1] <= st_s[1]                   # never more runs;
    if keep == 0:                               # fewer when every atom with U rows merges
        assert st_m[1] < st_s[1]
    print(f"L{level} nc={nc} keep={keep}: runs {st_s[1]} -> {st_m[1]}")


def test_merged_du_layout_other_precisions_and_rejects_pairs(emu):
    import oracle
    H = sphere(3)
    for prec, tol in ((1, 2e-6), (2, 2.0**-8)):
        rc, msg, x, y, _ = _merged(emu, H, 148, 0, precision=prec, seed=prec)
        assert rc == 0, msg
        ref = oracle.matvec(H.st, x)
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= tol
    # the multi-RHS layout has no merged form
    stats = (C.c_longlong * 8)()
    msg = C.create_string_buffer(512)
    x = np.zeros(H.nd)
    y = np.zeros(H.nd)
    assert emu.emu_matvec_pairs(C.cast(H.st, C.c_void_p), H.nd, 148, x.ctypes.data_as(C.POINTER(C.c_double)),
                                y.ctypes.data_as(C.POINTER(C.c_double)), stats, msg, 512) == 0


def test_merged_du_layout_needs_wider_stages(build_libs):
    """The merge's gain, on the planner's own per-CTA tables (C1 L5, 148
    CTAs): with 8 KB stages an atom's D and U columns together overflow one
    stage, so the CTA holding the most runs keeps them all; with 16 KB stages
    (the planner built with HBX_STAGE_BYTES=16384) merging takes that maximum
    down by the 6 U runs of its atoms."""
    from hacapk_b200 import configs
    lib16 = os.path.join(ROOT, "tests", "emu", "_build", "libplanemu16.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-DHBX_STAGE_BYTES=16384", "-o",
                    lib16, EMU_SRC, os.path.join(ROOT, "hacapk-magma_b200", "csrc", "hbx_plan.cpp")], check=True)
    H, _ = configs.c1(5)
    nc = 148

    def max_runs(lib, keep):
        b, r = (C.c_longlong * nc)(), (C.c_int * nc)()
        assert lib.emu_plan_cta_table(C.cast(H.st, C.c_void_p), H.nd, nc, 0, keep, b, r) == 0
        return max(r[:])

    lib8 = C.CDLL(EMU_LIB)
    lib16 = C.CDLL(lib16)
    for lib in (lib8, lib16):
        lib.emu_plan_cta_table.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.c_longlong), C.POINTER(C.c_int)]
    split8, merged8 = max_runs(lib8, -1), max_runs(lib8, 0)
    split16, merged16 = max_runs(lib16, -1), max_runs(lib16, 0)
    print(f"max runs per CTA: 8 KB {split8} -> {merged8}, 16 KB {split16} -> {merged16}")
    assert merged8 == split8
    assert merged16 <= split16 - 5


@pytest.mark.parametrize("precision,merge_keep", [(0, 4), (1, -1), (2, -1)])
def test_batch_chunk_table_covers_every_run(build_libs, precision, merge_keep):
    """The block-diagonal engine's chunk -> instance-range table (the batched
    solver's products skip chunks of finished instances with it) lists, for
    every 32 KB chunk of every CTA stream, each instance whose run bytes the
    chunk holds (FP64 streams: ~80 % of the chunks hold one instance; the
    smaller FP32 / BF16 streams share more chunks between instances)."""
    import ctypes as C
    from conftest import emu_lib
    from hacapk_b200 import abi, configs
    inst = configs.c5(count=24, seed=5, max_level=4)
    L = emu_lib()
    k = len(inst)
    sts = (C.c_void_p * k)(*[C.cast(H.st, C.c_void_p) for H, _ in inst])
    nds = (C.c_int * k)(*[int(H.nd) for H, _ in inst])
    stats = (C.c_longlong * 4)()
    bad = L.emu_chunk_table(sts, nds, k, 148, precision, merge_keep, stats)
    assert bad == 0
    chunks, one, none, runs = list(stats)
    assert runs > 0 and chunks > 0
    assert one + none <= chunks
    print(f"precision {precision}: {chunks} chunks, {one} with one instance, {none} empty, {runs} runs")
