"""hbx_matvec_noalloc: the allocation-free H-matvec for callers that cannot
call cudaMalloc while they run.  It must give the same result as hbx_matvec
(the existing entry point) on consecutive calls -- the static scratch keeps
the previous call's contents, so the second call checks that nothing stale
leaks into the result -- and reject matrices whose scratch does not fit.
Collected last so that a run stopping at the first failure has run the rest."""
import ctypes as C

import numpy as np
import pytest

from conftest import sphere

pytestmark = pytest.mark.gpu
TOL = 1e-13


def test_noalloc_matches_matvec_on_two_calls(gpu, build_libs):
    import torch
    from hacapk_b200 import abi
    from hacapk_b200.engine import Engine
    lib = abi.engine_lib()
    H = sphere(4)
    E = Engine(H.st, H.nd)
    assert E.info["zbu_len"] <= 131040
    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(2024)
    for call in range(2):
        x = torch.from_numpy(rng.standard_normal(H.nd)).to(gpu)
        z = torch.from_numpy(rng.standard_normal(H.nd)).to(gpu)
        y_ref = torch.empty_like(x)
        y_new = torch.empty_like(x)
        E.matvec_dev(x.data_ptr(), y_ref.data_ptr(), alpha=1.5, beta=-0.5, yin_ptr=z.data_ptr(), stream=s)
        st = lib.hbx_matvec_noalloc(E._h, 1.5, C.c_void_p(x.data_ptr()), -0.5, C.c_void_p(z.data_ptr()),
                                    C.c_void_p(y_new.data_ptr()), C.c_void_p(s))
        assert st == 0, lib.hbx_last_error()
        E.sync(s)
        ref, got = y_ref.cpu().numpy(), y_new.cpu().numpy()
        assert np.abs(got - ref).max() <= TOL * np.abs(ref).max(), f"call {call}"


def test_noalloc_rejects_scratch_beyond_its_limit(gpu, build_libs):
    from hacapk_b200 import abi
    from hacapk_b200.engine import Engine
    import test_plan as tp
    lib = abi.engine_lib()
    rng = np.random.default_rng(5)
    leaves = [(1, 70, 1, 1, 1, 1, rng.standard_normal(140)) for _ in range(2000)]  # ranks sum to 140000
    P, keep = tp._custom(leaves, 2)
    E = Engine(C.pointer(P), 2)
    x = np.ones(2)
    import torch
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    st = lib.hbx_matvec_noalloc(E._h, 1.0, C.c_void_p(xd.data_ptr()), 0.0, None, C.c_void_p(yd.data_ptr()),
                                None)
    assert st == 1
    assert b"static scratch holds 131040" in lib.hbx_last_error()
