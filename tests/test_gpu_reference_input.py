"""The reference's own input, bem-bb_inputs/input_10ts.pbs (10,400 flat
triangles, the ppohBEM kernel, leaf size 15, ACA+ 1e-6 -- the parameters of
its recorded run), taken through the drop-in entry points in the order its
Fortran driver calls them (m_HACApK_solve.f90:597-735):

  1. c_hacapk_adot_body_lfcpy_batch_sorted_  (copy H to the GPU);
  2. the CPU-vs-GPU product check with x = 1 (m_HACApK_solve.f90:705-735):
     zau = H 1 through c_hacapk_adot_body_lfmtx_batch_ against the
     reference's own compiled CPU product, relative 2-norm error;
  3. c_hacapk_bicgstab_cax_lfmtx_gpu_, c_hacapk_bicgstab_cax_lfmtx_flat_ and
     c_hacapk_bicgstab_cax_lfmtx_mgpu1_ (HACApK_SOLVER.c:421, :254, :815; the
     last is what the reference's default build calls, m_HACApK_use.f90:349)
     on b = 1 (unit potential), each within +-1 step of the oracle BiCGSTAB
     and below 1e-8 in the true residual, _mgpu1_ equal to _gpu_ bit for bit;
  4. c_hacapk_adot_body_lfdel_batch_.

The mesh comes from the committed fixture tests/golden/input_10ts_mesh.npz
(tests/golden/make_golden.py wrote it from the reference file)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_reference_input_through_the_drop_in_entry_points(gpu, build_libs):
    import oracle
    from conftest import reference_input_mesh
    from hacapk_b200 import abi, hmatrix
    from test_gpu_bicgstab import _control
    lib = abi.engine_lib()
    m = reference_input_mesh()
    assert m.faces.shape == (10400, 3)
    H = hmatrix.HostHMatrix(m, leaf_size=15, eta=2.0, aca_eps=1e-6, kernel=abi.KERNEL_PPOHBEM)
    n = H.nd
    nd = C.c_int(n)
    lib.c_hacapk_adot_body_lfcpy_batch_sorted_(C.byref(nd), H.st)
    # the driver's self-check: x = 1, GPU product against the CPU one
    x = np.ones(n)
    zau = np.zeros(n)
    zbu = np.zeros(max(1, H.st.contents.ktmax))
    tb, ts, tc = C.c_double(0), C.c_double(0), C.c_double(0)
    lib.c_hacapk_adot_body_lfmtx_batch_(abi.dptr(zau), H.st, abi.dptr(x), abi.dptr(zbu), C.byref(tb), C.byref(ts),
                                        C.byref(tc))
    ref = oracle.matvec_ref(H.st, x) if oracle.have_ref() else oracle.matvec(H.st, x)
    assert np.linalg.norm(zau - ref) / np.linalg.norm(ref) <= 1e-13
    assert tb.value > 0.0
    b = H.to_cluster(np.ones(n))
    _, n_ref, _, _ = oracle.bicgstab(H.st, b, tol=1e-8, max_iter=1000, kind="ref" if oracle.have_ref() else "restated")
    sols = {}
    for entry in ("c_hacapk_bicgstab_cax_lfmtx_gpu_", "c_hacapk_bicgstab_cax_lfmtx_flat_",
                  "c_hacapk_bicgstab_cax_lfmtx_mgpu1_"):
        ctl, buf = _control()
        u = np.zeros(n)
        nstp, lrtrn = C.c_int(-1), C.c_int(-1)
        getattr(lib, entry)(H.st, C.byref(ctl), abi.dptr(u), abi.dptr(b), ctl.param, C.byref(nd), C.byref(nstp),
                            C.byref(lrtrn))
        assert lrtrn.value == 0, entry
        assert n_ref - 1 <= nstp.value <= n_ref + 1, (entry, nstp.value, n_ref)
        r = b - oracle.matvec(H.st, u)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 1.05e-8, entry
        sols[entry] = (nstp.value, u)
    n_gpu, u_gpu = sols["c_hacapk_bicgstab_cax_lfmtx_gpu_"]
    n_mgpu, u_mgpu = sols["c_hacapk_bicgstab_cax_lfmtx_mgpu1_"]
    assert n_mgpu == n_gpu and np.array_equal(u_mgpu, u_gpu)
    lib.c_hacapk_adot_body_lfdel_batch_(H.st)
