"""bench.py's host-side CPU legs on the CPU: the reference's CPU products
(the per-leaf BLAS GEMV path on one thread and on every core, the OpenMP
product on every core) are timed and reported with the core count."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_host_matvecs_report_both_cpu_paths(build_libs):
    import bench
    from conftest import sphere
    H = sphere(2)
    out = bench.host_matvecs(H, seconds=0.05)
    cores = len(os.sched_getaffinity(0))
    assert out["cores"] == cores
    assert out["blas_gemv_ms_1_threads"] > 0 and out[f"blas_gemv_ms_{cores}_threads"] > 0
    assert out[f"omp_ms_{cores}_threads"] > 0


def test_a_failing_form_is_reported_beside_the_others(monkeypatch):
    """An exception in one form (an out-of-memory on a small box, say) is
    recorded as that form's "error" entry; the other forms still run and the
    bench line is still printed."""
    import argparse

    import bench

    def boom(args, dev, stream):
        raise RuntimeError("hbx_create: out of device memory")

    monkeypatch.setattr(bench, "solvers_form", lambda args, dev, stream: {"ok": 1})
    monkeypatch.setattr(bench, "autotune_form", boom)
    for name in ("precision_form", "mrhs_form", "adjoint_form", "batch_form"):
        monkeypatch.setattr(bench, name, lambda args, dev, stream: {"ok": 2})
    out = bench.measure_forms(argparse.Namespace(form=""), None, None)
    assert out["solvers_c1"] == {"ok": 1} and out["batch_c5"] == {"ok": 2}
    assert out["autotune_c1"]["error"].startswith("RuntimeError: hbx_create")
    assert list(bench.measure_forms(argparse.Namespace(form="mrhs_c3"), None, None)) == ["mrhs_c3"]
