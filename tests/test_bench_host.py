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
