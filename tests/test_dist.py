"""The multi-rank plumbing of bench.py on the CPU (gloo, world size 2): the
path does not shard -- N GPUs run N independent replicas -- so the only
collective steps are the barrier around the timed region and the max over
ranks of the measured times; and the reference arm runs on rank 0 alone."""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank), HBX_BENCH_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    w, r, _ = bench.dist_setup()
    bench.barrier(w)
    v = bench.reduce_max(1.5 * (r + 1), w)  # rank 1 measured the longer time
    bench.barrier(w)
    q.put((r, w, v))
    dist.destroy_process_group()


def test_barrier_and_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 2, 3.0), (1, 2, 3.0)]


def test_reference_arm_runs_on_rank_zero_only(build_libs):
    """torchrun with two ranks (gloo): exactly one JSON line, from rank 0,
    with impl = reference; both ranks exit 0."""
    env = dict(os.environ, HBX_BENCH_BACKEND="gloo")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--level", "2",
           "--steps", "1", "--warmup", "0"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["cpu_baseline"]["kind"] in ("port", "reference")
