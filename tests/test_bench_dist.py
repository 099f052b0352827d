"""bench.py's multi-rank path (independent replicas) on CPU with gloo,
world_size 2: the barrier and the whole-job aggregation (all ranks' units
over the slowest rank's time) agree on every rank."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        bench.dist_barrier(world)
        rate, t_max = bench.aggregate_rate(100.0 * (rank + 1), 1.0 + rank, world)
        q.put((rank, rate, t_max))
        bench.dist_barrier(world)
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, rate, t_max in got:
        assert t_max == pytest.approx(2.0)
        assert rate == pytest.approx(300.0 / 2.0)


def test_single_rank_aggregation_is_local():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_rate(50.0, 2.0, 1) == (25.0, 2.0)


def test_every_committed_profile_reads_as_traffic():
    """bench.py takes the roofline's `traffic` from the summaries under
    profiles/: every summary that carries the line must parse (a number of
    bytes per launch, or null where the state stays in L2)."""
    sys.path.insert(0, ROOT)
    import bench
    tags = [f[:-3] for f in os.listdir(os.path.join(ROOT, "profiles")) if f.endswith(".md")]
    assert tags
    for tag in tags:
        with open(os.path.join(ROOT, "profiles", tag + ".md")) as fh:
            carries = any(line.startswith("traffic_bytes_per_launch:") for line in fh)
        value = bench.profiled_traffic(tag)
        if carries and "closure" not in tag:
            assert isinstance(value, float) and value > 0, tag
        else:
            assert value is None or value > 0, tag


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` runs LBM-C's own step (host-compiled, all
    host threads) on a bounded sample of the workload and prints one JSON
    line with the arm's keys: the same metric and unit as the GPU arm,
    impl = reference, a cpu_baseline describing the run and an e2e with no
    host<->device bytes.  Host-only: no GPU is involved."""
    import json
    import subprocess

    sys.path.insert(0, ROOT)
    from oracle.oracle import reference_available
    if not reference_available("d3q15", "patched"):
        pytest.skip("oracle/_ref not built")
    run = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--size", "32", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert run.returncode == 0, run.stderr[-2000:]
    line = json.loads(run.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "GLUPS" and line["value"] > 0
    assert line["metric"].startswith("GLUPS (D3Q15 MRT porous 32^3")
    assert line["steps"] == 2 and line["warmup"] == 1 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["length"] == [32, 32, 32]
