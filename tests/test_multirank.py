"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): replicas
report the max over ranks, and the reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def run_ranks(body, world=2, timeout=120):
    port = free_port()
    script = textwrap.dedent(f"""
        import os, sys, datetime
        sys.path.insert(0, {ROOT!r})
        import torch.distributed as dist
        import bench
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        rank = dist.get_rank()
    """) + textwrap.dedent(body) + "\ndist.destroy_process_group()\n"
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", script], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        out, _ = p.communicate(timeout=timeout)
        assert p.returncode == 0, out
        outs.append(out)
    return outs


def test_max_over_ranks_gloo():
    outs = run_ranks("""
        v = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist, "cpu")
        print("RESULT", v)
    """)
    for o in outs:
        assert "RESULT [2.0, 10.0]" in o


def test_reference_arm_runs_on_rank0_only():
    outs = run_ranks("""
        class A: pass
        args = A(); args.N = 4096; args.steps = 1; args.warmup = 1; args.workload = "uniform4k"; args.gpus = 2
        bench.run_reference(args)
        dist.barrier()
    """, timeout=300)
    assert '"impl": "reference"' in outs[0]
    assert '"impl"' not in outs[1]


def test_shard_outputs_combine_gloo():
    """Sharding one problem: the ranks' partitions of the tree tile it, and
    the all-reduce of outputs that are nonzero only on each rank's own part
    gives the whole vector exactly (afmm2d_b200.shard.combine)."""
    outs = run_ranks("""
        import numpy as np, torch
        import afmm2d_b200 as A
        from afmm2d_b200 import shard
        world = dist.get_world_size()
        lev, k0, k1 = A.shard_range(6, rank, world)
        got = [None] * world
        dist.all_gather_object(got, (lev, k0, k1))
        assert all(g[0] == lev for g in got) and got[0][1] == 0 and got[-1][2] == 4 ** lev
        assert all(got[i][2] == got[i + 1][1] for i in range(world - 1))
        full = np.random.default_rng(5).standard_normal(4 ** lev * 7)
        part = np.zeros_like(full)
        part[k0 * 7:k1 * 7] = full[k0 * 7:k1 * 7]
        t = shard.combine(torch.from_numpy(part))
        assert np.array_equal(t.numpy(), full)
        print("RESULT ok", lev, k0, k1)
    """)
    for o in outs:
        assert "RESULT ok" in o
