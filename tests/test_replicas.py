"""The multi-GPU path of bench.py (replicas: every rank traverses its own
roots, no collective on the data path) run as two gloo ranks on CPU: the
max-over-ranks reduction and the per-rank root sets."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    # rank r: step 10 + r ms, 100 / (r + 1) GTEPS, e2e 90 / (r + 1)
    out = bench.reduce_over_ranks(10.0 + rank, 100.0 / (rank + 1), 90.0 / (rank + 1))
    q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        step, value, e2e = got[r]
        assert step == 11.0                 # the slowest rank's step
        assert abs(value - 2 * 50.0) < 1e-9  # world x the slowest rank's rate
        assert abs(e2e - 2 * 45.0) < 1e-9


def test_ranks_traverse_different_roots():
    # bench.py gives rank r the lcg(r) roots of the same graph
    n, src, dst = O.rmat_graph(12, 16, seed=5)
    off, _ = O.csr_build(n, src, dst)
    r0, r1 = O.pick_roots(off, 0, 64), O.pick_roots(off, 1, 64)
    assert not np.array_equal(r0, r1)
    deg = np.diff(off)
    assert (deg[r0] > 0).all() and (deg[r1] > 0).all()


def test_both_arms_describe_the_workload_alike():
    # the reference arm and the GPU arm print one `config` object for the
    # headline workload; how each ran it lives elsewhere in the line
    import sys
    sys.path.insert(0, ROOT)
    import bench
    desc = f"rmat-scale{bench.SCALE}-ef{bench.EDGE_FACTOR} seed {bench.GRAPH_SEED}"
    a = bench.workload_config(desc, bench.NUM_ROOTS, bench.SCALE, bench.GRAPH_SEED, 1 << 24, 259835455)
    b = bench.workload_config(desc, bench.NUM_ROOTS, bench.SCALE, bench.GRAPH_SEED, 1 << 24, 259835455)
    assert a == b and a["workload"].endswith("64 roots per step")
    assert a["roots"] == 64 and a["root_seed"] == 0 and "CSR 2.21 GB" in a["l2"]
    assert not {"mode", "parallelism", "graph_build_s", "roots_per_step"} & set(a)
