"""bench.py's multi-rank host logic on CPU: two gloo ranks on 127.0.0.1 agree
on the slowest rank's time, and each rank draws its own problem (weak
scaling over transmitters)."""
import importlib.util
import os
import socket

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def rank_main(rank, world, port, outdir):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = load_bench()
        got = b.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        np.save(os.path.join(outdir, f"max{rank}.npy"), np.array([got]))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    assert [float(np.load(tmp_path / f"max{r}.npy")[0]) for r in range(2)] == [15.0, 15.0]


def test_single_rank_is_identity_and_ranks_draw_different_problems():
    import isg
    b = load_bench()
    assert b.max_over_ranks(3.5, None, "cpu") == 3.5
    s = isg.Solver(4, numrx=16, max_rhs=1)
    g0, _ = b.make_inputs(s, 0)
    g1, _ = b.make_inputs(s, 1)
    assert not np.allclose(g0, g1)
