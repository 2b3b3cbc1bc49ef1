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


REF_ARM = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
sys.path.insert(0, sys.argv[0] and {root!r})
import bench
bench.LEVEL = 5
bench.run_reference_arm(bench.argparse.Namespace(steps=1, warmup=0), 0, 1)
maps = open("/proc/self/maps").read()
print(json.dumps({{"libisg": "/isg/libisg.so" in maps or "libisg_ref.so" in maps, "isg_module": "isg" in sys.modules,
                   "oracle_libs": sorted({{l.split()[-1].rsplit("/", 2)[-2] + "/" + l.split()[-1].rsplit("/", 1)[-1]
                                         for l in maps.splitlines() if "oracle" in l and l.endswith(".so")}})}}))
"""


def test_reference_arm_loads_no_library_of_the_package():
    """--impl reference builds its inputs from the oracle's generators and the
    reference's own tables and times only oracle/_ref (here at 128 x 128)."""
    import json
    import subprocess
    import sys

    import pytest
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libisgref.so")):
        pytest.skip("oracle/_ref not built")
    r = subprocess.run([sys.executable, "-c", REF_ARM.format(root=ROOT)], capture_output=True, text=True,
                       timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    arm, maps = lines[0], lines[-1]
    ours = load_bench()
    ours.LEVEL = 5
    assert arm["impl"] == "reference" and arm["value"] > 0 and arm["config"] == ours.workload_config(1)
    assert not maps["libisg"] and not maps["isg_module"], maps
    assert "_ref/libisgref.so" in maps["oracle_libs"], maps


def test_reference_inputs_equal_the_library_inputs():
    import isg
    from _oracle import Reference
    import pytest
    if not Reference.available():
        pytest.skip("oracle/_ref not built")
    b = load_bench()
    b.LEVEL = 5
    s = isg.Solver(5, numrx=32, max_rhs=1)
    g, bb = b.make_inputs(s, 0)
    rg, rb = b.reference_inputs(Reference(5, 2 * np.pi, 32), 0, [0, 7, 255])
    assert np.array_equal(rg.view(np.uint64), g.view(np.uint64))
    for tx in (0, 7, 255):
        assert np.array_equal(rb[tx].view(np.uint64), bb[tx].view(np.uint64)), tx
