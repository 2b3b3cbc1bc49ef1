"""The device-resident inversion loop (isg_dbim) against the reference's own
driver run (tests/golden/golden_dbim_l7.npz): same phantom, 4 plane waves,
32 receivers, 512 x 512 pixels, 3 Polak-Ribiere iterations, inner solves to
1e-4.  Complex64 fields with FP64 contrast and reductions: the history agrees
to 1e-3 relative and the final contrast to 2e-3 (the reference's own
FP64 runs at this tolerance differ by ~1e-4)."""
import os

import numpy as np
import pytest

import isg
from _oracle import rel

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_dbim_l7.npz")


@pytest.mark.parametrize("engine", [isg.ENGINE_SIMT, isg.ENGINE_TENSOR])
def test_dbim_matches_reference_driver(engine):
    import torch
    d = dict(np.load(GOLDEN))
    ntx = int(d["ntx"])
    s = isg.Solver(int(d["level"]), numrx=int(d["numrx"]), max_rhs=ntx)
    chi_true = torch.from_numpy(d["phantom"].astype(np.float64) * 0.1 + 0j).cuda()
    inc = torch.from_numpy(s.plane_waves(ntx, order=isg.ORDER_RASTER).astype(np.complex64)).cuda()
    tol = float(d["tol"])
    mes = s.measure(inc, chi_true, order=isg.ORDER_RASTER, tol=tol, engine=engine)
    chi, hist = s.dbim(inc, mes, chi_true=chi_true, iterations=3, order=isg.ORDER_RASTER, tol=tol, engine=engine)
    ref = d["hist"]
    got = np.array([[h["misfit"], h["object_error"], h["reg_cost"], h["grad_norm"], h["object_norm"]] for h in hist])
    for col in (0, 1, 3, 4):
        m = np.abs(ref[:, col]) > 0
        assert np.max(np.abs(got[m, col] - ref[m, col]) / np.abs(ref[m, col])) < 1e-3, (col, got[:, col], ref[:, col])
    alpha = np.array([h["alpha"] for h in hist[1:]])
    assert np.max(np.abs(alpha - d["alpha"]) / np.abs(d["alpha"])) < 1e-3
    assert rel(chi.cpu().numpy(), d["cg2"]) < 2e-3
    assert hist[-1]["solves"] == ntx * (1 + 3 * 3)


def test_dbim_warm_start_keeps_the_result_and_saves_iterations():
    """Each transmitter's total-field and adjoint solves start from its fields of
    the previous iteration: the inversion follows the same history to the inner
    tolerance (1e-5), with fewer BiCGSTAB iterations.  256 x 256 pixels, three
    ellipses eps_r in [1.2, 1.6], 8 plane waves, 32 receivers."""
    import torch
    s = isg.Solver(6, numrx=32, max_rhs=8)
    chi_true = torch.from_numpy(s.phantom(seed=55, count=3, axis=(1.5, 3.0), eps=(1.2, 1.6))).cuda()
    inc = torch.from_numpy(s.plane_waves(8, order=isg.ORDER_RASTER).astype(np.complex64)).cuda()
    mes = s.measure(inc, chi_true, order=isg.ORDER_RASTER, tol=1e-6, engine=isg.ENGINE_TENSOR)
    runs = {}
    for warm in (False, True):
        chi, hist = s.dbim(inc, mes, chi_true=chi_true, iterations=4, order=isg.ORDER_RASTER, tol=1e-5,
                           engine=isg.ENGINE_TENSOR, warm_start=warm)
        runs[warm] = (chi.cpu().numpy(), hist)
    (c0, h0), (c1, h1) = runs[False], runs[True]
    print("dbim iterations cold", h0[-1]["iterations"], "warm", h1[-1]["iterations"])
    assert h1[-1]["solves"] == h0[-1]["solves"]
    assert h1[-1]["iterations"] < h0[-1]["iterations"]
    m0 = np.array([h["misfit"] for h in h0])
    m1 = np.array([h["misfit"] for h in h1])
    assert np.max(np.abs(m1 - m0) / m0) < 1e-3, (m0, m1)
    assert rel(c1, c0) < 1e-3


def test_sharded_driver_on_one_gpu_matches_isg_dbim():
    """isg.dbim_dist with the library's operators (one rank, no group) follows
    the device-resident loop: same history to 1e-3 and contrast to 2e-3
    (complex64 fields, different summation order)."""
    import torch
    from isg import dbim_dist
    d = dict(np.load(GOLDEN))
    ntx = int(d["ntx"])
    s = isg.Solver(int(d["level"]), numrx=int(d["numrx"]), max_rhs=ntx)
    chi_true = torch.from_numpy(d["phantom"].astype(np.float64) * 0.1 + 0j).cuda()
    inc = torch.from_numpy(s.plane_waves(ntx, order=isg.ORDER_RASTER).astype(np.complex64)).cuda()
    tol = float(d["tol"])
    mes = s.measure(inc, chi_true, order=isg.ORDER_RASTER, tol=tol, engine=isg.ENGINE_TENSOR)
    chi, hist = s.dbim(inc, mes, chi_true=chi_true, iterations=3, order=isg.ORDER_RASTER, tol=tol,
                       engine=isg.ENGINE_TENSOR)
    inc_t = torch.from_numpy(s.plane_waves(ntx).astype(np.complex64)).cuda()   # tree order
    ops = dbim_dist.GpuOps(s, engine=isg.ENGINE_TENSOR, tol=tol)
    chi2, hist2 = dbim_dist.dbim(ops, inc_t, mes, float(s.opts.k0), iterations=3)
    um = s.host_table("unkmap")
    chi2_raster = chi2.cpu().numpy()[um]
    assert rel(chi2_raster, chi.cpu().numpy()) < 2e-3
    m1 = np.array([h["misfit"] for h in hist])
    m2 = np.array([h["misfit"] for h in hist2])
    assert np.max(np.abs(m2 - m1) / m1) < 1e-3, (m1, m2)


def test_dbim_checkpoint_files_follow_the_reference(tmp_path):
    """With a checkpoint directory the loop writes what the reference's
    write_error writes (setup_born.cpp:171-242): cg_<i>.bin, the contrast in
    raster order as complex128, and hist.txt, one line of five numbers per
    record.  The last file is the returned contrast, the history lines are the
    returned records, and the reference's own cg_2.bin of the same run agrees
    to the parity tolerance of the history test (2e-3)."""
    import torch
    d = dict(np.load(GOLDEN))
    ntx = int(d["ntx"])
    s = isg.Solver(int(d["level"]), numrx=int(d["numrx"]), max_rhs=ntx)
    chi_true = torch.from_numpy(d["phantom"].astype(np.float64) * 0.1 + 0j).cuda()
    inc = torch.from_numpy(s.plane_waves(ntx, order=isg.ORDER_RASTER).astype(np.complex64)).cuda()
    tol = float(d["tol"])
    mes = s.measure(inc, chi_true, order=isg.ORDER_RASTER, tol=tol, engine=isg.ENGINE_TENSOR)
    chi, hist = s.dbim(inc, mes, chi_true=chi_true, iterations=3, order=isg.ORDER_RASTER, tol=tol,
                       engine=isg.ENGINE_TENSOR, checkpoint=str(tmp_path))
    files = sorted(p.name for p in tmp_path.iterdir())
    assert files == ["cg_0.bin", "cg_1.bin", "cg_2.bin", "hist.txt"]
    cg2 = np.fromfile(tmp_path / "cg_2.bin", dtype=np.complex128)
    assert np.array_equal(cg2, chi.cpu().numpy())
    assert rel(cg2, d["cg2"]) < 2e-3
    lines = np.loadtxt(tmp_path / "hist.txt")
    assert lines.shape == (4, 5)
    want = np.array([[h["misfit"], h["object_error"], h["reg_cost"], h["grad_norm"], h["object_norm"]] for h in hist])
    assert np.allclose(lines, want, rtol=1e-5)


def test_sharded_driver_through_a_one_rank_nccl_group():
    """The sharded loop with its exchanges (the gradient, step-length and
    misfit sums of mom.cpp:271, 313-314, 362) as NCCL all-reduces of device
    tensors in a one-rank group on this GPU: the same inversion as the loop
    without a group, bit for bit (a one-rank sum is the identity)."""
    import datetime
    import os
    import socket
    import torch
    import torch.distributed as dist
    from isg import dbim_dist
    d = dict(np.load(GOLDEN))
    ntx = int(d["ntx"])
    s = isg.Solver(int(d["level"]), numrx=int(d["numrx"]), max_rhs=ntx)
    chi_tree = torch.from_numpy(s.raster_to_tree(d["phantom"].astype(np.float64) * 0.1 + 0j)).cuda()
    tol = float(d["tol"])
    inc_t = torch.from_numpy(s.plane_waves(ntx).astype(np.complex64)).cuda()
    mes = s.measure(inc_t, chi_tree, order=isg.ORDER_TREE, tol=tol, engine=isg.ENGINE_TENSOR)
    ops = dbim_dist.GpuOps(s, engine=isg.ENGINE_TENSOR, tol=tol)
    chi0, hist0 = dbim_dist.dbim(ops, inc_t, mes, float(s.opts.k0), iterations=2)
    os.environ["NCCL_NVLS_ENABLE"] = "0"
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", 0))
    try:
        chi1, hist1 = dbim_dist.dbim(ops, inc_t, mes, float(s.opts.k0), iterations=2, group=dist.group.WORLD)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    assert torch.equal(chi1, chi0)
    assert [h["misfit"] for h in hist1] == [h["misfit"] for h in hist0]
