"""Batched BiCGSTAB on the GPU against the reference's golden solves and an
FP64 oracle solve converged far below the tolerance.

Bar: every GPU solve reaches true relative residual <= tol (1e-5) and its field
is within 1e-4 (relative L2) of the FP64 oracle field."""
import os

import numpy as np
import pytest

import isg
from _oracle import Oracle, disk_contrast, plane_wave, rel

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def torch_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).cuda()


def host(t):
    return t.detach().cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("engine", [isg.ENGINE_SIMT, isg.ENGINE_TENSOR])
@pytest.mark.parametrize("name", ["golden_l4.npz", "golden_l5.npz"])
@pytest.mark.parametrize("hermitian", [False, True])
def test_bicgs_matches_reference(name, hermitian, engine):
    d = dict(np.load(os.path.join(GOLDEN, name)))
    s = isg.Solver(int(d["level"]), numrx=int(d["numrx"]))
    o = Oracle(int(d["level"]), numrx=int(d["numrx"]))
    g, b = d["g"], d["b"]
    x = torch_dev(np.zeros_like(b))
    info = s.bicgs(x, torch_dev(g), torch_dev(b), hermitian=hermitian, tol=1e-5, engine=engine)[0]
    assert info["status"] == 0, info
    assert info["true_residual"] <= 1e-5
    ref_iters = int(d["bicgs_adj_iters" if hermitian else "bicgs_fwd_iters"])
    assert abs(info["iterations"] - ref_iters) <= 2, (info, ref_iters)
    xt, _, _ = o.bicgs(g, b, hermitian, 1e-11, 500)
    assert rel(host(x), xt) < 1e-4
    assert rel(host(x), d["bicgs_adj" if hermitian else "bicgs_fwd"]) < 1e-4


def test_batched_masks_uneven_difficulty():
    """RHS of different difficulty converge independently in one batch."""
    s = isg.Solver(5, max_rhs=6)
    o = Oracle(5)
    pos = o.pos()
    g = disk_contrast(pos, radius=3.0, chi=0.4)
    B = np.stack([plane_wave(pos, 2 * np.pi * j / 6) * (10.0 ** (j - 3)) for j in range(6)])
    B[2] = 0  # zero RHS: converged before the first iteration (bicgs.cpp:111-122)
    X = torch_dev(np.zeros_like(B))
    infos = s.bicgs(X, torch_dev(g), torch_dev(B), tol=1e-5)
    Xh = host(X)
    for j, inf in enumerate(infos):
        assert inf["status"] == 0, (j, inf)
        if j == 2:
            assert inf["iterations"] == 0 and np.abs(Xh[j]).max() == 0
            continue
        assert inf["true_residual"] <= 1e-5
        xt, _, _ = o.bicgs(g, B[j], False, 1e-11, 500)
        assert rel(Xh[j], xt) < 1e-4


@pytest.mark.parametrize("engine", [isg.ENGINE_SIMT, isg.ENGINE_TENSOR])
def test_converged_columns_are_skipped_without_changing_the_others(engine):
    """512 x 512 pixels (MLFMA levels 2 .. 6, so the banded tensor-core M2M and
    the tiled L2L run at the coarse levels).  Two RHS solved in a batch of
    four whose other two are zero (inactive from the start, so every tree
    block holding only their columns returns at once, and mixed blocks skip
    them) give the same fields, iteration counts and residuals bit for bit as
    the two solved on their own."""
    import torch
    s = isg.Solver(7, numrx=16, max_rhs=4)
    chi = s.raster_to_tree(s.phantom(seed=77, count=4, axis=(1.0, 3.0), eps=(1.1, 1.6)))
    g = torch.from_numpy(((2 * np.pi) ** 2 * chi).astype(np.complex64)).cuda()
    b2 = torch.from_numpy(s.plane_waves(16, first=3, count=2).astype(np.complex64)).cuda()
    b4 = torch.zeros((4, s.numunk), dtype=torch.complex64, device="cuda")
    b4[0], b4[2] = b2[0], b2[1]
    opts = isg.default_solve_opts(tol=1e-5, maxit=400, engine=engine, check_every=2)
    x2, x4 = torch.zeros_like(b2), torch.zeros_like(b4)
    inf2 = s.bicgs(x2, g, b2, opts=opts)
    inf4 = s.bicgs(x4, g, b4, opts=opts)
    torch.cuda.synchronize()
    assert [i["iterations"] for i in inf4] == [inf2[0]["iterations"], 0, inf2[1]["iterations"], 0]
    assert all(i["status"] == 0 for i in inf4) and all(0 <= i["true_residual"] <= 1e-5 for i in inf2)
    assert [inf4[0]["true_residual"], inf4[2]["true_residual"]] == [i["true_residual"] for i in inf2]
    assert torch.equal(x4[0], x2[0]) and torch.equal(x4[2], x2[1])
    assert not x4[1].abs().max().item() and not x4[3].abs().max().item()


def test_caller_guess_and_iteration_cap():
    s = isg.Solver(4, max_rhs=2)
    o = Oracle(4)
    pos = o.pos()
    g = disk_contrast(pos, radius=1.5, chi=0.5)
    b = plane_wave(pos, 0.7)
    xt, _, _ = o.bicgs(g, b, False, 1e-11, 500)
    # a good initial guess needs fewer iterations
    x = torch_dev(xt * (1 + 1e-3))
    inf = s.bicgs(x, torch_dev(g), torch_dev(b), guess=isg.GUESS_CALLER)[0]
    x0 = torch_dev(np.zeros_like(b))
    inf0 = s.bicgs(x0, torch_dev(g), torch_dev(b))[0]
    assert inf["status"] == 0 and inf["iterations"] < inf0["iterations"]
    assert rel(host(x), xt) < 1e-4
    # the iteration cap is reported per RHS
    x1 = torch_dev(np.zeros_like(b))
    inf1 = s.bicgs(x1, torch_dev(g), torch_dev(b), maxit=2, true_residual=0)[0]
    assert inf1["status"] == 1 and inf1["iterations"] == 2


def test_nonfinite_input_is_reported():
    """A NaN in one RHS is flagged for that RHS only; the other converges."""
    s = isg.Solver(4, max_rhs=2)
    o = Oracle(4)
    pos = o.pos()
    g = disk_contrast(pos, radius=1.5, chi=0.3)
    B = np.stack([plane_wave(pos, 0.1), plane_wave(pos, 0.2)])
    B[1, 17] = np.nan
    X = torch_dev(np.zeros_like(B))
    infos = s.bicgs(X, torch_dev(g), torch_dev(B))
    assert infos[0]["status"] == 0
    assert infos[1]["status"] == 3


def test_graph_replay_matches_direct_launches():
    """The iteration block replayed as a CUDA graph (captured on the first poll,
    reused by the next call with the same buffers) gives the same iterations
    and fields as launching every kernel, and counts the same launches."""
    import torch
    s = isg.Solver(5, numrx=16, max_rhs=3, device=0)
    s.setup_gpu()  # the table kernels of set-up stay out of the counted launches
    o = Oracle(5)
    pos = o.pos()
    g = torch.from_numpy(disk_contrast(pos, radius=2.0, chi=0.4).astype(np.complex64)).cuda()
    b = torch.from_numpy(np.stack([plane_wave(pos, a) for a in (0.0, 1.0, 2.0)]).astype(np.complex64)).cuda()
    stream = torch.cuda.Stream()
    runs = []
    for graph in (0, 1, 1):
        x = torch.zeros_like(b)
        n0 = isg.kernel_launches()
        info = s.bicgs(x, g, b, tol=1e-6, engine=isg.ENGINE_TENSOR, check_every=3, graph=graph, stream=stream)
        stream.synchronize()
        runs.append((x.cpu().numpy(), [i["iterations"] for i in info], isg.kernel_launches() - n0))
        assert all(i["status"] == 0 for i in info)
    (x0, it0, l0), (x1, it1, l1), (x2, it2, l2) = runs
    assert it0 == it1 == it2
    assert l0 == l1 == l2
    assert np.array_equal(x0, x1) and np.array_equal(x1, x2)
