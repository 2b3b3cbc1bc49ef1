"""The CUDA MLFMA operator through the C ABI against the FP64 oracle and the
reference's golden vectors.  Complex64 arithmetic: operator outputs agree to
~1e-6 relative; the tolerance written here is 2e-5."""
import os

import numpy as np
import pytest

import isg
from _oracle import Oracle, disk_contrast, rel

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 2e-5


def torch_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).cuda()


def host(t):
    return t.detach().cpu().numpy().astype(np.complex128)


@pytest.fixture(scope="module", params=["golden_l4.npz", "golden_l5.npz"])
def case(request):
    d = dict(np.load(os.path.join(GOLDEN, request.param)))
    s = isg.Solver(int(d["level"]), float(d["k0"]), numrx=int(d["numrx"]), max_rhs=4)
    s.setup_gpu()
    return d, s


ENGINES = [isg.ENGINE_SIMT, isg.ENGINE_TENSOR]


@pytest.mark.parametrize("engine", ENGINES)
def test_mlfma_matches_reference(case, engine):
    d, s = case
    x = torch_dev(d["x"])
    assert rel(host(s.mlfma(x, engine=engine)), d["mlfma"]) < TOL
    assert rel(host(s.mlfmah(x, engine=engine)), d["mlfmah"]) < TOL


def test_mlfma_against_dense_rows(case):
    d, s = case
    r = host(s.mlfma(torch_dev(d["x"])))
    assert rel(r[d["dense_rows"]], d["dense"]) < 3e-5


@pytest.mark.parametrize("engine", ENGINES)
def test_matvec_forward_and_adjoint(case, engine):
    d, s = case
    o = Oracle(int(d["level"]), numrx=int(d["numrx"]))
    x, g = d["x"], d["g"]
    for h in (False, True):
        y = host(s.matvec(torch_dev(x), torch_dev(g), hermitian=h, engine=engine))
        assert rel(y, o.matvec(x, g, h)) < TOL


def test_aggregate_and_aggregateh(case):
    d, s = case
    assert rel(host(s.aggregate(torch_dev(d["x"]))), d["aggregate"]) < TOL
    assert rel(host(s.aggregateh(torch_dev(d["rx"]))), d["aggregateh"]) < TOL


def test_batched_rhs_equal_single(case):
    d, s = case
    rng = np.random.default_rng(11)
    X = rng.standard_normal((4, s.numunk)) + 1j * rng.standard_normal((4, s.numunk))
    g = d["g"]
    Yb = host(s.matvec(torch_dev(X), torch_dev(g)))
    for j in range(4):
        yj = host(s.matvec(torch_dev(X[j]), torch_dev(g)))
        assert rel(Yb[j], yj) < 1e-6
    # per-RHS contrasts (g_stride = U)
    G = np.stack([g * (1 + 0.1 * j) for j in range(4)])
    Yg = host(s.matvec(torch_dev(X), torch_dev(G)))
    o = Oracle(int(d["level"]), numrx=int(d["numrx"]))
    for j in range(4):
        assert rel(Yg[j], o.matvec(X[j], G[j])) < TOL


def test_orders_round_trip(case):
    d, s = case
    x = torch_dev(d["x"])
    for o in (isg.ORDER_RASTER, isg.ORDER_BLOCKED):
        y = s.reorder(x, isg.ORDER_TREE, o)
        back = s.reorder(y, o, isg.ORDER_TREE)
        assert np.array_equal(host(back), host(x))
    # the operator gives the same answer in every ordering
    r_tree = host(s.mlfma(x))
    xr = s.reorder(x, isg.ORDER_TREE, isg.ORDER_RASTER)
    r_r = s.mlfma(xr, order=isg.ORDER_RASTER)
    assert rel(host(s.reorder(r_r, isg.ORDER_RASTER, isg.ORDER_TREE)), r_tree) < 1e-6


def test_linearity(case):
    d, s = case
    rng = np.random.default_rng(3)
    a = rng.standard_normal(s.numunk) + 1j * rng.standard_normal(s.numunk)
    b = rng.standard_normal(s.numunk) + 1j * rng.standard_normal(s.numunk)
    ra, rb = host(s.mlfma(torch_dev(a))), host(s.mlfma(torch_dev(b)))
    rab = host(s.mlfma(torch_dev(2 * a - 3j * b)))
    assert rel(rab, 2 * ra - 3j * rb) < 1e-5


def test_smallest_grid_level3():
    o = Oracle(3)
    s = isg.Solver(3)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(o.U) + 1j * rng.standard_normal(o.U)
    assert rel(host(s.mlfma(torch_dev(x))), o.mlfma(x)) < TOL
    g = disk_contrast(o.pos(), radius=0.8)
    assert rel(host(s.matvec(torch_dev(x), torch_dev(g), hermitian=True)), o.matvec(x, g, True)) < TOL


@pytest.mark.parametrize("level", [3, 6, 7])
def test_tensor_engine_matches_simt(level):
    """3xFP16 tcgen05 leaf stages agree with complex-FP32 SIMT on random batches,
    including the tile edges of grids smaller than one 16 x 8 leaf tile."""
    s = isg.Solver(level, max_rhs=3)
    rng = np.random.default_rng(level)
    U = s.numunk
    X = rng.standard_normal((3, U)) + 1j * rng.standard_normal((3, U))
    X[1] *= 1e-3  # per-tile scaling must follow the magnitude
    G = (rng.standard_normal(U) + 1j * rng.standard_normal(U)) * 10
    xs, gs = torch_dev(X), torch_dev(G)
    for h in (False, True):
        a = host(s.matvec(xs, gs, hermitian=h, engine=isg.ENGINE_SIMT, order=isg.ORDER_BLOCKED))
        b = host(s.matvec(xs, gs, hermitian=h, engine=isg.ENGINE_TENSOR, order=isg.ORDER_BLOCKED))
        for j in range(3):
            assert rel(b[j], a[j]) < 5e-6, (h, j, rel(b[j], a[j]))
    a = host(s.mlfma(xs, engine=isg.ENGINE_SIMT))
    b = host(s.mlfma(xs, engine=isg.ENGINE_TENSOR))
    for j in range(3):
        assert rel(b[j], a[j]) < 5e-6
