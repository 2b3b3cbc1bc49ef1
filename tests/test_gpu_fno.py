"""The learned warm start on the GPU: forward pass, loss and gradient of the
CUDA kernels against the FP64 numpy oracle, and a trained network's effect on
the forward solves it seeds.

Tolerances, FP32 network (tensor=False): outputs 1e-4 relative and gradients
1e-3 relative to their norm (the network's Born-field input comes from the
FP32 MLFMA, which agrees with the FP64 oracle operator to ~1e-5).  BF16
network (tensor=True, the default: tcgen05 products of BF16 operands with FP32
accumulation): every operand is rounded to 8 significant bits (relative 2^-9)
before its product, through up to ten chained products, so outputs are held to
3e-2 and gradients to 5e-2 of their norm (2e-1 per parameter block) - a
misplaced element of a tensor-core tile gives errors of order 1."""
import numpy as np
import pytest

import isg
from _fno_oracle import FnoOracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


def cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).cuda()


TOL = {False: dict(out=1e-4, loss=1e-4, grad=1e-3, block=1e-2),
       True: dict(out=3e-2, loss=3e-2, grad=5e-2, block=2e-1)}


@pytest.mark.parametrize("tensor", [False, True])
def test_fno_forward_loss_and_gradient_match_the_oracle(tensor):
    from _oracle import Oracle
    C, M, L, S = 4, 3, 2, 2
    t = TOL[tensor]
    s = isg.Solver(3, numrx=16, max_rhs=4, device=0)  # 32 x 32 pixels
    s.setup_gpu()
    orc = Oracle(3, numrx=16)
    um = s.host_table("unkmap")
    s.fno_create(width=C, modes=M, layers=L, batch=S, seed=5, tensor=tensor)
    o = FnoOracle(N=s.side, C=C, M=M, L=L, k0=float(s.opts.k0))
    assert isg.lib().isg_fno_param_count(s._h) == o.nparam
    rng = np.random.default_rng(11)
    p = rng.normal(0, 0.3, o.nparam).astype(np.float32)
    s.fno_set_params(p)
    assert np.array_equal(s.fno_params(0), p)
    n, U = 3, s.numunk
    chi = np.stack([s.phantom(seed=40 + j, count=2, eps=(1.2, 1.8), tand_max=0.1) for j in range(n)])
    G = (2 * np.pi) ** 2 * chi
    B = np.stack([np.exp(1j * 2 * np.pi * rng.uniform() * np.arange(U) / U) for _ in range(n)])
    Uf = B + 0.2 * (rng.normal(size=(n, U)) + 1j * rng.normal(size=(n, U)))
    G, B, Uf = (a.astype(np.complex64).astype(np.complex128) for a in (G, B, Uf))
    # first Born fields from the FP64 oracle operator (the GPU's FP32 MLFMA agrees to ~1e-5)
    S1 = np.stack([B[j] - orc.matvec(s.raster_to_tree(B[j]), s.raster_to_tree(G[j]))[um] for j in range(n)])
    x = s.fno_apply(cuda(G), cuda(B), order=isg.ORDER_RASTER).cpu().numpy()
    for j in range(n):
        want, _ = o.forward(p.astype(np.float64), G[j], B[j], S1[j])
        assert rel(x[j], want) < t["out"], (j, rel(x[j], want))
    loss = s.fno_grad(cuda(G), cuda(B), cuda(Uf), order=isg.ORDER_RASTER)
    want_loss, want_grad = o.loss_grad(p.astype(np.float64), G, B, S1, Uf)
    assert abs(loss - want_loss) <= t["loss"] * want_loss, (loss, want_loss)
    got = s.fno_params(1).astype(np.float64)
    assert rel(got, want_grad) < t["grad"], rel(got, want_grad)
    for name, (off, cnt) in o.lay.items():
        assert rel(got[off:off + cnt], want_grad[off:off + cnt]) < t["block"], (name, rel(got[off:off + cnt],
                                                                                          want_grad[off:off + cnt]))
    # tree order is the same network on reordered vectors
    xt = s.fno_apply(cuda(s.raster_to_tree(G)), cuda(s.raster_to_tree(B)), order=isg.ORDER_TREE).cpu().numpy()
    assert rel(xt, s.raster_to_tree(x)) < 1e-6


@pytest.mark.parametrize("tensor", [False, True])
def test_fno_residual_loss_gradient_matches_the_oracle(tensor):
    from _oracle import Oracle
    C, M, L = 4, 3, 2
    t = TOL[tensor]
    s = isg.Solver(4, numrx=16, max_rhs=2, device=0)  # 64 x 64 pixels
    s.setup_gpu()
    s.fno_create(width=C, modes=M, layers=L, batch=2, seed=6, tensor=tensor)
    fo = FnoOracle(N=s.side, C=C, M=M, L=L, k0=float(s.opts.k0))
    orc = Oracle(4, numrx=16)
    um = s.host_table("unkmap")
    rng = np.random.default_rng(12)
    p = rng.normal(0, 0.2, fo.nparam).astype(np.float32)
    s.fno_set_params(p)
    n, U = 2, s.numunk
    G = np.stack([(2 * np.pi) ** 2 * s.phantom(seed=70 + j, count=2, eps=(1.1, 1.4)) for j in range(n)])
    B = s.plane_waves(16, first=3, count=n, order=isg.ORDER_RASTER)
    G, B = G.astype(np.complex64).astype(np.complex128), B.astype(np.complex64).astype(np.complex128)

    def apply(x, g, herm):
        return orc.matvec(s.raster_to_tree(x), s.raster_to_tree(g), herm)[um]

    want_loss, want_grad = fo.residual_loss_grad(p.astype(np.float64), G, B, lambda x, g: apply(x, g, False),
                                                 lambda x, g: apply(x, g, True))
    loss = s.fno_grad(cuda(G), cuda(B), None, order=isg.ORDER_RASTER)
    assert abs(loss - want_loss) <= t["loss"] * want_loss, (loss, want_loss)
    assert rel(s.fno_params(1).astype(np.float64), want_grad) < t["grad"]


def test_bf16_network_matches_fp32_network_at_512():
    """The default network (width 32, 12 x 24 modes, 4 layers) at 512 x 512
    pixels, where the tensor-core GEMMs run several row and column tiles and
    split K over CTAs: BF16 outputs and gradients against the FP32 network
    with the same parameters."""
    s = isg.Solver(7, numrx=16, max_rhs=4, device=0)
    s.setup_gpu()
    rng = np.random.default_rng(21)
    n = 4
    G = np.stack([(2 * np.pi) ** 2 * s.raster_to_tree(s.phantom(seed=300 + j, count=8, eps=(1.1, 1.5)))
                  for j in range(n)])
    B = s.line_sources(128, 40.0, first=5, count=n)
    Uf = B + 0.3 * (rng.normal(size=B.shape) + 1j * rng.normal(size=B.shape))
    out = {}
    for tensor in (False, True):
        s.fno_create(seed=3, tensor=tensor)
        if not tensor:
            p = s.fno_params(0)
        s.fno_set_params(p)
        x = s.fno_apply(cuda(G), cuda(B)).cpu().numpy() - B
        loss = s.fno_grad(cuda(G), cuda(B), cuda(Uf))
        out[tensor] = (x, loss, s.fno_params(1).astype(np.float64))
    (x32, l32, g32), (x16, l16, g16) = out[False], out[True]
    print("bf16 vs fp32: network output", rel(x16, x32), "loss", abs(l16 - l32) / l32, "gradient", rel(g16, g32))
    assert rel(x16, x32) < 3e-2
    assert abs(l16 - l32) <= 3e-2 * l32
    assert rel(g16, g32) < 5e-2


def _problems(s, seeds, angles, ntx=64):
    """(g, b) pairs in tree order: contrasts from seeds, plane waves at the given Tx indices."""
    G, B = [], []
    for sd in seeds:
        chi = s.raster_to_tree(s.phantom(seed=sd, count=3, axis=(0.6, 1.6), eps=(1.1, 1.5)))
        for a in angles(sd):
            G.append((2 * np.pi) ** 2 * chi)
            B.append(s.plane_waves(ntx, first=a, count=1)[0])
    return np.array(G), np.array(B)


def test_trained_warm_start_reduces_iterations():
    import torch
    s = isg.Solver(4, numrx=16, max_rhs=64, device=0)  # 64 x 64 pixels, 6.4 wavelengths
    s.setup_gpu()
    rng = np.random.default_rng(5)
    Gtr, Btr = _problems(s, range(100, 132), lambda sd: rng.choice(64, 2, replace=False))
    Gte, Bte = _problems(s, range(900, 908), lambda sd: rng.choice(64, 2, replace=False))
    # solver-generated total fields for training
    gt, bt = cuda(Gtr), cuda(Btr)
    ut = torch.zeros_like(bt)
    for j in range(0, len(bt), 64):
        info = s.bicgs(ut[j:j + 64], gt[j:j + 64], bt[j:j + 64], tol=1e-6, engine=isg.ENGINE_TENSOR)
        assert all(i["status"] == 0 for i in info)
    ge, be = cuda(Gte), cuda(Bte)

    def iterations(guess):
        x = torch.zeros_like(be)
        info = s.bicgs(x, ge, be, tol=1e-5, guess=guess, engine=isg.ENGINE_TENSOR)
        assert all(i["status"] == 0 and i["true_residual"] <= 1e-5 for i in info), info
        return float(np.mean([i["iterations"] for i in info]))

    def train(steps, supervised):
        first = loss = None
        idx = np.arange(len(bt))
        for step in range(steps):
            lr = 3e-3 if step < 2 * steps // 3 else 1e-3
            if supervised:
                sel = torch.from_numpy(rng.choice(idx, 16, replace=False)).cuda()
                loss = s.fno_train_step(gt[sel], bt[sel], ut[sel], lr=lr)
            else:  # residual loss on fresh problems: no solved fields needed
                Gf, Bf = _problems(s, rng.integers(10 ** 6, size=8), lambda sd: rng.choice(64, 2, replace=False))
                loss = s.fno_train_step(cuda(Gf), cuda(Bf), None, lr=lr)
            first = loss if first is None else first
        return first, loss

    zero = iterations(isg.GUESS_ZERO)
    res = {}
    for name, plan in (("field", [(600, True)]), ("residual", [(600, False)])):
        s.fno_create(width=24, modes=8, layers=4, batch=16, seed=2)
        hist = [train(n, sup) for n, sup in plan]
        res[name] = (hist, s.fno_grad(ge, be, None), iterations(isg.GUESS_LEARNED))
    print("fno zero-start iterations", zero)
    for k, v in res.items():
        print("fno", k, "train", v[0], "held-out initial residual^2", v[1], "iterations", v[2])
    hist, _, its = res["field"]
    assert hist[0][1] < 0.5 * hist[0][0]
    assert its < zero


def test_learned_seeds_leave_the_inversion_unchanged():
    """isg_dbim with ISG_GUESS_LEARNED seeds the forward solves from the
    network and the adjoint solves through it (x0 = conj(g N(g, conj(y)))).
    Every solve still runs to the same true residual, so the inversion's
    contrast and misfit history equal the zero-start ones to the solver
    tolerance; the seeded adjoint solves start from a non-zero residual."""
    import torch
    level, ntx, nrx, radius = 5, 8, 64, 40.0
    s = isg.Solver(level, numrx=nrx, max_rhs=ntx, device=0)  # 128 x 128 pixels
    s.set_nearfield_receivers(radius)
    inc = cuda(s.line_sources(ntx, radius))
    chi_true = torch.from_numpy(s.raster_to_tree(s.phantom(seed=91, count=3, axis=(1.0, 2.5), eps=(1.1, 1.4)))).cuda()
    mes = s.measure(inc, chi_true, tol=1e-6, engine=isg.ENGINE_TENSOR)
    s.fno_create(width=8, modes=4, layers=2, batch=4, seed=7)
    out = {}
    for name, guess in (("zero", isg.GUESS_ZERO), ("learned", isg.GUESS_LEARNED)):
        chi, hist = s.dbim(inc, mes, chi_true=chi_true, iterations=2, regular=0.2, tol=1e-6,
                           engine=isg.ENGINE_TENSOR, guess=guess)
        out[name] = (chi.cpu().numpy(), np.array([h["misfit"] for h in hist]), hist[-1]["iterations"])
    (cz, mz, iz), (cl, ml, il) = out["zero"], out["learned"]
    print("dbim bicgs iterations: zero start", iz, "learned seeds", il)
    assert rel(cl, cz) < 1e-3
    assert np.max(np.abs(ml - mz) / mz) < 1e-3
    assert il != iz  # the seeds reached the solves
