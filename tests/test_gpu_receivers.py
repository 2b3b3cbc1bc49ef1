"""Near-field receivers (the reference's commented dense form,
setup_born.cpp:52-60): go[m][n] = integrate(rx_m, pos_n) for receivers on a
circle, applied as tcgen05 GEMMs (csrc/isg_rxnear.cu), against the FP64
oracle's dense operator built with its own integrate (integrate.cpp:15-41),
whose entries are pinned here against the reference's compiled integrate.

Bars: 2e-5 relative for the operators (complex64 data, 3xFP16 products); for
the inversion with line-source transmitters and near-field receivers on a
40-wavelength circle (the config-5 geometry on 128 x 128 pixels), history to
1e-3 and contrast to 2e-3 against the oracle's inversion, as the far-field
parity tests."""
import math

import numpy as np
import pytest

import isg
from _oracle import Oracle, Reference, oracle_dbim, rel

pytestmark = pytest.mark.gpu


def cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).cuda()


@pytest.mark.parametrize("level,numrx,radius,nrhs", [(4, 32, 10.0, 3), (3, 200, 6.0, 130)])
def test_receivers_match_the_dense_oracle(level, numrx, radius, nrhs):
    s = isg.Solver(level, numrx=numrx, max_rhs=nrhs, device=0)
    s.set_nearfield_receivers(radius)
    o = Oracle(level, numrx=numrx)
    o.set_nearfield(radius)
    rng = np.random.default_rng(level)
    X = rng.standard_normal((nrhs, s.numunk)) + 1j * rng.standard_normal((nrhs, s.numunk))
    X[1] *= 1e-3  # per-RHS scaling
    Rv = rng.standard_normal((nrhs, numrx)) + 1j * rng.standard_normal((nrhs, numrx))
    X32, R32 = X.astype(np.complex64).astype(np.complex128), Rv.astype(np.complex64).astype(np.complex128)
    got = s.receive(cuda(X)).cpu().numpy()
    goth = s.receiveh(cuda(Rv)).cpu().numpy()
    for j in range(nrhs):
        assert rel(got[j], o.receive(X32[j])) < 2e-5, j
        assert rel(goth[j], o.receiveh(R32[j])) < 2e-5, j


def test_oracle_dense_rows_follow_the_reference_integrate():
    if not Reference.available():
        pytest.skip("oracle/_ref not built")
    o = Oracle(4, numrx=8)
    o.set_nearfield(10.0)
    ref = Reference(4, 2 * math.pi, 8)
    pos = o.pos()
    rng = np.random.default_rng(1)
    for m in (0, 3, 7):
        for n in rng.integers(o.U, size=5):
            e = np.zeros(o.U, np.complex128)
            e[n] = 1
            want = ref.integrate(10.0 * complex(math.cos(2 * math.pi * m / 8), math.sin(2 * math.pi * m / 8)), pos[n])
            assert abs(o.receive(e)[m] - want) <= 1e-12 * abs(want)


def test_nearfield_inversion_matches_the_oracle():
    """Line sources and 64 receivers on a 40-wavelength circle, 128 x 128
    pixels, 8 transmitters, 3 Polak-Ribiere iterations, Tikhonov weight 0.5,
    inner solves to 1e-6."""
    level, ntx, nrx, radius, iters, tol, reg = 5, 8, 64, 40.0, 3, 1e-6, 0.5
    s = isg.Solver(level, numrx=nrx, max_rhs=ntx, device=0)
    s.set_nearfield_receivers(radius)
    o = Oracle(level, numrx=nrx)
    o.set_nearfield(radius)
    chi_tree = s.raster_to_tree(s.phantom(seed=81, count=3, axis=(1.0, 2.5), eps=(1.1, 1.4)))
    inc = s.line_sources(ntx, radius, order=isg.ORDER_TREE)
    import torch
    chi_d = torch.from_numpy(chi_tree).cuda()
    want_chi, want_hist, want_alpha, _ = oracle_dbim(o, inc, chi_tree, iters, reg, tol, 500)
    mes = s.measure(cuda(inc), chi_d, order=isg.ORDER_TREE, tol=tol, engine=isg.ENGINE_TENSOR)
    want_mes = np.stack([o.receive(chi_tree * (2 * np.pi) ** 2 * o.bicgs(chi_tree * (2 * np.pi) ** 2, b, False, tol,
                                                                          500)[0]) for b in inc[:2]])
    assert rel(mes.cpu().numpy()[:2], want_mes) < 1e-4
    chi, hist = s.dbim(cuda(inc), mes, chi_true=chi_d, iterations=iters, regular=reg, order=isg.ORDER_TREE, tol=tol,
                       engine=isg.ENGINE_TENSOR)
    got = np.array([[h["misfit"], h["object_error"], h["reg_cost"], h["grad_norm"], h["object_norm"]] for h in hist])
    print("near-field inversion misfit", got[:, 0], "oracle", want_hist[:, 0])
    assert got[-1, 0] < 0.5 * got[0, 0]  # the inversion makes progress
    for col in range(5):
        m = np.abs(want_hist[:, col]) > 0
        err = np.max(np.abs(got[m, col] - want_hist[m, col]) / np.abs(want_hist[m, col]))
        assert err < 1e-3, (col, got[:, col], want_hist[:, col])
    assert rel(chi.cpu().numpy(), want_chi) < 2e-3
