"""Tikhonov regularisation and measurement noise of the inversion path.

(1) isg_dbim with regular > 0: the reference adds regular^2 chi to the
    gradient and to the Born step of every transmitter (mom.cpp:32, 268-269,
    359-360).  Against the FP64 oracle's inversion loop (orc_dbim) with the same
    weight on 128 x 128 pixels (three ellipses eps_r in [1.1, 1.3], 8 plane
    waves, 32 far-field receivers, 3 Polak-Ribiere iterations, inner solves to
    1e-6): history to 1e-3 relative, contrast to 2e-3, as the unregularised
    parity test against the reference's own driver.  regular = 1 moves the
    result well beyond that tolerance (the oracle's iteration-3 misfit is 0.106
    against 0.094 without it), so the term is exercised.
(2) isg_measure with noise > 0 adds complex Gaussian noise of standard
    deviation noise * ||mes|| / sqrt(2 ntx numrx) per real component: the same
    seed gives the same data, and the added noise has that size and no bias.
"""
import numpy as np
import pytest

import isg
from _oracle import Oracle, oracle_dbim, rel

pytestmark = pytest.mark.gpu
LEVEL, NTX, NRX, ITER, TOL, REG = 5, 8, 32, 3, 1e-6, 1.0


def setup(max_rhs=NTX):
    import torch
    s = isg.Solver(LEVEL, numrx=NRX, max_rhs=max_rhs)
    chi_tree = s.raster_to_tree(s.phantom(seed=77, count=3, axis=(1.0, 2.5), eps=(1.1, 1.3)))
    inc = s.plane_waves(NTX, order=isg.ORDER_TREE)
    return s, chi_tree, inc, torch.from_numpy(chi_tree).cuda(), torch.from_numpy(inc.astype(np.complex64)).cuda()


@pytest.mark.parametrize("engine", [isg.ENGINE_SIMT, isg.ENGINE_TENSOR])
def test_regularised_inversion_matches_the_oracle(engine):
    s, chi_tree, inc, chi_d, inc_d = setup()
    o = Oracle(LEVEL, numrx=NRX)
    want_chi, want_hist, want_alpha, _ = oracle_dbim(o, inc, chi_tree, ITER, REG, TOL, 500)
    _, free_hist, _, _ = oracle_dbim(o, inc, chi_tree, ITER, 0.0, TOL, 500)
    assert abs(free_hist[-1, 0] - want_hist[-1, 0]) > 0.05 * want_hist[-1, 0]  # the weight matters

    mes = s.measure(inc_d, chi_d, order=isg.ORDER_TREE, tol=TOL, engine=engine)
    chi, hist = s.dbim(inc_d, mes, chi_true=chi_d, iterations=ITER, regular=REG, order=isg.ORDER_TREE, tol=TOL,
                       engine=engine)
    got = np.array([[h["misfit"], h["object_error"], h["reg_cost"], h["grad_norm"], h["object_norm"]] for h in hist])
    for col in range(5):
        m = np.abs(want_hist[:, col]) > 0
        err = np.max(np.abs(got[m, col] - want_hist[m, col]) / np.abs(want_hist[m, col]))
        assert err < 1e-3, (col, got[:, col], want_hist[:, col])
    alpha = np.array([h["alpha"] for h in hist[1:]])
    assert np.max(np.abs(alpha - want_alpha) / np.abs(want_alpha)) < 1e-3
    assert rel(chi.cpu().numpy(), want_chi) < 2e-3


def test_measurement_noise_has_the_stated_size():
    s, chi_tree, inc, chi_d, inc_d = setup()
    clean = s.measure(inc_d, chi_d, order=isg.ORDER_TREE, tol=TOL, engine=isg.ENGINE_TENSOR).cpu().numpy()
    noisy = [s.measure(inc_d, chi_d, noise=0.01, seed=sd, order=isg.ORDER_TREE, tol=TOL,
                       engine=isg.ENGINE_TENSOR).cpu().numpy() for sd in (5, 5, 6)]
    assert np.array_equal(noisy[0], noisy[1])          # seeded
    assert not np.array_equal(noisy[0], noisy[2])
    M = NTX * NRX
    sigma = 0.01 * np.linalg.norm(clean) / np.sqrt(2 * M)
    for n in (noisy[0], noisy[2]):
        d = (n.astype(np.complex128) - clean.astype(np.complex128)).ravel()
        parts = np.concatenate([d.real, d.imag])       # 2M real samples of N(0, sigma^2)
        ratio = np.std(parts) / sigma
        assert abs(ratio - 1) < 4 * np.sqrt(1 / (2 * 2 * M)) + 0.01, ratio
        assert abs(np.mean(parts)) < 4 * sigma / np.sqrt(2 * M)
        assert abs(np.linalg.norm(d) / np.linalg.norm(clean) - 0.01) < 0.002
