"""The FP64 numpy restatement of the learned warm start: its hand-written
gradient against central finite differences (CPU only)."""
import numpy as np

from _fno_oracle import FnoOracle


def test_fno_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    o = FnoOracle(N=8, C=3, M=2, L=2)
    p = rng.normal(0, 0.4, o.nparam)
    G = (rng.normal(size=(2, 64)) + 1j * rng.normal(size=(2, 64))) * 8
    B = np.exp(1j * rng.uniform(0, 2 * np.pi, (2, 64)))
    U = B + 0.3 * (rng.normal(size=(2, 64)) + 1j * rng.normal(size=(2, 64)))
    S1 = 0.5 * (rng.normal(size=(2, 64)) + 1j * rng.normal(size=(2, 64)))
    loss, grad = o.loss_grad(p, G, B, S1, U)
    assert abs(loss - o.loss(p, G, B, S1, U)) < 1e-12
    used = [i for name, (off, n) in o.lay.items() for i in range(off, off + n)]
    h = 1e-6
    for i in rng.choice(used, 40, replace=False):
        q = p.copy()
        q[i] += h
        lp = o.loss(q, G, B, S1, U)
        q[i] -= 2 * h
        lm = o.loss(q, G, B, S1, U)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_fno_layout_is_padded_to_four_floats():
    o = FnoOracle(N=16, C=5, M=3, L=3)
    offs = sorted(off for off, _ in o.lay.values())
    assert all(off % 4 == 0 for off in offs)
    assert o.nparam % 4 == 0
