"""Large grids: 2048^2 and 4096^2 pixels (204.8 and 409.6 wavelengths, 9 and
10 MLFMA levels) on a Gaussian-random-field contrast (correlation length 2
wavelengths, eps_r in [1.0, 1.1]; with eps_r up to 1.6 BiCGSTAB still sits
near residual 1e-3 after 6000 iterations at 2048^2, a property of the
system, not of this implementation).  Every RHS reaches the true residual 1e-5
with the tensor-core engine, and its field agrees with the complex-FP32 SIMT
engine's, an independent implementation of the leaf stages, to 1e-4
relative (both solves stop at residual 1e-5)."""
import numpy as np
import pytest

import isg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level", [9, 10])
def test_large_grid_solves(level):
    import torch
    s = isg.Solver(level, numrx=32, max_rhs=2, device=0)
    s.setup_gpu()
    chi = s.phantom(seed=4000 + level, kind=1, eps=(1.0, 1.1), corr_len=2.0)
    g = torch.from_numpy((s.opts.k0 ** 2 * s.raster_to_tree(chi)).astype(np.complex64)).cuda()
    b = torch.from_numpy(s.plane_waves(8, first=1, count=2).astype(np.complex64)).cuda()
    xs = {}
    for eng in (isg.ENGINE_TENSOR, isg.ENGINE_SIMT):
        x = torch.zeros_like(b)
        info = s.bicgs(x, g, b, tol=1e-5, maxit=2000, engine=eng, check_every=4)
        assert all(i["status"] == 0 and 0 <= i["true_residual"] <= 1e-5 for i in info), info
        xs[eng] = x
        print("level", level, "engine", eng, "iterations", [i["iterations"] for i in info])
    d = torch.linalg.vector_norm(xs[isg.ENGINE_TENSOR] - xs[isg.ENGINE_SIMT]) / torch.linalg.vector_norm(xs[isg.ENGINE_SIMT])
    assert d.item() < 1e-4, d.item()
