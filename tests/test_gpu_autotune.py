"""The launch-shape autotuner: it picks one of the candidate shapes per level,
and the operator's output does not depend on the choice (same complex64
kernels, per-output order unchanged; 1e-5 relative for the tensor engine,
whose per-CTA FP16 scale depends on how many tiles a CTA holds)."""
import numpy as np
import pytest

import isg
from _oracle import Oracle, disk_contrast

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("engine", [isg.ENGINE_SIMT, isg.ENGINE_TENSOR])
def test_autotune_keeps_the_operator(engine):
    import torch
    s = isg.Solver(6, numrx=16, max_rhs=8, device=0)
    s.setup_gpu()
    o = Oracle(6, numrx=16)
    g = torch.from_numpy(disk_contrast(o.pos(), radius=4.0, chi=0.4).astype(np.complex64)).cuda()
    rng = np.random.default_rng(3)
    x = torch.from_numpy((rng.normal(size=(8, s.numunk)) + 1j * rng.normal(size=(8, s.numunk))).astype(np.complex64)).cuda()
    before = s.matvec(x, g, engine=engine).cpu().numpy()
    got = s.autotune(8, engine)
    assert all(v in (1, 2, 4, 8, 16, 32, 64) for v in got["m2l_rows"][2:])
    assert all(v in (32, 64) for v in got["l2l_cols"][3:])
    assert all(v in (32, 64) for v in got["m2m_cols"][2:-1])
    assert got["near_pair"] in ((1, 2) if engine == isg.ENGINE_TENSOR else (0,))
    after = s.matvec(x, g, engine=engine).cpu().numpy()
    assert np.linalg.norm(after - before) / np.linalg.norm(before) < 1e-5
    info = s.bicgs(torch.zeros_like(x), g, x, tol=1e-5, engine=engine)
    assert all(i["status"] == 0 and 0 <= i["true_residual"] <= 1e-5 for i in info)
