"""Independent forward problems of mixed grid size solved together
(isg.multi.MultiSolver): every RHS reaches the true residual, and each field
matches the same problem solved alone to 1e-4 relative (both solves stop at
residual 1e-5, complex64)."""
import numpy as np
import pytest

import isg
from isg.multi import MultiSolver

pytestmark = pytest.mark.gpu


def test_mixed_sizes_match_single_problem_solves():
    import torch
    rng = np.random.default_rng(8)
    ms = MultiSolver(max_rhs=8, engine=isg.ENGINE_TENSOR)
    problems = []
    for j, lvl in enumerate([3, 5, 4, 3, 5, 4, 4]):
        s = ms.solver(lvl)
        chi = s.raster_to_tree(s.phantom(seed=300 + j, count=3, axis=(0.5, 1.5), eps=(1.1, 1.8), tand_max=0.05))
        ntx = int(rng.integers(1, 6))
        b = s.plane_waves(16, first=int(rng.integers(16)), count=ntx)
        problems.append((torch.from_numpy(((2 * np.pi) ** 2 * chi).astype(np.complex64)).cuda(),
                         torch.from_numpy(b.astype(np.complex64)).cuda()))
    out = ms.solve(problems, tol=1e-5)
    for (g, b), (x, infos) in zip(problems, out):
        assert all(i["status"] == 0 and 0 <= i["true_residual"] <= 1e-5 for i in infos), infos
        s = ms.solver(isg.multi.level_of(g.shape[-1]))
        x1 = torch.zeros_like(b)
        s.bicgs(x1, g, b, tol=1e-5, engine=isg.ENGINE_TENSOR)
        err = (torch.linalg.vector_norm(x - x1) / torch.linalg.vector_norm(x1)).item()
        assert err < 1e-4, err
