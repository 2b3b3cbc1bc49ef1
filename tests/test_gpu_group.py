"""isg_bicgs_group: independent problems of different grid sizes solved
together, each block of iterations of all of them one CUDA graph with a branch
per problem.  Every member's fields, iteration counts and residuals equal
those of its own isg_bicgs call bit for bit (the same kernels on the same
data), and the group's graph launches come once per poll for all members."""
import numpy as np
import pytest

import isg

pytestmark = pytest.mark.gpu


def _problem(s, seed, ntx):
    import torch
    rng = np.random.default_rng(seed)
    chi = s.raster_to_tree(s.phantom(seed=seed, count=3, axis=(0.5, 1.5), eps=(1.1, 1.6)))
    g = torch.from_numpy(((2 * np.pi) ** 2 * chi).astype(np.complex64)).cuda()
    b = torch.from_numpy(s.plane_waves(16, first=int(rng.integers(16)), count=ntx).astype(np.complex64)).cuda()
    return g, b


@pytest.mark.parametrize("engine", [isg.ENGINE_SIMT, isg.ENGINE_TENSOR])
def test_group_solve_equals_separate_solves(engine):
    import torch
    sizes = [(3, 5), (5, 7), (4, 3)]  # (level, transmitters): 32^2, 128^2 and 64^2 pixels
    solvers = [isg.Solver(lvl, numrx=16, max_rhs=8, device=0) for lvl, _ in sizes]
    probs = [_problem(s, 40 + i, n) for i, (s, (_, n)) in enumerate(zip(solvers, sizes))]
    side = torch.cuda.Stream()
    opts = isg.default_solve_opts(tol=1e-5, maxit=500, engine=engine, check_every=2)
    want = []
    for s, (g, b) in zip(solvers, probs):
        x = torch.zeros_like(b)
        want.append((x, s.bicgs(x, g, b, opts=opts, stream=side)))
    torch.cuda.synchronize()
    xs = [torch.zeros_like(b) for _, b in probs]
    n0 = isg.kernel_launches()
    got = isg.bicgs_group([(s, x, g, b) for s, x, (g, b) in zip(solvers, xs, probs)], opts=opts, stream=side)
    torch.cuda.synchronize()
    assert isg.kernel_launches() > n0
    for (x_want, inf_want), x, inf in zip(want, xs, got):
        assert all(i["status"] == 0 and 0 <= i["true_residual"] <= 1e-5 for i in inf), inf
        assert [i["iterations"] for i in inf] == [i["iterations"] for i in inf_want]
        assert [i["true_residual"] for i in inf] == [i["true_residual"] for i in inf_want]
        assert torch.equal(x, x_want)


def test_group_refuses_a_context_twice():
    import torch
    s = isg.Solver(3, numrx=16, max_rhs=4, device=0)
    g, b = _problem(s, 7, 2)
    with pytest.raises(isg.IsgError):
        isg.bicgs_group([(s, torch.zeros_like(b), g, b), (s, torch.zeros_like(b), g, b)], check=True,
                        stream=torch.cuda.Stream())
