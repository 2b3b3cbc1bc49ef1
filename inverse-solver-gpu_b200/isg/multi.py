"""Many independent forward problems of uneven grid size in one call.

Problems that share a grid size become one multi-RHS block: every transmitter
of every such problem is one right-hand side, with its own contrast (g_stride =
numunk) and its own convergence mask, in chunks of at most `max_rhs`.  The
size groups are solved together by isg_bicgs_group, one chunk of every group
per call: each block of iterations of all of them is one CUDA-graph launch
(one branch per grid size) and one host poll.  The reference solves one
problem at a time (mom.cpp:250-350); this is the library's batching of its
solve path, with the same per-RHS results.
"""
from __future__ import annotations

from . import ENGINE_TENSOR, ORDER_TREE, Solver, bicgs_group, default_solve_opts


def level_of(numunk: int, box: int = 8) -> int:
    """The reference `level` of a square grid with numunk pixels (mom.cpp:137)."""
    side = int(round(numunk ** 0.5))
    if side * side != numunk or side % box:
        raise ValueError(f"{numunk} unknowns is not a square grid of {box}-pixel leaves")
    n, lvl = side // box, 1
    while n > 1:
        if n % 2:
            raise ValueError(f"grid side {side} is not {box} x a power of two")
        n //= 2
        lvl += 1
    return lvl


class MultiSolver:
    """Forward solves for a list of (g, b) problems of mixed grid sizes.

    g: (U,) complex64 contrast k0^2 (eps_r - 1) of one problem; b: (ntx, U)
    complex64 incident fields of its transmitters; both device tensors in
    `order`.  One Solver per grid size is built on first use and kept."""

    def __init__(self, max_rhs: int = 256, device: int = 0, engine: int = ENGINE_TENSOR, numrx: int = 32):
        self.max_rhs, self.device, self.engine, self.numrx = max_rhs, device, engine, numrx
        self.solvers: dict[int, Solver] = {}

    def solver(self, level: int) -> Solver:
        if level not in self.solvers:
            s = Solver(level, numrx=self.numrx, max_rhs=self.max_rhs, device=self.device)
            s.setup_gpu()
            self.solvers[level] = s
        return self.solvers[level]

    def solve(self, problems, tol: float = 1e-5, maxit: int = 300, order: int = ORDER_TREE, check_every: int = 2):
        """Returns, per problem, (x: (ntx, U) total fields, list of per-RHS info dicts)."""
        import torch
        groups: dict[int, list[int]] = {}
        for p, (g, b) in enumerate(problems):
            groups.setdefault(level_of(g.shape[-1]), []).append(p)
        out: list = [None] * len(problems)
        for lvl in groups:
            self.solver(lvl)
        opts = default_solve_opts(tol=tol, maxit=maxit, engine=self.engine, check_every=check_every)
        # (problem, transmitter) pairs of each group, in order, cut into chunks of max_rhs
        chunks = {lvl: [] for lvl in groups}
        for lvl, idx in groups.items():
            pairs = [(p, t) for p in idx for t in range(problems[p][1].shape[0])]
            chunks[lvl] = [pairs[c:c + self.max_rhs] for c in range(0, len(pairs), self.max_rhs)]
        xs = {p: torch.zeros_like(problems[p][1]) for p in range(len(problems))}
        infos = {p: [None] * problems[p][1].shape[0] for p in range(len(problems))}
        stream = torch.cuda.Stream(device=self.device)
        with torch.cuda.stream(stream):
            for r in range(max(len(c) for c in chunks.values())):
                members, picks = [], []
                for lvl in sorted(chunks):
                    if r >= len(chunks[lvl]):
                        continue
                    chunk = chunks[lvl][r]
                    G = torch.stack([problems[p][0] for p, _ in chunk])
                    B = torch.stack([problems[p][1][t] for p, t in chunk])
                    members.append((self.solver(lvl), torch.zeros_like(B), G, B))
                    picks.append(chunk)
                res = bicgs_group(members, order=order, opts=opts, stream=stream)
                for (_, X, _, _), chunk, inf in zip(members, picks, res):
                    for j, (p, t) in enumerate(chunk):
                        xs[p][t].copy_(X[j])
                        infos[p][t] = inf[j]
        stream.synchronize()
        for p in range(len(problems)):
            out[p] = (xs[p], infos[p])
        return out
