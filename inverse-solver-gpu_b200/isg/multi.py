"""Many independent forward problems of uneven grid size in one call.

Problems that share a grid size become one multi-RHS block: every transmitter
of every such problem is one right-hand side, with its own contrast (g_stride =
numunk) and its own convergence mask inside isg_bicgs, in chunks of at most
`max_rhs`.  The size groups run at the same time, each driven by its own host
thread on its own CUDA stream (isg_bicgs releases the interpreter while it
polls convergence).  The reference solves one problem at a time (mom.cpp:250-350);
this is the library's batching of its solve path, with the same per-RHS
results.
"""
from __future__ import annotations

import threading

from . import ENGINE_TENSOR, ORDER_TREE, Solver, default_solve_opts


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
        errors: list = []
        for lvl in groups:
            self.solver(lvl)  # built here, not in the worker threads
        torch.cuda.synchronize(self.device)  # the inputs are complete before other streams read them

        def run(level: int, idx: list[int]):
            try:
                s = self.solver(level)
                stream = torch.cuda.Stream(device=self.device)
                opts = default_solve_opts(tol=tol, maxit=maxit, engine=self.engine, check_every=check_every)
                # (problem, transmitter) pairs of the group, in order
                pairs = [(p, t) for p in idx for t in range(problems[p][1].shape[0])]
                infos = {p: [None] * problems[p][1].shape[0] for p in idx}
                with torch.cuda.stream(stream):
                    xs = {p: torch.zeros_like(problems[p][1]) for p in idx}
                    for c0 in range(0, len(pairs), self.max_rhs):
                        chunk = pairs[c0:c0 + self.max_rhs]
                        G = torch.stack([problems[p][0] for p, _ in chunk])
                        B = torch.stack([problems[p][1][t] for p, t in chunk])
                        X = torch.zeros_like(B)
                        inf = s.bicgs(X, G, B, order=order, opts=opts, stream=stream)
                        for j, (p, t) in enumerate(chunk):
                            xs[p][t].copy_(X[j])
                            infos[p][t] = inf[j]
                stream.synchronize()
                for p in idx:
                    out[p] = (xs[p], infos[p])
            except Exception as e:  # reported on the calling thread
                errors.append(e)

        threads = [threading.Thread(target=run, args=(lvl, idx)) for lvl, idx in sorted(groups.items())]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        if errors:
            raise errors[0]
        return out
