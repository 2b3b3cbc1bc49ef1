"""Transmitter-sharded distorted-Born inversion across ranks.

The reference splits its transmitters over the MPI_COMM_DBIM ranks
(mom.cpp:99-111) and runs the Polak-Ribiere loop of mom.cpp:222-399 on each
rank's block; the only exchanges are sums over transmitters: the U-length
gradient (mom.cpp:271, 362) and the scalars of the step length and the misfit
(mom.cpp:313-314, setup_born.cpp:239-240).  This driver is that loop over a
torch.distributed process group (NCCL for device tensors, gloo for host ones;
no group runs it on one rank), with the per-transmitter work delegated to an
`ops` object:

    ops.solve(g, B, hermitian) -> X   BiCGSTAB for every row of B (isg_bicgs)
    ops.G(X) / ops.Gh(X)              G x and conj(G conj x) (isg_mlfma)
    ops.aggregate(X) -> rx            far-field receivers (isg_aggregate)
    ops.aggregateh(rx) -> Y           back-projection (isg_aggregateh)

`GpuOps` binds them to an isg.Solver.  Vectors are in tree order; fields keep
the dtype of `inc`, the contrast, gradient and direction are complex128 and
every sum is FP64, as in the single-GPU loop (isg_dbim).
"""
from __future__ import annotations

import torch

from . import ENGINE_TENSOR, default_solve_opts


class GpuOps:
    """The library's operators of one Solver (one GPU)."""

    def __init__(self, solver, engine: int = ENGINE_TENSOR, tol: float = 1e-4, maxit: int = 300,
                 check_every: int = 2):
        self.s, self.engine = solver, engine
        self.opts = default_solve_opts(tol=tol, maxit=maxit, engine=engine, check_every=check_every)
        self.iterations = 0

    def solve(self, g, B, hermitian: bool):
        X = torch.zeros_like(B)
        info = self.s.bicgs(X, g, B, hermitian=hermitian, opts=self.opts, check=True)
        self.iterations += sum(i["iterations"] for i in info)
        return X

    def G(self, X):
        return self.s.mlfma(X, engine=self.engine)

    def Gh(self, X):
        return self.s.mlfmah(X, engine=self.engine)

    def aggregate(self, X):
        return self.s.aggregate(X)

    def aggregateh(self, rx):
        return self.s.aggregateh(rx)


def shard(ntx: int, rank: int, world: int) -> range:
    """Contiguous block of transmitters of one rank (sizes differ by at most one)."""
    base, extra = divmod(ntx, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def _sum(t: torch.Tensor, group) -> torch.Tensor:
    if group is not None:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def dbim(ops, inc: torch.Tensor, mes: torch.Tensor, k0: float, iterations: int = 3, regular: float = 0.0,
         group=None):
    """Runs the inversion on this rank's transmitters inc (n, U) with measured
    far fields mes (n, numrx); `group` is an initialised torch.distributed
    group or None.  Returns (chi (U,) complex128, history), identical on every
    rank; history[i] = dict(misfit, grad_norm, object_norm, alpha, beta)."""
    dev, fdt = inc.device, inc.dtype
    c128 = torch.complex128
    k2 = k0 * k0
    n, U = inc.shape
    mes = mes.to(c128)
    o = torch.zeros(U, dtype=c128, device=dev)
    tot = inc.clone()                       # mom.cpp:225-229: total field = incident
    mesd = -mes
    mesnorm = _sum(mes.abs().pow(2).sum().reshape(1), group).item()

    def g_of(chi):
        return (k2 * chi).to(fdt)           # mom.cpp:288-289

    def gradient(g):
        # mom.cpp:247-271: od = sum_tx conj(tot) (y + mlfmah(x)), y = aggregateh(mesd),
        # x the adjoint solve with right-hand side conj(g) y; plus regular^2 chi per transmitter
        y = ops.aggregateh(mesd.to(fdt))
        X = ops.solve(g, g.conj() * y, True)
        Y = (y + ops.Gh(X)).to(c128)
        od = (tot.to(c128).conj() * Y).sum(0) + n * regular * regular * o
        return _sum(od, group)

    def record(od, alpha=0.0, beta=0.0):
        mis = _sum(mesd.abs().pow(2).sum().reshape(1), group).item()
        return {"misfit": mis / mesnorm, "grad_norm": od.abs().pow(2).sum().item(),
                "object_norm": o.abs().pow(2).sum().item(), "alpha": alpha, "beta": complex(beta)}

    g = g_of(o)
    od = gradient(g)
    hist = [record(od)]
    ot = od.clone()
    for _ in range(iterations):
        # mom.cpp:280-316: Born-linearised step length alpha = Re<mesd, J ot> / |J ot|^2
        Y = tot * (k2 * ot).to(fdt)
        X = ops.solve(g, ops.G(Y), False)
        rhs = ops.aggregate(Y + g * X).to(c128)
        t = torch.stack([(mesd.conj() * rhs).sum().real, rhs.abs().pow(2).sum()]).to(torch.float64)
        t = _sum(t, group)
        alpha = (t[0] / t[1]).item()
        # mom.cpp:318-336: step, re-solve the total fields, new residual of the data
        o = o - alpha * ot
        g = g_of(o)
        tot = ops.solve(g, inc, False)
        mesd = ops.aggregate(g * tot).to(c128) - mes
        save = od
        od = gradient(g)
        # mom.cpp:383-399: Polak-Ribiere beta = <od, od - save> / |save|^2, ot = od + beta ot
        beta = ((od * (od - save).conj()).sum() / save.abs().pow(2).sum()).item()
        ot = od + beta * ot
        hist.append(record(od, alpha, beta))
    return o, hist
