"""The transmitter-sharded inversion driver (isg.dbim_dist) on CPU: two gloo
ranks on 127.0.0.1 give the same contrast and history as one rank, and one
rank reproduces the FP64 oracle's single-process inversion (orc_dbim) on the
same data.  The per-transmitter operators are the FP64 oracle's."""
import os
import socket

import numpy as np
import pytest
import torch

from isg import dbim_dist
from _oracle import Oracle, disk_contrast, oracle_dbim, plane_wave, rel

LEVEL, NTX, ITER, TOL = 4, 4, 2, 1e-9
K0 = 2 * np.pi


class OracleOps:
    """ops for dbim_dist backed by the FP64 oracle (torch CPU complex128 tensors)."""

    def __init__(self, o):
        self.o = o

    def solve(self, g, B, hermitian):
        gn = g.numpy()
        return torch.from_numpy(np.stack([self.o.bicgs(gn, b, hermitian, TOL, 1000)[0] for b in B.numpy()]))

    def G(self, X):
        return torch.from_numpy(np.stack([self.o.mlfma(x) for x in X.numpy()]))

    def Gh(self, X):
        return torch.from_numpy(np.stack([self.o.mlfmah(x) for x in X.numpy()]))

    def aggregate(self, X):
        return torch.from_numpy(np.stack([self.o.aggregate(x) for x in X.numpy()]))

    def aggregateh(self, R):
        return torch.from_numpy(np.stack([self.o.aggregateh(r) for r in R.numpy()]))


def problem():
    o = Oracle(LEVEL, numrx=16)
    pos = o.pos()
    chi_true = disk_contrast(pos, radius=1.2, chi=0.2) / K0 ** 2 + 0.02 * (pos.real > 0.5) * (np.abs(pos) < 2)
    inc = np.stack([plane_wave(pos, 2 * np.pi * t / NTX) for t in range(NTX)])
    g = chi_true * K0 ** 2
    mes = np.stack([o.aggregate(g * o.bicgs(g, b, False, TOL, 1000)[0]) for b in inc])
    return o, chi_true, inc, mes


def run_rank(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        o, chi_true, inc, mes = problem()
        blk = dbim_dist.shard(NTX, rank, world)
        chi, hist = dbim_dist.dbim(OracleOps(o), torch.from_numpy(inc[blk.start:blk.stop]),
                                   torch.from_numpy(mes[blk.start:blk.stop]), K0, ITER, group=dist.group.WORLD)
        np.save(os.path.join(outdir, f"chi{rank}.npy"), chi.numpy())
        np.save(os.path.join(outdir, f"mis{rank}.npy"), np.array([h["misfit"] for h in hist]))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_every_transmitter_once():
    for ntx in (1, 4, 7, 256):
        for world in (1, 2, 3, 8):
            got = [t for r in range(world) for t in dbim_dist.shard(ntx, r, world)]
            assert got == list(range(ntx))


def test_two_gloo_ranks_match_one_rank_and_the_oracle(tmp_path):
    import torch.multiprocessing as mp
    o, chi_true, inc, mes = problem()
    chi1, hist1 = dbim_dist.dbim(OracleOps(o), torch.from_numpy(inc), torch.from_numpy(mes), K0, ITER)
    mp.spawn(run_rank, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        chi2 = np.load(tmp_path / f"chi{r}.npy")
        assert rel(chi2, chi1.numpy()) < 1e-10
        assert np.allclose(np.load(tmp_path / f"mis{r}.npy"), [h["misfit"] for h in hist1], rtol=1e-10)
    chi_o, hist_o, alpha_o, _ = oracle_dbim(o, inc, chi_true, ITER, 0.0, TOL, 1000)
    assert rel(chi1.numpy(), chi_o) < 1e-8
    assert np.allclose([h["alpha"] for h in hist1[1:]], alpha_o, rtol=1e-8)
    assert np.allclose([h["misfit"] for h in hist1], hist_o[:, 0], rtol=1e-8)
