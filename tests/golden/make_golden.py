"""Generates the golden fixtures in this folder from the reference's own CPU
path (oracle/_ref/libisgref.so, compiled from the reference sources by
oracle/Makefile).  The reference ships no tests or vectors of its own, so these
pin both the restated oracle and the CUDA path.

    make -C oracle && python tests/golden/make_golden.py

Inputs are seeded (numpy PCG64) and stored beside the outputs.  Every complex
array is complex128 in the reference's tree order.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from _oracle import Reference, disk_contrast, plane_wave  # noqa: E402

K0 = 2 * np.pi


def cplx(rng, n):
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def make(level: int, numrx: int, seed: int, dense_rows: int) -> dict:
    ref = Reference(level, K0, numrx)
    rng = np.random.default_rng(seed)
    U = ref.U
    out = {"level": level, "numrx": numrx, "k0": K0, "numsamp": np.array(ref.ns, np.int32)}
    x = cplx(rng, U)
    rx = cplx(rng, numrx)
    out["x"] = x
    out["rx"] = rx
    out["mlfma"] = ref.mlfma(x)
    out["mlfmah"] = ref.mlfmah(x)
    out["aggregate"] = ref.aggregate(x)
    out["aggregateh"] = ref.aggregateh(rx)
    pos = ref.table("pos", 0, U, "c")
    out["pos"] = pos
    # Dense MoM rows through the reference's integrate() (integrate.cpp:15-41).
    rows = np.sort(rng.choice(U, dense_rows, replace=False))
    dense = np.zeros(dense_rows, np.complex128)
    for i, m in enumerate(rows):
        dense[i] = sum(ref.integrate(pos[m], pos[n]) * x[n] for n in range(U))
    out["dense_rows"] = rows.astype(np.int32)
    out["dense"] = dense
    # One forward and one adjoint BiCGSTAB solve (bicgs.cpp:88-179), tol 1e-5.
    g = disk_contrast(pos, K0, radius=0.2 * pos.real.max() * 2, chi=0.3)
    b = plane_wave(pos, 0.3, K0)
    out["g"] = g
    out["b"] = b
    xf, itf = ref.bicgs(g, b, False, 1e-5, 300)
    xa, ita = ref.bicgs(g, b, True, 1e-5, 300)
    out["bicgs_fwd"] = xf
    out["bicgs_fwd_iters"] = np.int32(itf)
    out["bicgs_adj"] = xa
    out["bicgs_adj_iters"] = np.int32(ita)
    # Small tables.
    out["near_slot4_row0"] = ref.table("near", 0, 9 * 4096, "c")[4 * 4096:4 * 4096 + 64]
    out["trans2"] = ref.table("trans", 2, 49 * ref.ns[2], "c")
    out["interp0"] = ref.table("interp", 0, ref.ns[0] * 30, "d")
    out["intind0"] = ref.table("intind", 0, ref.ns[0] * 30, "i")
    return out


def main():
    if not Reference.available():
        sys.exit("oracle/_ref/libisgref.so is missing: run make -C oracle first")
    cases = {"golden_l4.npz": make(4, 32, 1004, 48), "golden_l5.npz": make(5, 32, 1005, 16)}
    for name, data in cases.items():
        np.savez_compressed(os.path.join(HERE, name), **data)
        print(name, {k: np.shape(v) for k, v in data.items()})


if __name__ == "__main__":
    main()
