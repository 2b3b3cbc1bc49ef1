"""Runs the reference's own inversion driver once (oracle/_ref/mom_cpu, built by
oracle/Makefile from the reference's mom.cpp, setup_born.cpp and CPU solver
sources) and stores its outputs as a fixture for the inversion loop.

    make -C oracle && python tests/golden/make_golden_dbim.py

The driver is fixed at level 7 (512 x 512 pixels, mom.cpp:6) and reads its
phantom as text from ../phantoms/phantom_256.txt (setup_born.cpp:105-113,
value * 0.1 = contrast, raster order).  The phantom written there is a seeded
set of ellipses from the library's generator.  The fixture keeps the phantom
values as read (float32), the misfit history (hist.txt, setup_born.cpp:239),
the contrast after the first and last iterations (cg_0.bin, cg_2.bin, raster
order) and the printed
step lengths and Polak-Ribiere coefficients (mom.cpp:316,395).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "inverse-solver-gpu_b200"))
MOM = os.path.join(ROOT, "oracle", "_ref", "mom_cpu")
LEVEL, NTX, NRX = 7, 4, 32


def main():
    import isg
    if not os.path.exists(MOM):
        sys.exit("oracle/_ref/mom_cpu is missing: run make -C oracle first")
    s = isg.Solver(LEVEL, numrx=NRX)
    chi = s.phantom(seed=7007, count=3, axis=(1.0, 3.0), eps=(1.1, 1.5))
    vals = (chi.real / 0.1).astype(np.float32)
    with tempfile.TemporaryDirectory() as tmp:
        run = os.path.join(tmp, "run")
        os.makedirs(run)
        os.makedirs(os.path.join(tmp, "phantoms"))
        with open(os.path.join(tmp, "phantoms", "phantom_256.txt"), "w") as f:
            f.write("\n".join(repr(float(v)) for v in vals) + "\n")
        with open(os.path.join(run, "internodes001.dat"), "w") as f:
            f.write("0\n")
        env = dict(os.environ, NUMFREQ="1", NUMTX=str(NTX), TXPROC=str(NTX), NUMRX=str(NRX), MLFMA="1",
                   MINFREQ="1", MAXFREQ="1")
        t0 = time.time()
        out = subprocess.run([MOM], cwd=run, env=env, capture_output=True, text=True, check=True).stdout
        print(f"reference driver ran in {time.time() - t0:.1f} s")
        hist = np.loadtxt(os.path.join(run, "hist.txt"))
        cg = np.stack([np.fromfile(os.path.join(run, f"cg_{i}.bin"), dtype=np.complex128) for i in range(3)])
    alphas = [float(m) for m in re.findall(r"alpha: (\S+)", out)]
    betas = [complex(float(a), float(b)) for a, b in re.findall(r"PR beta: (\S+) (\S+)", out)]
    iters = [int(m) for m in re.findall(r"NUMBER OF \d ITERATIONS: (\d+)", out)]
    # first and last iterates, complex64 (the parity bar is ~1e-4)
    np.savez_compressed(os.path.join(HERE, "golden_dbim_l7.npz"), level=LEVEL, ntx=NTX, numrx=NRX, tol=1e-4,
                        phantom=vals, hist=hist, cg0=cg[0].astype(np.complex64), cg2=cg[2].astype(np.complex64),
                        alpha=np.array(alphas), beta=np.array(betas),
                        solve_iters=np.array(iters, np.int32))
    print("hist", hist)
    print("alpha", alphas, "beta", betas)


if __name__ == "__main__":
    main()
