"""ctypes access to the checkers: the restated oracle (oracle/liboracle.so), its
seeded input generators, and the reference's own compiled CPU path
(oracle/_ref/libisgref.so).

Test infrastructure only.  Both libraries are built by oracle/Makefile; the
reference one needs the reference tree at build time and is then used prebuilt.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libisgref.so")
REF_GPU_LIB = os.path.join(ORACLE_DIR, "_ref", "libisgref_gpu.so")

_P, _I, _D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double


def build_oracle() -> None:
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("isg_oracle.c", "isg_inputs.c", "isg_oracle.h")]
    if not os.path.exists(ORACLE_LIB) or any(os.path.getmtime(ORACLE_LIB) < os.path.getmtime(p)
                                             for p in srcs if os.path.exists(p)):
        subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True, capture_output=True)


def _arr(a: np.ndarray) -> int:
    assert a.flags.c_contiguous
    return a.ctypes.data


class Oracle:
    """FP64 restated oracle in the reference's tree order."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            build_oracle()
            L = ctypes.CDLL(ORACLE_LIB)
            L.orc_create.restype = _P
            L.orc_create.argtypes = [_I, _D, _D, _I, _I, _I, _I]
            L.orc_destroy.argtypes = [_P]
            L.orc_numunk.argtypes = [_P]
            L.orc_numsamp.argtypes = [_P, _I]
            L.orc_table.restype = _P
            L.orc_table.argtypes = [_P, ctypes.c_char_p, _I]
            for f in ("orc_mlfma", "orc_mlfmah", "orc_aggregate", "orc_aggregateh", "orc_dense_matvec"):
                getattr(L, f).argtypes = [_P, _P, _P]
            L.orc_matvec.argtypes = [_P, _P, _P, _P, _I]
            L.orc_bicgs.argtypes = [_P, _P, _P, _P, _I, _D, _I, ctypes.POINTER(_D)]
            L.orc_set_nearfield.argtypes = [_P, _D]
            L.orc_receive.argtypes = [_P, _P, _P]
            L.orc_receiveh.argtypes = [_P, _P, _P]
            L.orc_bicgs.restype = _I
            cls._lib = L
        return cls._lib

    def __init__(self, level: int, k0: float = 2 * np.pi, res: float = 0.1, numrx: int = 32, box: int = 8,
                 beta: int = 5, ninter: int = 30):
        self.L = self.lib()
        self.h = self.L.orc_create(level, k0, res, box, beta, ninter, numrx)
        assert self.h
        self.level, self.numrx = level, numrx
        self.U = self.L.orc_numunk(self.h)
        self.ns = [self.L.orc_numsamp(self.h, i) for i in range(level)]

    def __del__(self):
        try:
            self.L.orc_destroy(self.h)
        except Exception:
            pass

    def table(self, name: str, lvl: int, n: int, kind: str) -> np.ndarray:
        ct = ctypes.c_int if kind == "i" else ctypes.c_double
        cnt = 2 * n if kind == "c" else n
        p = self.L.orc_table(self.h, name.encode(), lvl)
        a = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ct)), shape=(cnt,)).copy()
        return a.view(np.complex128) if kind == "c" else a

    def _out(self, n):
        return np.zeros(n, np.complex128)

    def mlfma(self, x):
        x = np.ascontiguousarray(x, np.complex128)
        r = self._out(self.U)
        self.L.orc_mlfma(self.h, _arr(x), _arr(r))
        return r

    def mlfmah(self, x):
        x = np.ascontiguousarray(x, np.complex128)
        r = self._out(self.U)
        self.L.orc_mlfmah(self.h, _arr(x), _arr(r))
        return r

    def dense(self, x):
        x = np.ascontiguousarray(x, np.complex128)
        r = self._out(self.U)
        self.L.orc_dense_matvec(self.h, _arr(x), _arr(r))
        return r

    def matvec(self, x, g, hermitian=False):
        x = np.ascontiguousarray(x, np.complex128)
        g = np.ascontiguousarray(g, np.complex128)
        y = self._out(self.U)
        self.L.orc_matvec(self.h, _arr(x), _arr(g), _arr(y), int(hermitian))
        return y

    def bicgs(self, g, b, hermitian=False, tol=1e-5, maxit=300, x0=None):
        x = np.zeros(self.U, np.complex128) if x0 is None else np.array(x0, np.complex128)
        g = np.ascontiguousarray(g, np.complex128)
        b = np.ascontiguousarray(b, np.complex128)
        err = ctypes.c_double()
        it = self.L.orc_bicgs(self.h, _arr(x), _arr(g), _arr(b), int(hermitian), tol, maxit, ctypes.byref(err))
        return x, it, err.value

    def aggregate(self, x):
        x = np.ascontiguousarray(x, np.complex128)
        rx = self._out(self.numrx)
        self.L.orc_aggregate(self.h, _arr(x), _arr(rx))
        return rx

    def aggregateh(self, rx):
        rx = np.ascontiguousarray(rx, np.complex128)
        x = self._out(self.U)
        self.L.orc_aggregateh(self.h, _arr(x), _arr(rx))
        return x

    def pos(self):
        return self.table("pos", 0, self.U, "c")

    def set_nearfield(self, radius: float):
        """Near-field receivers at this radius (orc_dbim then uses them); 0 removes them."""
        self.L.orc_set_nearfield(self.h, radius)

    def receive(self, x):
        x = np.ascontiguousarray(x, np.complex128)
        rx = self._out(self.numrx)
        self.L.orc_receive(self.h, _arr(x), _arr(rx))
        return rx

    def receiveh(self, rx):
        rx = np.ascontiguousarray(rx, np.complex128)
        x = self._out(self.U)
        self.L.orc_receiveh(self.h, _arr(x), _arr(rx))
        return x


def _oracle_lib():
    L = Oracle.lib()
    L.orc_in_ellipses.argtypes = [_I, _D, _I, _D, _D, _D, _D, _D, ctypes.c_uint64, _P]
    L.orc_in_plane_waves.argtypes = [_I, _D, _D, _I, _I, _I, _P, _P]
    return L


def seeded_ellipses(side: int, seed: int, count: int, axis=(1.0, 3.0), eps=(1.1, 1.5), tand_max: float = 0.0,
                    res: float = 0.1) -> np.ndarray:
    """Contrast chi = eps_r - 1 (complex128, raster order) from the oracle's
    restatement of the library's ellipse generator (bit-identical)."""
    chi = np.zeros(side * side, np.complex128)
    _oracle_lib().orc_in_ellipses(side, res, count, axis[0], axis[1], eps[0], eps[1], tand_max, seed, _arr(chi))
    return chi


def seeded_plane_waves(side: int, ntx: int, first: int, count: int, unkmap: np.ndarray | None,
                       k0: float = 2 * np.pi, res: float = 0.1) -> np.ndarray:
    """Plane waves of transmitters first..first+count-1 of ntx (complex128),
    in tree order through unkmap (raster order when None)."""
    out = np.zeros((count, side * side), np.complex128)
    um = None if unkmap is None else np.ascontiguousarray(unkmap, np.int32)
    _oracle_lib().orc_in_plane_waves(side, res, k0, ntx, first, count, None if um is None else _arr(um), _arr(out))
    return out


class Reference:
    """The reference's own CPU path (one global instance per process)."""

    _lib = None
    _path = REF_LIB

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls._path)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = ctypes.CDLL(cls._path)
            L.ref_setup.argtypes = [_I, _D, _I]
            L.ref_table.restype = _P
            L.ref_table.argtypes = [ctypes.c_char_p, _I]
            for f in ("ref_mlfma", "ref_mlfmah", "ref_aggregate", "ref_aggregateh"):
                getattr(L, f).argtypes = [_P, _P]
            L.ref_bicgs.argtypes = [_P, _P, _P, _I, _D, _I]
            L.ref_integrate.argtypes = [_D, _D, _D, _D, _P]
            cls._lib = L
        return cls._lib

    def __init__(self, level: int, k0: float = 2 * np.pi, numrx: int = 32):
        self.L = self.lib()
        assert self.L.ref_setup(level, k0, numrx) == 0
        self.level, self.numrx = level, numrx
        self.U = self.L.ref_numunk()
        self.ns = [self.L.ref_numsamp(i) for i in range(level)]

    def table(self, name: str, lvl: int, n: int, kind: str) -> np.ndarray:
        ct = ctypes.c_int if kind == "i" else ctypes.c_double
        cnt = 2 * n if kind == "c" else n
        p = self.L.ref_table(name.encode(), lvl)
        a = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ct)), shape=(cnt,)).copy()
        return a.view(np.complex128) if kind == "c" else a

    def mlfma(self, x):
        x = np.array(x, np.complex128)
        r = np.zeros(self.U, np.complex128)
        self.L.ref_mlfma(_arr(x), _arr(r))
        return r

    def mlfmah(self, x):
        x = np.array(x, np.complex128)
        r = np.zeros(self.U, np.complex128)
        self.L.ref_mlfmah(_arr(x), _arr(r))
        return r

    def aggregate(self, x):
        x = np.array(x, np.complex128)
        rx = np.zeros(self.numrx, np.complex128)
        self.L.ref_aggregate(_arr(x), _arr(rx))
        return rx

    def aggregateh(self, rx):
        rx = np.array(rx, np.complex128)
        x = np.zeros(self.U, np.complex128)
        self.L.ref_aggregateh(_arr(x), _arr(rx))
        return x

    def bicgs(self, g, b, hermitian=False, tol=1e-5, maxit=300):
        x = np.zeros(self.U, np.complex128)
        g = np.array(g, np.complex128)
        b = np.array(b, np.complex128)
        it = self.L.ref_bicgs(_arr(x), _arr(g), _arr(b), int(hermitian), tol, maxit)
        return x, it

    def integrate(self, t: complex, b: complex) -> complex:
        out = np.zeros(2)
        self.L.ref_integrate(t.real, t.imag, b.real, b.imag, _arr(out))
        return complex(out[0], out[1])


class ReferenceGpu(Reference):
    """The reference's own GPU path (gpu.cu, kernels.cu, matvec_gpu.cu,
    bicgs_gpu.cu: FP64 on the GPU, the product its Makefile links) behind the
    same harness and entry points.  Load it in a process of its own: its error
    handler exits the process on any CUDA error (kernels.h gpuAssert)."""

    _lib = None
    _path = REF_GPU_LIB


def rel(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def disk_contrast(pos: np.ndarray, k0: float = 2 * np.pi, radius: float = 2.0, chi: float = 0.3) -> np.ndarray:
    """g = k0^2 chi inside a disk (a simple fixed phantom for fixtures)."""
    return (k0 * k0 * chi * (np.abs(pos) < radius)).astype(np.complex128)


def plane_wave(pos: np.ndarray, angle: float, k0: float = 2 * np.pi) -> np.ndarray:
    """exp(i k0 d.r) (setup_born.cpp:62-65)."""
    return np.exp(1j * k0 * (np.cos(angle) * pos.real + np.sin(angle) * pos.imag))


def oracle_dbim(o: "Oracle", inc: np.ndarray, chi_true: np.ndarray, iterations: int, regular: float = 0.0,
                tol: float = 1e-4, maxit: int = 300):
    """orc_dbim: the reference's measurement + Polak-Ribiere inversion loop in FP64 (tree order)."""
    L = o.L
    L.orc_dbim.argtypes = [_P, _I, _P, _P, _I, _D, _D, _I, _P, _P, _P, _P]
    ntx = inc.shape[0]
    inc = np.ascontiguousarray(inc, np.complex128)
    chi_true = np.ascontiguousarray(chi_true, np.complex128)
    chi = np.zeros(o.U, np.complex128)
    hist = np.zeros((iterations + 1, 5))
    alpha = np.zeros(iterations)
    beta = np.zeros(iterations, np.complex128)
    L.orc_dbim(o.h, ntx, _arr(inc), _arr(chi_true), iterations, regular, tol, maxit, _arr(chi), _arr(hist),
               _arr(alpha), _arr(beta))
    return chi, hist, alpha, beta
