"""Python binding of libisg.so, the B200 MLFMA inverse-scattering solver.

It mirrors the reference's call surface (merthidayetoglu/inverse-solver-GPU,
vars.h:14-38): ``setup_mlfma`` (constructor), ``setup_gpu``, ``mlfma`` /
``mlfmah``, ``matvec``, ``bicgs``, ``aggregate`` / ``aggregateh``.  Device
vectors are torch complex64 CUDA tensors of shape (U,) or (nrhs, U); torch is
only the allocator here, every operation runs in libisg.so's CUDA kernels.
The library must be built (``inverse-solver-gpu_b200/build.py``); nothing falls
back to a CPU path.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libisg.so")

ORDER_TREE, ORDER_RASTER, ORDER_BLOCKED = 0, 1, 2
ENGINE_SIMT, ENGINE_TENSOR = 0, 1
GUESS_ZERO, GUESS_CALLER, GUESS_LEARNED = 0, 1, 2

STATUS = {0: "ok", 1: "not converged", 2: "breakdown", 3: "non-finite", 4: "CUDA error", 5: "bad argument",
          6: "timeout", 7: "no device", 8: "unsupported"}


class IsgError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        super().__init__(f"isg: {STATUS.get(status, status)}{': ' + msg if msg else ''}")
        self.status = status


class Opts(ctypes.Structure):
    _fields_ = [("level", ctypes.c_int), ("box", ctypes.c_int), ("res", ctypes.c_double), ("k0", ctypes.c_double),
                ("beta", ctypes.c_int), ("ninter", ctypes.c_int), ("numrx", ctypes.c_int), ("max_rhs", ctypes.c_int),
                ("device", ctypes.c_int)]


class SolveOpts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("maxit", ctypes.c_int), ("guess", ctypes.c_int),
                ("check_every", ctypes.c_int), ("true_residual", ctypes.c_int), ("max_restarts", ctypes.c_int),
                ("engine", ctypes.c_int), ("graph", ctypes.c_int)]


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("matvecs", ctypes.c_int), ("status", ctypes.c_int),
                ("restarts", ctypes.c_int), ("residual", ctypes.c_double), ("true_residual", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class GroupMember(ctypes.Structure):
    _fields_ = [("ctx", ctypes.c_void_p), ("x", ctypes.c_void_p), ("g", ctypes.c_void_p), ("g_stride", ctypes.c_int64),
                ("b", ctypes.c_void_p), ("nrhs", ctypes.c_int), ("info", ctypes.POINTER(SolveInfo))]


class DbimOpts(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("regular", ctypes.c_double), ("start_from_chi", ctypes.c_int),
                ("solve", SolveOpts), ("warm_start", ctypes.c_int), ("checkpoint", ctypes.c_char_p)]


class DbimRecord(ctypes.Structure):
    _fields_ = [("misfit", ctypes.c_double), ("object_error", ctypes.c_double), ("reg_cost", ctypes.c_double),
                ("grad_norm", ctypes.c_double), ("object_norm", ctypes.c_double), ("alpha", ctypes.c_double),
                ("beta_re", ctypes.c_double), ("beta_im", ctypes.c_double), ("solves", ctypes.c_int64),
                ("iterations", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class Phantom(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("count", ctypes.c_int), ("axis_min", ctypes.c_double),
                ("axis_max", ctypes.c_double), ("eps_min", ctypes.c_double), ("eps_max", ctypes.c_double),
                ("tand_max", ctypes.c_double), ("corr_len", ctypes.c_double), ("seed", ctypes.c_uint64)]


class FnoOpts(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("modes", ctypes.c_int), ("layers", ctypes.c_int), ("batch", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("tensor", ctypes.c_int)]


_lib = None

# Every entry point declared in include/isg.h, with its ctypes signature.
_P, _I, _D, _L = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64
SIGNATURES = {
    "isg_default_opts": (None, [ctypes.POINTER(Opts)]),
    "isg_default_solve_opts": (None, [ctypes.POINTER(SolveOpts)]),
    "isg_create": (_I, [ctypes.POINTER(Opts), ctypes.POINTER(_P)]),
    "isg_setup_gpu": (_I, [_P]),
    "isg_destroy": (None, [_P]),
    "isg_status_string": (ctypes.c_char_p, [_I]),
    "isg_last_error": (ctypes.c_char_p, [_P]),
    "isg_numunk": (_I, [_P]),
    "isg_side": (_I, [_P]),
    "isg_numsamp": (_I, [_P, _I]),
    "isg_levels": (_I, [_P]),
    "isg_host_table": (_I, [_P, ctypes.c_char_p, _I, ctypes.POINTER(_P), ctypes.POINTER(_L)]),
    "isg_reorder": (_I, [_P, _P, _P, _I, _I, _I, _P]),
    "isg_mlfma": (_I, [_P, _P, _P, _I, _I, _I, _I, _P]),
    "isg_matvec": (_I, [_P, _P, _P, _L, _P, _I, _I, _I, _I, _P]),
    "isg_bicgs": (_I, [_P, _P, _P, _L, _P, _I, _I, _I, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveInfo), _P]),
    "isg_bicgs_group": (_I, [_I, ctypes.POINTER(GroupMember), _I, _I, ctypes.POINTER(SolveOpts), _P]),
    "isg_aggregate": (_I, [_P, _P, _P, _I, _I, _P]),
    "isg_aggregateh": (_I, [_P, _P, _P, _I, _I, _P]),
    "isg_aggregate_noalloc": (_I, [_P, _P, _P, _I, _I, _P]),
    "isg_set_nearfield_receivers": (_I, [_P, _D]),
    "isg_receive": (_I, [_P, _P, _P, _I, _I, _P]),
    "isg_receiveh": (_I, [_P, _P, _P, _I, _I, _P]),
    "isg_default_dbim_opts": (None, [ctypes.POINTER(DbimOpts)]),
    "isg_measure": (_I, [_P, _I, _P, _P, _I, _D, ctypes.c_uint64, ctypes.POINTER(SolveOpts), _P, _P]),
    "isg_dbim": (_I, [_P, _I, _P, _P, _P, _P, _I, ctypes.POINTER(DbimOpts), ctypes.POINTER(DbimRecord), _P]),
    "isg_kernel_launches": (ctypes.c_int64, []),
    "isg_time_stages": (_I, [_P, _I, _I, _I, _P]),
    "isg_make_phantom": (_I, [_P, ctypes.POINTER(Phantom), _P]),
    "isg_make_plane_waves": (_I, [_P, _I, _I, _I, _I, _P]),
    "isg_make_line_sources": (_I, [_P, _I, _I, _I, _D, _I, _P]),
    "isg_autotune": (_I, [_P, _I, _I, _P]),
    "isg_tuned": (_I, [_P, _I, _I, ctypes.POINTER(_I)]),
    "isg_default_fno_opts": (None, [ctypes.POINTER(FnoOpts)]),
    "isg_fno_create": (_I, [_P, ctypes.POINTER(FnoOpts)]),
    "isg_fno_param_count": (_L, [_P]),
    "isg_fno_params": (_I, [_P, _P, _L, _I, _I]),
    "isg_fno_apply": (_I, [_P, _P, _L, _P, _P, _I, _I, _P]),
    "isg_fno_grad": (_I, [_P, _P, _L, _P, _P, _I, _I, ctypes.POINTER(_D), _P]),
    "isg_fno_train_step": (_I, [_P, _P, _L, _P, _P, _I, _I, ctypes.c_float, ctypes.POINTER(_D), _P]),
}


def lib() -> ctypes.CDLL:
    """Loads libisg.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise ImportError(f"{LIBPATH} is missing: build it with inverse-solver-gpu_b200/build.py")
        L = ctypes.CDLL(LIBPATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(t) -> int | None:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream(stream) -> int | None:
    """The caller's stream, defaulting to torch's current stream (0 is CUDA's legacy default).

    A torch stream other than the current one first waits for the work queued
    on the current stream, where torch made the call's input tensors (an
    indexing kernel, or a copy from pageable host memory whose DMA may still
    be in flight when `.to()` returns): the library's kernels then never read
    an input before it is written."""
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream or None
    if hasattr(stream, "wait_stream") and hasattr(stream, "device"):
        import torch
        cur = torch.cuda.current_stream(stream.device)
        if cur.cuda_stream != stream.cuda_stream:
            stream.wait_stream(cur)
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def bicgs_group(members, hermitian: bool = False, order: int = ORDER_TREE, opts: SolveOpts | None = None,
                stream=None, check: bool = False, **kw) -> list[list[dict]]:
    """isg_bicgs_group: BiCGSTAB for several independent problems at once.
    members: (solver, x, g, b) per problem, distinct Solvers (contexts) on one
    device, tensors as for Solver.bicgs.  Returns per member its per-RHS info."""
    o = opts if opts is not None else default_solve_opts(**kw)
    arr = (GroupMember * len(members))()
    infos = []
    for i, (s, x, g, b) in enumerate(members):
        n = s._nrhs(b)
        inf = (SolveInfo * n)()
        infos.append(inf)
        arr[i].ctx, arr[i].x, arr[i].g, arr[i].b, arr[i].nrhs = s._h, _ptr(x), _ptr(g), _ptr(b), n
        arr[i].g_stride = 0 if g.dim() == 1 else s.numunk
        arr[i].info = ctypes.cast(inf, ctypes.POINTER(SolveInfo))
    st = lib().isg_bicgs_group(len(members), arr, int(hermitian), order, ctypes.byref(o), _stream(stream))
    if st in (4, 5, 7, 8) or (check and st != 0):
        members[0][0]._check(st, "bicgs_group")
    return [[i.as_dict() for i in inf] for inf in infos]


def kernel_launches() -> int:
    """Kernels launched by libisg.so in this process so far."""
    return int(lib().isg_kernel_launches())


def default_solve_opts(**kw) -> SolveOpts:
    o = SolveOpts()
    lib().isg_default_solve_opts(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Solver:
    """One MLFMA operator on a grid of ``8 * 2**(level-1)`` pixels per side.

    The constructor is the reference's ``setup_mlfma`` (setup_mlfma.cpp:50);
    ``setup_gpu`` uploads the tables (gpu.cu:69) and is also run implicitly by
    the first device call.
    """

    def __init__(self, level: int, k0: float = 2 * math.pi, res: float = 0.1, numrx: int = 32, max_rhs: int = 1,
                 device: int = 0, box: int = 8, beta: int = 5, ninter: int = 30):
        L = lib()
        o = Opts()
        L.isg_default_opts(ctypes.byref(o))
        o.level, o.k0, o.res, o.numrx, o.max_rhs, o.device = level, k0, res, numrx, max_rhs, device
        o.box, o.beta, o.ninter = box, beta, ninter
        h = ctypes.c_void_p()
        st = L.isg_create(ctypes.byref(o), ctypes.byref(h))
        if st != 0:
            raise IsgError(st, "isg_create")
        self._h = h
        self.opts = o
        self.level = level
        self.numunk = L.isg_numunk(h)
        self.side = L.isg_side(h)
        self.numrx = numrx
        self.max_rhs = max_rhs
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib().isg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != 0:
            raise IsgError(st, f"{what}: {lib().isg_last_error(self._h).decode()}")

    # ---- tables ----
    def numsamp(self, lvl: int) -> int:
        return lib().isg_numsamp(self._h, lvl)

    def host_table(self, name: str, lvl: int = 0) -> np.ndarray:
        """Copy of a FP64 setup table in the reference's layout."""
        data, count = ctypes.c_void_p(), ctypes.c_int64()
        self._check(lib().isg_host_table(self._h, name.encode(), lvl, ctypes.byref(data), ctypes.byref(count)),
                    f"host_table({name})")
        if name in ("intind", "antind", "intindh", "antindh", "numsamp", "numterm", "unkmap", "tree_of_blocked",
                    "raster_of_blocked"):
            ct, dt = ctypes.c_int, np.int32
        elif name in ("interp", "anterp", "interph", "anterph", "clusize"):
            ct, dt = ctypes.c_double, np.float64
        else:
            ct, dt = ctypes.c_double, np.complex128
        n = count.value * (2 if dt == np.complex128 else 1)
        buf = np.ctypeslib.as_array(ctypes.cast(data, ctypes.POINTER(ct)), shape=(n,)).copy()
        return buf.view(np.complex128) if dt == np.complex128 else buf.astype(dt)

    # ---- device ----
    def setup_gpu(self):
        self._check(lib().isg_setup_gpu(self._h), "setup_gpu")

    def _nrhs(self, t) -> int:
        return 1 if t.dim() == 1 else t.shape[0]

    def _empty_like(self, x):
        import torch
        return torch.empty_like(x)

    def mlfma(self, x, r=None, conj: bool = False, order: int = ORDER_TREE, engine: int = ENGINE_SIMT, stream=None):
        """r = G x (mlfma, matvec_gpu.cu:65); conj=True gives mlfmah."""
        r = self._empty_like(x) if r is None else r
        self._check(lib().isg_mlfma(self._h, _ptr(x), _ptr(r), self._nrhs(x), int(conj), order, engine,
                                    _stream(stream)), "mlfma")
        return r

    def mlfmah(self, x, r=None, order: int = ORDER_TREE, engine: int = ENGINE_SIMT, stream=None):
        return self.mlfma(x, r, True, order, engine, stream)

    def matvec(self, x, g, y=None, hermitian: bool = False, order: int = ORDER_TREE, engine: int = ENGINE_SIMT,
               stream=None):
        """y = x - G(g x) or its adjoint (matvec, bicgs_gpu.cu:61)."""
        y = self._empty_like(x) if y is None else y
        gs = 0 if g.dim() == 1 else self.numunk
        self._check(lib().isg_matvec(self._h, _ptr(x), _ptr(g), gs, _ptr(y), self._nrhs(x), int(hermitian), order,
                                     engine, _stream(stream)), "matvec")
        return y

    def bicgs(self, x, g, b, hermitian: bool = False, order: int = ORDER_TREE, opts: SolveOpts | None = None,
              stream=None, check: bool = False, **kw) -> list[dict]:
        """BiCGSTAB for every RHS of b (bicgs, bicgs_gpu.cu:116); x is overwritten."""
        o = opts if opts is not None else default_solve_opts(**kw)
        R = self._nrhs(b)
        info = (SolveInfo * R)()
        gs = 0 if g.dim() == 1 else self.numunk
        st = lib().isg_bicgs(self._h, _ptr(x), _ptr(g), gs, _ptr(b), R, int(hermitian), order, ctypes.byref(o),
                             info, _stream(stream))
        if st in (4, 5, 7, 8) or (check and st != 0):
            self._check(st, "bicgs")
        return [i.as_dict() for i in info]

    def aggregate(self, x, rx=None, order: int = ORDER_TREE, stream=None):
        """Far-field receiver samples of x (aggregate, matvec_gpu.cu:266)."""
        import torch
        R = self._nrhs(x)
        if rx is None:
            rx = torch.empty((R, self.numrx) if x.dim() == 2 else (self.numrx,), dtype=torch.complex64,
                             device=x.device)
        self._check(lib().isg_aggregate(self._h, _ptr(x), _ptr(rx), R, order, _stream(stream)), "aggregate")
        return rx

    def aggregateh(self, rx, x=None, order: int = ORDER_TREE, stream=None):
        """Back-projection of receiver samples (aggregateh, matvec_gpu.cu:369)."""
        import torch
        R = 1 if rx.dim() == 1 else rx.shape[0]
        if x is None:
            x = torch.empty((R, self.numunk) if rx.dim() == 2 else (self.numunk,), dtype=torch.complex64,
                            device=rx.device)
        self._check(lib().isg_aggregateh(self._h, _ptr(x), _ptr(rx), R, order, _stream(stream)), "aggregateh")
        return x

    # ---- near-field receivers ----
    def set_nearfield_receivers(self, radius: float):
        """numrx receivers on a circle of this radius (wavelengths); 0 returns to far field."""
        self._check(lib().isg_set_nearfield_receivers(self._h, radius), "set_nearfield_receivers")

    def receive(self, x, rx=None, order: int = ORDER_TREE, stream=None):
        """Receiver samples go x (near-field receivers) or the far-field aggregate."""
        import torch
        R = self._nrhs(x)
        if rx is None:
            rx = torch.empty((R, self.numrx) if x.dim() == 2 else (self.numrx,), dtype=torch.complex64,
                             device=x.device)
        self._check(lib().isg_receive(self._h, _ptr(x), _ptr(rx), R, order, _stream(stream)), "receive")
        return rx

    def receiveh(self, rx, x=None, order: int = ORDER_TREE, stream=None):
        """Back-projection conj(go)^T rx (near-field receivers) or the far-field aggregateh."""
        import torch
        R = 1 if rx.dim() == 1 else rx.shape[0]
        if x is None:
            x = torch.empty((R, self.numunk) if rx.dim() == 2 else (self.numunk,), dtype=torch.complex64,
                            device=rx.device)
        self._check(lib().isg_receiveh(self._h, _ptr(x), _ptr(rx), R, order, _stream(stream)), "receiveh")
        return x

    # ---- launch-shape autotuner ----
    def autotune(self, nrhs: int = 1, engine: int = ENGINE_TENSOR, stream=None) -> dict:
        """Times candidate launch shapes on nrhs RHS and keeps the fastest; returns the choices."""
        self._check(lib().isg_autotune(self._h, nrhs, engine, _stream(stream)), "autotune")
        return self.tuned()

    def tuned(self) -> dict:
        v = ctypes.c_int()
        out = {}
        for what, name in enumerate(("m2l_rows", "l2l_cols", "m2m_cols")):
            out[name] = []
            for lvl in range(self.level):
                self._check(lib().isg_tuned(self._h, what, lvl, ctypes.byref(v)), "tuned")
                out[name].append(v.value)
        self._check(lib().isg_tuned(self._h, 3, 0, ctypes.byref(v)), "tuned")
        out["near_pair"] = v.value
        return out

    # ---- learned warm start ----
    def fno_create(self, width: int = 32, modes: int = 12, layers: int = 4, batch: int = 4, seed: int = 1,
                   tensor: bool = True):
        """Attach a freshly initialised neural-operator warm start (ISG_GUESS_LEARNED); tensor: BF16
        tcgen05 products with FP32 accumulation (default), else FP32 on the CUDA cores."""
        o = FnoOpts()
        lib().isg_default_fno_opts(ctypes.byref(o))
        o.width, o.modes, o.layers, o.batch, o.seed, o.tensor = width, modes, layers, batch, seed, int(tensor)
        self._check(lib().isg_fno_create(self._h, ctypes.byref(o)), "fno_create")

    def fno_params(self, which: int = 0) -> np.ndarray:
        """Flat FP32 parameters (which 0) or the last gradient (which 1)."""
        n = lib().isg_fno_param_count(self._h)
        out = np.empty(n, dtype=np.float32)
        self._check(lib().isg_fno_params(self._h, out.ctypes.data, n, which, 0), "fno_params")
        return out

    def fno_set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(lib().isg_fno_params(self._h, p.ctypes.data, p.size, 0, 1), "fno_set_params")

    def fno_apply(self, g, b, order: int = ORDER_TREE, stream=None):
        """x = b + N(g, b): the warm start for the forward solves of b."""
        import torch
        x = torch.empty_like(b)
        gs = 0 if g.dim() == 1 else self.numunk
        self._check(lib().isg_fno_apply(self._h, _ptr(g), gs, _ptr(b), _ptr(x), self._nrhs(b), order,
                                        _stream(stream)), "fno_apply")
        return x

    def fno_grad(self, g, b, u=None, order: int = ORDER_TREE, stream=None) -> float:
        """Loss and gradient (fno_params(1)): field error against u, or the initial residual when u is None."""
        loss = ctypes.c_double()
        gs = 0 if g.dim() == 1 else self.numunk
        self._check(lib().isg_fno_grad(self._h, _ptr(g), gs, _ptr(b), _ptr(u), self._nrhs(b), order,
                                       ctypes.byref(loss), _stream(stream)), "fno_grad")
        return loss.value

    def fno_train_step(self, g, b, u=None, lr: float = 1e-3, order: int = ORDER_TREE, stream=None) -> float:
        loss = ctypes.c_double()
        gs = 0 if g.dim() == 1 else self.numunk
        self._check(lib().isg_fno_train_step(self._h, _ptr(g), gs, _ptr(b), _ptr(u), self._nrhs(b), order, lr,
                                             ctypes.byref(loss), _stream(stream)), "fno_train_step")
        return loss.value

    def time_stages(self, nrhs: int = 1, engine: int = ENGINE_SIMT, reps: int = 5) -> dict:
        """Mean device ms per matvec stage (P2M, M2M, M2L+L2L, L2P+near, total)."""
        out = np.zeros(5)
        self._check(lib().isg_time_stages(self._h, nrhs, engine, reps, out.ctypes.data), "time_stages")
        return dict(zip(("p2m", "m2m", "m2l_l2l", "near", "total"), out.tolist()))

    # ---- inversion ----
    def measure(self, inc, chi, noise: float = 0.0, seed: int = 0, order: int = ORDER_TREE, stream=None, **solve):
        """Synthetic far-field data of contrast chi (setup_born.cpp:139-149): (ntx, numrx) complex64."""
        import torch
        ntx = 1 if inc.dim() == 1 else inc.shape[0]
        mes = torch.empty((ntx, self.numrx), dtype=torch.complex64, device=inc.device)
        so = default_solve_opts(**{"tol": 1e-4, **solve})
        self._check(lib().isg_measure(self._h, ntx, _ptr(inc), _ptr(chi), order, noise, seed, ctypes.byref(so),
                                      _ptr(mes), _stream(stream)), "measure")
        return mes

    def dbim(self, inc, mes, chi=None, chi_true=None, iterations: int = 3, regular: float = 0.0,
             order: int = ORDER_TREE, start_from_chi: bool = False, warm_start: bool = False,
             checkpoint: str | None = None, stream=None, **solve):
        """The reference's inversion loop (mom.cpp:222-399); returns (chi, history records)."""
        import torch
        ntx = 1 if inc.dim() == 1 else inc.shape[0]
        if chi is None:
            chi = torch.zeros(self.numunk, dtype=torch.complex128, device=inc.device)
        o = DbimOpts()
        lib().isg_default_dbim_opts(ctypes.byref(o))
        o.iterations, o.regular, o.start_from_chi = iterations, regular, int(start_from_chi)
        o.warm_start = int(warm_start)
        o.checkpoint = checkpoint.encode() if checkpoint else None
        for k, v in solve.items():
            setattr(o.solve, k, v)
        hist = (DbimRecord * (iterations + 1))()
        self._check(lib().isg_dbim(self._h, ntx, _ptr(inc), _ptr(mes), _ptr(chi_true), _ptr(chi), order,
                                   ctypes.byref(o), hist, _stream(stream)), "dbim")
        return chi, [h.as_dict() for h in hist]

    def reorder(self, x, frm: int, to: int, out=None, stream=None):
        out = self._empty_like(x) if out is None else out
        self._check(lib().isg_reorder(self._h, _ptr(x), _ptr(out), self._nrhs(x), frm, to, _stream(stream)),
                    "reorder")
        return out

    # ---- seeded inputs ----
    def phantom(self, seed: int, count: int = 3, axis=(1.0, 3.0), eps=(1.1, 1.5), tand_max: float = 0.0,
                kind: int = 0, corr_len: float = 2.0) -> np.ndarray:
        """Contrast chi = eps_r - 1 (complex128, raster order)."""
        p = Phantom(kind, count, axis[0], axis[1], eps[0], eps[1], tand_max, corr_len, seed)
        out = np.zeros(self.numunk, np.complex128)
        self._check(lib().isg_make_phantom(self._h, ctypes.byref(p), out.ctypes.data), "phantom")
        return out

    def plane_waves(self, ntx: int, first: int = 0, count: int | None = None, order: int = ORDER_TREE) -> np.ndarray:
        n = ntx if count is None else count
        out = np.zeros((n, self.numunk), np.complex128)
        self._check(lib().isg_make_plane_waves(self._h, ntx, first, n, order, out.ctypes.data), "plane_waves")
        return out

    def line_sources(self, ntx: int, radius: float, first: int = 0, count: int | None = None,
                     order: int = ORDER_TREE) -> np.ndarray:
        n = ntx if count is None else count
        out = np.zeros((n, self.numunk), np.complex128)
        self._check(lib().isg_make_line_sources(self._h, ntx, first, n, radius, order, out.ctypes.data),
                    "line_sources")
        return out

    def raster_to_tree(self, a: np.ndarray) -> np.ndarray:
        """Raster-order host array to tree order (the reference's o[unkmap[n]] = val, setup_born.cpp:105-112)."""
        um = self.host_table("unkmap")
        out = np.empty_like(a)
        out[..., um] = a
        return out
