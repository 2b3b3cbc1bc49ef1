"""The C ABI: libisg.so loads, exports every entry point include/*.h declares,
and rejects bad arguments, all without touching a GPU."""
import ctypes
import glob
import os
import re

import pytest

import isg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        if "extern \"C\"" not in src:
            continue
        for m in re.finditer(r"\b(isg_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = isg.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_the_abi():
    missing = [n for n in declared_functions() if n not in isg.SIGNATURES]
    assert not missing, missing


def test_create_rejects_bad_options():
    L = isg.lib()
    o = isg.Opts()
    L.isg_default_opts(ctypes.byref(o))
    h = ctypes.c_void_p()
    for field, bad in (("level", 2), ("box", 4), ("ninter", 7), ("numrx", 0), ("max_rhs", 0), ("k0", -1.0)):
        o2 = isg.Opts.from_buffer_copy(o)
        setattr(o2, field, bad)
        assert L.isg_create(ctypes.byref(o2), ctypes.byref(h)) == 5, field


def test_create_needs_no_gpu_and_reports_sizes():
    s = isg.Solver(6, numrx=64)
    assert s.numunk == 256 * 256 and s.side == 256
    assert [s.numsamp(i) for i in range(6)] == [1036, 556, 308, 176, 104, 68]
    assert isg.lib().isg_levels(s._h) == 6


def test_status_strings():
    L = isg.lib()
    assert L.isg_status_string(0) == b"ok"
    assert L.isg_status_string(2) == b"breakdown"


def test_unknown_table_is_bad_arg():
    s = isg.Solver(4)
    with pytest.raises(isg.IsgError):
        s.host_table("no_such_table")


def test_refapi_library_exports_the_reference_names():
    """libisg_ref.so defines every routine of include/isg_refapi.h under the
    reference's own C++ names and leaves the driver's globals undefined."""
    import subprocess
    lib = os.path.join(ROOT, "inverse-solver-gpu_b200", "isg", "libisg_ref.so")
    out = subprocess.run(["nm", "-D", "-C", lib], capture_output=True, text=True, check=True).stdout
    defined = {ln.split(" T ", 1)[1].strip() for ln in out.splitlines() if " T " in ln}
    c = "std::complex<double>*"
    want = ["setup_mlfma()", "setup_gpu()", "setup_bicgs()", f"bicgs({c}, {c}, {c}, bool)",
            f"matvec({c}, {c}, {c}, bool)", f"mlfma({c}, {c})", f"mlfmah({c}, {c})", f"aggregate({c}, {c})",
            f"aggregateh({c}, {c})"]
    assert not [w for w in want if w not in defined], defined
    undefined = {ln.split()[-1] for ln in out.splitlines() if " U " in ln}
    for g in ("res", "box", "level", "k0", "numunk", "numrx", "toli", "iti", "pos", "unkmap"):
        assert g in undefined, g


def test_library_does_not_need_the_driver_library():
    """libisg.so records only the CUDA runtime: the driver entry points it uses
    (tensor-map encoding) are looked up at run time, so the library loads on a
    machine without a driver and fails there with ISG_NO_DEVICE instead."""
    import subprocess
    out = subprocess.run(["readelf", "-d", isg.LIBPATH], capture_output=True, text=True, check=True).stdout
    needed = re.findall(r"\(NEEDED\)\s+Shared library: \[([^\]]+)\]", out)
    assert any(n.startswith("libcudart") for n in needed), needed
    assert not [n for n in needed if n.startswith("libcuda.")], needed


def test_create_rejects_batches_wider_than_a_grid_row_limit():
    o = isg.Opts()
    isg.lib().isg_default_opts(ctypes.byref(o))
    h = ctypes.c_void_p()
    o.level, o.max_rhs = 4, 65536
    assert isg.lib().isg_create(ctypes.byref(o), ctypes.byref(h)) == 5
    o.max_rhs = 65535
    assert isg.lib().isg_create(ctypes.byref(o), ctypes.byref(h)) == 0
    isg.lib().isg_destroy(h)
