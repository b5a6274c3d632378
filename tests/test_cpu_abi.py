"""Host-side checks of the C ABI that need no GPU.

libqqcd_gpu.so loads, exports every entry point include/qqcd_gpu.h declares, rejects
bad arguments before touching a device, reports a missing GPU with QQ_NO_DEVICE
instead of falling back to the CPU, and its host-only part -- the reference's
lagged-Fibonacci generator (G/lagfib.f90), which the noise sources draw from --
matches the oracle bit for bit."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import baylorlqcd_b200 as qq
import oracle

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "qqcd_gpu.h"


def header_symbols():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(qq_\w+)\s*\(", text)))


def gpu_present():
    import torch

    return torch.cuda.is_available()


def test_header_lists_the_exported_symbols():
    assert header_symbols() == sorted(qq.EXPORTED)


def test_library_exports_every_header_symbol():
    lib = C.CDLL(str(qq.LIB_PATH))
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_declares_every_symbol():
    lib = qq.load_library()
    for s in header_symbols():
        f = getattr(lib, s)
        assert f.restype is not None or s == "qq_last_error"
        assert f.argtypes is not None


@pytest.mark.parametrize("dims,msg", [((6, 4, 4, 8), "multiples of 4"), ((4, 4, 4, 0), "multiples of 4")])
def test_bad_geometry_rejected_before_device(dims, msg):
    with pytest.raises(qq.QQError) as e:
        qq.Lattice(*dims)
    assert e.value.status == qq.QQ_BAD_ARG and msg in str(e.value)


def test_bad_boundary_rejected():
    with pytest.raises(qq.QQError) as e:
        qq.Lattice(4, 4, 4, 8, bc=(1, 1, 2, -1))
    assert e.value.status == qq.QQ_BAD_ARG


def test_uneven_batch_rejects_bad_arguments_before_device():
    """qq_fermprop_uneven checks every group before it starts a solve (no device needed)."""
    lib = qq.load_library()
    meth = qq.qq_method(16, 6, 32, 4, 1e-10, 0, 1, 0, 1e-5)
    assert lib.qq_fermprop_uneven(0, None, C.byref(meth), 1, None) == qq.QQ_BAD_ARG
    buf = np.zeros(8)
    groups = (qq.qq_uneven_group * 2)()
    for i in range(2):  # null context in both groups (positional, as fermprop_uneven builds them)
        groups[i] = qq.qq_uneven_group(None, 1, (C.c_double * 2)(0.15, 0.0), buf.ctypes.data, buf.ctypes.data,
                                       buf.ctypes.data, buf.ctypes.data, None)
    assert lib.qq_fermprop_uneven(2, groups, C.byref(meth), 1, None) == qq.QQ_BAD_ARG
    assert b"group 0" in lib.qq_last_error()


def test_loop_driver_entry_points_reject_bad_arguments_before_device():
    """qq_vev and qq_discon check their context and arguments first (no device needed)."""
    lib = qq.load_library()
    io = (C.c_int * 3)(1, 1, 1)
    J = np.zeros(2 * 8 * 6 * 5 * 9)
    assert lib.qq_vev(None, 0.15, io, J.ctypes.data, None, None) == qq.QQ_BAD_ARG
    meth = qq.qq_method(16, 6, 32, 4, 1e-10, 0, 0, 0, 1e-5)
    assert lib.qq_discon(None, 2, 1, 0.15, C.byref(meth), io, 6, 5, 5, J.ctypes.data, None, None) == qq.QQ_BAD_ARG
    assert b"null" in lib.qq_last_error()


def test_missing_gpu_fails_loudly():
    """No CPU fallback: without a device the context cannot be created."""
    if gpu_present():
        pytest.skip("a GPU is present")
    with pytest.raises(qq.QQError) as e:
        qq.Lattice(4, 4, 4, 8)
    assert e.value.status == qq.QQ_NO_DEVICE


def test_package_never_touches_the_oracle():
    """The oracle is test infrastructure: nothing in the product imports or loads it."""
    for p in list((ROOT / "baylorlqcd_b200").rglob("*.py")) + list((ROOT / "baylorlqcd_b200" / "csrc").glob("*")):
        text = p.read_text(errors="replace")
        assert not re.search(r"\boracle\b|liboracle|oq_", text), p


@pytest.mark.parametrize("myid,iseed", [(0, 13), (0, 0), (3, 13), (0, 987654), (7, 2**20)])
def test_lagfib_bit_exact_with_oracle(myid, iseed):
    qq.initlagfib(myid, iseed)
    a = np.concatenate([qq.rnds(1000), qq.rnds(3000)])  # state carries across calls
    oracle.initlagfib(myid, iseed)
    b = oracle.rnds(4000)
    assert np.array_equal(a, b)
    assert a.min() > 0.0 and a.max() < 1.0


def test_lagfib_seeds_differ():
    qq.initlagfib(0, 13)
    a = qq.rnds(64)
    qq.initlagfib(1, 13)
    b = qq.rnds(64)
    assert not np.array_equal(a, b)


def test_lagfib_rejects_negative_delay():
    with pytest.raises(qq.QQError) as e:
        qq.initlagfib(0, -13)
    assert e.value.status == qq.QQ_BAD_ARG
    with pytest.raises(ValueError):
        oracle.initlagfib(0, -13)


def test_rnds_argument_checks():
    lib = qq.load_library()
    assert lib.qq_rnds(-1, None) == qq.QQ_BAD_ARG
    assert b"rnds" in lib.qq_last_error()
