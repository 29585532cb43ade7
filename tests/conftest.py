"""Shared fixtures.  Tests marked `gpu` need a B200 and run the native
library; everything else runs on the CPU (oracle, compiler, host logic,
host-compiled device arithmetic)."""

from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"
FIXTURES = GOLDEN / "fixtures"
HOSTSIM_SRC = ROOT / "tests" / "hostsim" / "hostsim.cpp"
HOSTSIM_LIB = ROOT / "tests" / "hostsim" / "libhostsim.so"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 GPU and the native library")


@pytest.fixture(scope="session")
def hostsim():
    """The device code's arithmetic compiled for the host (test-only)."""
    csrc = ROOT / "gpjson_b200" / "csrc"
    deps = [HOSTSIM_SRC, csrc / "host_io.h"] + list(csrc.glob("*.cuh"))
    if not HOSTSIM_LIB.exists() or any(d.stat().st_mtime > HOSTSIM_LIB.stat().st_mtime for d in deps):
        # built beside the target and renamed over it, so that a library
        # mapped by another process is never rewritten in place
        tmp = HOSTSIM_LIB.with_suffix(f".{os.getpid()}.tmp")
        subprocess.run(
            ["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-pthread", "-o", str(tmp), str(HOSTSIM_SRC)],
            check=True,
        )
        tmp.replace(HOSTSIM_LIB)
    L = ctypes.CDLL(str(HOSTSIM_LIB))
    P = ctypes.c_void_p
    L.hs_build_index.restype = ctypes.c_int64
    L.hs_build_index.argtypes = [P, ctypes.c_int64, ctypes.c_int, P, P, P, ctypes.c_int64]
    L.hs_build_index_lines.restype = ctypes.c_int64
    L.hs_build_index_lines.argtypes = [P, ctypes.c_int64, ctypes.c_int, P, P, P, ctypes.c_int64]
    L.hs_find_values.restype = None
    L.hs_find_values.argtypes = [P, ctypes.c_int64, P, ctypes.c_int64, P, P, ctypes.c_int, P, ctypes.c_int, P, P,
                                 ctypes.c_int]
    L.hs_query_items.restype = ctypes.c_int64
    L.hs_query_items.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int64, P]
    L.hs_classify.restype = None
    L.hs_classify.argtypes = [P, ctypes.c_int64, P]
    L.hs_escaped_mask.restype = ctypes.c_uint64
    L.hs_escaped_mask.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
    L.hs_read_ranges.restype = ctypes.c_int
    L.hs_read_ranges.argtypes = [ctypes.c_char_p, P, P, P, ctypes.c_int, ctypes.c_int]
    L.hs_rb_new.restype = P
    L.hs_rb_new.argtypes = []
    L.hs_rb_delete.restype = None
    L.hs_rb_delete.argtypes = [P]
    L.hs_rb_take.restype = P
    L.hs_rb_take.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
    L.hs_rb_give.restype = None
    L.hs_rb_give.argtypes = [P, P, ctypes.c_uint64]
    L.hs_rb_keep_elems.restype = ctypes.c_uint64
    L.hs_rb_keep_elems.argtypes = []
    return L


@pytest.fixture(scope="session")
def gpjson():
    """A native GPJSON context on cuda:0 (GPU tests only)."""
    import gpjson_b200 as gj

    g = gj.GPJSON(0)
    yield g
    g.close()


def fixture_bytes(rel: str) -> bytes:
    return (FIXTURES / rel).read_bytes()
