"""Shared fixtures: repo on sys.path, the `gpu` marker, and the CPU checkers.

``-m "not gpu"`` runs everything that needs no GPU: the oracle against the
golden fixtures, the host-compiled copy of the device evaluator against the
oracle, host-side logic and the C ABI's exported symbols.  ``-m gpu`` runs the
parity tests proper through the C ABI on a B200.
"""
from __future__ import annotations

import ctypes
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

HOSTEMU_SRC = ROOT / "tests" / "hostemu" / "hostemu.cpp"
HOSTEMU_LIB = ROOT / "tests" / "hostemu" / "libksim_hostemu.so"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs through libksim_b200.so)")


@pytest.fixture(scope="session")
def oracle_port():
    """Build (if needed) and return the oracle module with the C port loaded."""
    from oracle import oracle
    if not oracle.PORT_LIB.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "port"], check=True)
    return oracle


@pytest.fixture(scope="session")
def oracle_module(oracle_port):
    """The oracle module (``program_sample`` and the oracle classes)."""
    return oracle_port


@pytest.fixture(scope="session")
def ref_oracle(oracle_port):
    """The reference's own zx_eval.hpp (``oracle/_ref``) as an oracle class;
    the C restatement (pinned to it bit for bit by the CPU suite) where that
    library was not built."""
    if oracle_port.RefOracle.available():
        return oracle_port.RefOracle
    import warnings
    warnings.warn("oracle/_ref is not built: checking against the C restatement")
    return oracle_port.PortOracle


def _build_hostemu():
    srcs = [HOSTEMU_SRC, ROOT / "ksim_b200" / "csrc" / "image.cpp"]
    deps = srcs + list((ROOT / "ksim_b200" / "csrc").glob("*.cuh")) + \
        list((ROOT / "ksim_b200" / "csrc").glob("*.h"))
    if HOSTEMU_LIB.exists() and HOSTEMU_LIB.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
                    "-I", str(ROOT / "ksim_b200" / "csrc"), "-o", str(HOSTEMU_LIB),
                    *map(str, srcs)], check=True)


@pytest.fixture(scope="session")
def hostemu():
    """ctypes handle on the host-compiled device evaluator (test-only)."""
    from ksim_b200._abi import GraphDesc
    _build_hostemu()
    L = ctypes.CDLL(str(HOSTEMU_LIB))
    u8p = ctypes.POINTER(ctypes.c_uint8)
    L.hostemu_eval.argtypes = [ctypes.POINTER(GraphDesc), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               u8p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                               ctypes.c_void_p]
    L.hostemu_sample.argtypes = [ctypes.POINTER(GraphDesc), ctypes.c_int, ctypes.c_int, u8p,
                                 ctypes.c_int64, ctypes.c_uint64, ctypes.c_int, u8p,
                                 ctypes.c_void_p]
    L.hostemu_stats.argtypes = [ctypes.POINTER(GraphDesc), ctypes.c_int, ctypes.c_int,
                                ctypes.c_void_p]
    L.hostemu_error.restype = ctypes.c_char_p
    L.hostemu_valuation.argtypes = [ctypes.c_void_p]
    L.hostemu_valuation.restype = ctypes.c_uint32
    return L


@pytest.fixture(scope="session")
def cuda_device():
    """Fail (not skip) when a gpu-marked test runs without a usable device."""
    from ksim_b200._abi import lib
    n = lib().ksim_device_count()
    assert n > 0, "no CUDA device visible to libksim_b200.so"
    return 0
