"""The C++ driver's solve calls (libppf_cxx.so, include/ppf_cxx_driver.h):
mpi_poisson::mpi_Poisson_FFT{1..5}(dx2, dmx2) reading the global PRHS and
writing the global P in the driver's axis order (x2 = wall-normal axis,
00_C/examples/modules.hpp:223-232, module_solve_poisson.cpp:47-52).

A harness translation unit defines the driver's globals (as the driver's own
module_global.cpp / module_mpi_subdomain.cpp do) and is linked against
libppf_cxx.so with g++.  Without a GPU: the library loads against the
harness, exports what its header declares, and rejects bad set-ups.  On the
GPU: the result, read back from P, equals the handle API's solve of the
axis-permuted problem bit for bit and the oracle within the FP64 tolerance."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import pascal_poisson_fft_b200 as ppf
from pascal_poisson_fft_b200 import workloads as W
from _util import gpu_solve, oracle_solve, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pascal_poisson_fft_b200")
TOL64 = 1e-12
_dp = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = os.path.join(PKG, "libppf_cxx.so")
    if not os.path.exists(cxx):
        from pascal_poisson_fft_b200 import build as b
        b.build_cxx_driver()
    out = str(tmp_path_factory.mktemp("cxx") / "libharness.so")
    subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-o", out,
                    os.path.join(ROOT, "tests", "cxx_driver", "harness.cpp"), f"-L{PKG}", "-l:libppf_cxx.so",
                    f"-Wl,-rpath,{PKG}"], check=True)
    H = ctypes.CDLL(out, mode=ctypes.RTLD_GLOBAL)
    H.harness_setup.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [ctypes.c_int] * 4 + [_dp, _dp]
    H.harness_set_prhs.argtypes = [_dp, ctypes.c_long]
    H.harness_get_p.argtypes = [_dp, ctypes.c_long]
    H.harness_get_p.restype = ctypes.c_long
    D = ctypes.CDLL(os.path.join(PKG, "libppf_cxx.so"), mode=ctypes.RTLD_GLOBAL)
    D.ppf_cxx_poisson_fft.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int]
    D.ppf_cxx_last_error.restype = ctypes.c_char_p
    return H, D


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)


def header_c_symbols():
    txt = open(os.path.join(ROOT, "include", "ppf_cxx_driver.h")).read()
    return sorted(set(re.findall(r"PPF_CXX_API\s+(?:const\s+)?\w+\s*\*?\s*(ppf_cxx_\w+)\s*\(", txt)))


def test_library_exports_what_the_header_declares(harness):
    _, D = harness
    names = header_c_symbols()
    assert names == ["ppf_cxx_last_error", "ppf_cxx_poisson_fft", "ppf_cxx_release", "ppf_cxx_set_precision"]
    for n in names:
        assert hasattr(D, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(PKG, "libppf_cxx.so")],
                         capture_output=True, text=True, check=True).stdout
    for v in range(1, 6):
        # mpi_poisson::mpi_Poisson_FFT<v>(std::vector<double> const&, std::vector<double> const&)
        assert f"_ZN11mpi_poisson16mpi_Poisson_FFT{v}ERKSt6vectorIdSaIdEES4_" in out


def _setup_driver(H, p, np1=1):
    """Our problem p (x, y, z = wall) set up in the driver's axes
    (x1 = x, x2 = z, x3 = y); returns (dx2, dmx2)."""
    m = p.metrics
    H.harness_setup(p.n1m, p.n3m, p.n2m, p.L1, p.L3, p.L2, int(p.pbc[0]), int(p.pbc[2]), int(p.pbc[1]),
                    np1, _p(m["dmx1"]), _p(m["dmx2"]))
    prhs = np.ascontiguousarray(p.f.transpose(1, 0, 2))      # (z, y, x) -> (k = y, j = z, i = x)
    H.harness_set_prhs(_p(prhs), prhs.size)
    return np.ascontiguousarray(m["dx3"]), np.ascontiguousarray(m["dmx3"])


def test_rejects_bad_setups_without_touching_the_gpu(harness):
    H, D = harness
    p = W.random_problem(np.random.default_rng(5), 16, 12, 10, (1, 1, 0))
    dx2, dmx2 = _setup_driver(H, p, np1=2)
    assert D.ppf_cxx_poisson_fft(1, _p(dx2), _p(dmx2), dx2.size) == -1
    assert b"one subdomain per GPU" in D.ppf_cxx_last_error()
    dx2, dmx2 = _setup_driver(H, p)
    assert D.ppf_cxx_poisson_fft(1, _p(dx2), _p(dmx2), 3) == -1
    assert b"dx2/dmx2" in D.ppf_cxx_last_error()
    assert D.ppf_cxx_poisson_fft(6, _p(dx2), _p(dmx2), dx2.size) == -1
    assert D.ppf_cxx_set_precision(5, 0) == -1


@pytest.mark.gpu
@pytest.mark.parametrize("pbc,variant", [((1, 1, 0), 1), ((1, 0, 0), 4), ((0, 1, 0), 2), ((0, 0, 0), 5),
                                         ((1, 1, 1), 3)])
def test_driver_solve_equals_handle_api(harness, pbc, variant):
    H, D = harness
    rng = np.random.default_rng(40 + variant)
    p = W.random_problem(rng, 48, 40, 36, pbc, beta=0.0 if pbc[2] else 1.5)
    dx2, dmx2 = _setup_driver(H, p)
    rc = D.ppf_cxx_poisson_fft(variant, _p(dx2), _p(dmx2), dx2.size)
    assert rc == 0, D.ppf_cxx_last_error()
    n = (p.n1m + 2) * (p.n2m + 2) * (p.n3m + 2)
    out = np.empty(n)
    assert H.harness_get_p(out.ctypes.data_as(_dp), n) == n
    P_drv = out.reshape(p.n2m + 2, p.n3m + 2, p.n1m + 2).transpose(1, 0, 2)   # (k, j, i) -> (z, y, x)
    assert np.array_equal(P_drv, gpu_solve(p))
    assert rel_l2(P_drv, oracle_solve(p)) < TOL64


@pytest.mark.gpu
def test_driver_mixed_precision(harness):
    H, D = harness
    p = W.random_problem(np.random.default_rng(47), 64, 48, 40, (1, 1, 0), beta=1.5)
    dx2, dmx2 = _setup_driver(H, p)
    assert D.ppf_cxx_set_precision(ppf.PPF_MIXED, 3) == 0
    try:
        assert D.ppf_cxx_poisson_fft(1, _p(dx2), _p(dmx2), dx2.size) == 0, D.ppf_cxx_last_error()
    finally:
        D.ppf_cxx_set_precision(ppf.PPF_FP64, 0)
    n = (p.n1m + 2) * (p.n2m + 2) * (p.n3m + 2)
    out = np.empty(n)
    H.harness_get_p(out.ctypes.data_as(_dp), n)
    P_drv = out.reshape(p.n2m + 2, p.n3m + 2, p.n1m + 2).transpose(1, 0, 2)
    assert rel_l2(P_drv, oracle_solve(p)) < 1e-10
    assert D.ppf_cxx_release() == 0
