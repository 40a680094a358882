"""The C ABI library loads and exports what include/ppf.h declares; the
host-side validation paths run without a GPU."""
import os
import re

import pytest

import pascal_poisson_fft_b200 as ppf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "ppf.h")).read()
    return sorted(set(re.findall(r"PPF_API\s+(?:const\s+)?\w+\s*\*?\s*(ppf_\w+)\s*\(", txt)))


def test_header_lists_every_symbol():
    assert header_symbols() == sorted(ppf.EXPORTED_SYMBOLS)


def test_library_exports_every_header_symbol():
    L = ppf.lib()
    for name in header_symbols():
        assert hasattr(L, name), name


def header_prototypes():
    """name -> list of parameter declarations, from include/ppf.h"""
    txt = open(os.path.join(ROOT, "include", "ppf.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"PPF_API\s+(?:const\s+)?\w+\s*\*?\s*(ppf_\w+)\s*\(([^)]*)\)", txt):
        params = " ".join(m.group(2).split())
        out[m.group(1)] = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
    return out


def test_every_binding_declares_its_argument_types():
    """Without argtypes ctypes passes a Python int as a 32-bit C int, which
    truncates device pointers and stream handles: every exported function
    has them, one per declared parameter, pointer parameters as pointers."""
    import ctypes
    L = ppf.lib()
    for name, params in header_prototypes().items():
        at = getattr(L, name).argtypes
        assert at is not None, name
        assert len(at) == len(params), (name, len(at), params)
        for decl, t in zip(params, at):
            if "*" in decl:
                assert t is ctypes.c_void_p or issubclass(t, ctypes._Pointer), (name, decl, t)
            elif decl.split()[0] == "int":
                assert t is ctypes.c_int, (name, decl, t)
            elif decl.split()[0] == "double":
                assert t is ctypes.c_double, (name, decl, t)


def test_version_string():
    assert b"sm_100a" in ppf.lib().ppf_version()


@pytest.mark.parametrize("args,msg", [
    ((7, 8, 8), "even"),
    ((8, 8, 2), "too small"),
    ((14, 8, 8), "not a product"),
    ((8, 8, 2000), "1024"),
])
def test_descriptor_validation(args, msg):
    with pytest.raises(ppf.PPFError) as e:
        ppf.Plan(*args, 1.0, 1.0)
    assert msg in str(e.value)


def test_tdma_argument_validation():
    L = ppf.lib()
    assert L.ppf_tdma_many(None, None, None, None, 4, 4, None) == -1
    assert b"null" in L.ppf_last_error()
    assert L.ppf_tdma_cycl_many(1, 1, 1, 1, 4, 2, None) == -1


def test_module_api_state_errors():
    L = ppf.lib()
    L.ppf_cuda_poisson_fft_clean()
    assert L.ppf_cuda_poisson_fft_initial() == -5          # PPF_ERR_STATE
    assert L.ppf_cuda_poisson_fft_1d(1, 1, 1, 1, 1, 1) == -5


def test_post_argument_validation():
    L = ppf.lib()
    assert L.ppf_ghost_update(None, 4, 4, 4, 1, 1, 0, None, None, None, 1, None) == -1
    assert b"null" in L.ppf_last_error()
    # a wall axis (z here) needs its dmx array for the Neumann extrapolation
    assert L.ppf_ghost_update(1, 4, 4, 4, 1, 1, 0, None, None, None, 1, None) == -1
    assert b"wall axis 3" in L.ppf_last_error()
    assert L.ppf_cell_to_node(None, 4, 4, 4, None, None, None, None, None) == -1
