"""Generates the committed golden fixtures (run from the repository root):

    python tests/golden/gen_golden.py

tdma_ref.npz   -- seeded diagonally dominant systems (plain and cyclic) and
                  their solutions computed by the reference's own
                  00_C/PaScaL_TDMA/src/tdmas.cpp (tdma_many, tdma_cycl_many),
                  compiled from the reference tree by oracle/Makefile.  Note:
                  that file's tdma_cycl_many indexes with the row count as the
                  stride, so its cyclic result is only the cyclic solve when
                  n_sys == n_row; the cyclic cases here are square.
solve_npref.npz -- seeded small Poisson problems for all four x/y boundary
                  pairs, uniform and stretched z, periodic and Neumann z, with
                  the solution of tests/npref.py (an independent scipy.fft /
                  numpy restatement of the method).
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle as O  # noqa: E402
import npref  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def dd_system(rng, n_sys, n_row):
    a = rng.uniform(-1, 1, (n_row, n_sys))
    c = rng.uniform(-1, 1, (n_row, n_sys))
    b = (np.abs(a) + np.abs(c) + rng.uniform(0.5, 2.0, (n_row, n_sys))) * rng.choice([-1.0, 1.0], (n_row, n_sys))
    d = rng.standard_normal((n_row, n_sys))
    return a, b, c, d


def gen_tdma():
    ref = O.ref_tdmas()
    if ref is None:
        raise SystemExit("oracle/_ref/libref_tdmas.so missing: run make -C oracle with the reference tree present")
    rng = np.random.Generator(np.random.PCG64(20240601))
    out = {}
    dp = ctypes.POINTER(ctypes.c_double)
    cases = [("many", 7, 9), ("many", 33, 64), ("many", 5, 1), ("many", 4, 2), ("many", 128, 17),
             ("cycl", 9, 9), ("cycl", 16, 16), ("cycl", 3, 3)]
    for i, (kind, ns, nr) in enumerate(cases):
        a, b, c, d = dd_system(rng, ns, nr)
        aa, bb, cc, xx = (np.ascontiguousarray(v.copy()) for v in (a, b, c, d))
        fn = ref.tdma_many if kind == "many" else ref.tdma_cycl_many
        fn(aa.ctypes.data_as(dp), bb.ctypes.data_as(dp), cc.ctypes.data_as(dp), xx.ctypes.data_as(dp), ns, nr)
        for k, v in (("a", a), ("b", b), ("c", c), ("d", d), ("x", xx)):
            out[f"{i}_{k}"] = v
        out[f"{i}_kind"] = np.array(kind)
    out["ncases"] = np.array(len(cases))
    np.savez_compressed(os.path.join(HERE, "tdma_ref.npz"), **out)


def gen_solve():
    rng = np.random.Generator(np.random.PCG64(7))
    out = {}
    i = 0
    for (n1, n2, n3) in [(8, 6, 5), (16, 12, 10)]:
        for pbc in [(1, 1, 0), (0, 0, 0), (0, 1, 0), (1, 0, 0), (1, 1, 1)]:
            for beta in (0.0, 1.5):
                if pbc[2] and beta:
                    continue
                L1, L2, L3 = 2 * np.pi, 3.0, 1.0
                _, _, dmx1 = npref.mesh(n1, L1, True, 0.0, pbc[0])
                _, _, dmx2 = npref.mesh(n2, L2, True, 0.0, pbc[1])
                _, dx3, dmx3 = npref.mesh(n3, L3, beta == 0.0, 2 * beta, pbc[2])
                f = rng.standard_normal((n3, n2, n1))
                P = npref.solve(f, L1, L2, pbc, dmx1, dmx2, dmx3, dx3)
                for k, v in (("f", f), ("P", P), ("dmx1", dmx1), ("dmx2", dmx2), ("dmx3", dmx3), ("dx3", dx3)):
                    out[f"{i}_{k}"] = v
                out[f"{i}_meta"] = np.array([n1, n2, n3, *pbc], dtype=np.int64)
                out[f"{i}_L"] = np.array([L1, L2, L3])
                i += 1
    out["ncases"] = np.array(i)
    np.savez_compressed(os.path.join(HERE, "solve_npref.npz"), **out)


if __name__ == "__main__":
    gen_tdma()
    gen_solve()
    print("written", os.listdir(HERE))
