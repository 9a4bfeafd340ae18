"""ctypes front end of the CPU restatement (libpatref.so) and a runner for the
compiled reference (_ref/ref_harness).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py's CPU-baseline leg.  The product never imports
this module.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpatref.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.patref_set_basis.argtypes = [ctypes.c_int, ip, ip, ip, ip, ip, dp, dp, ctypes.c_int, dp, dp, ctypes.c_int]
        L.patref_boys.argtypes = [ctypes.c_int, ctypes.c_double, dp]
        L.patref_rys.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.patref_eri_block.argtypes = [ctypes.c_int] * 4 + [dp]
        L.patref_gmat.argtypes = [ctypes.c_int, dp, dp, dp, dp, ctypes.c_int]
        L.patref_gmat.restype = ctypes.c_longlong
        L.patref_oneints.argtypes = [dp, dp, dp]
        L.patref_dpm.argtypes = [dp]
        L.patref_enuc.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


class Oracle:
    """Restatement bound to one basis (the library keeps one basis at a time)."""

    def __init__(self, basis):
        self.basis = basis
        self._keep = basis.flat_arrays()
        f = self._keep
        lib().patref_set_basis(basis.nshell, _p(f["l"], ctypes.c_int), _p(f["cen"], ctypes.c_int),
                               _p(f["off"], ctypes.c_int), _p(f["nst"], ctypes.c_int),
                               _p(f["prim_off"], ctypes.c_int), _p(f["alpha"]), _p(f["coef"]),
                               basis.ncen, _p(f["charges"]), _p(f["coords"]), basis.skipcen)

    @staticmethod
    def boys(m, T):
        F = np.zeros(m + 1)
        lib().patref_boys(m, T, _p(F))
        return F

    @staticmethod
    def rys(n, T):
        x = np.zeros(n)
        w = np.zeros(n)
        if lib().patref_rys(n, T, _p(x), _p(w)) != 0:
            raise ValueError("bad root count")
        return x, w

    def eri_block(self, a, b, c, d):
        sh = self.basis.shells
        out = np.zeros(sh[a].nst * sh[b].nst * sh[c].nst * sh[d].nst)
        lib().patref_eri_block(a, b, c, d, _p(out))
        return out.reshape(sh[a].nst, sh[b].nst, sh[c].nst, sh[d].nst)

    def gmat(self, PA, PB=None, start=0):
        no2 = self.basis.norb * (self.basis.norb + 1) // 2
        PA = np.ascontiguousarray(PA, dtype=np.float64)
        uhf = PB is not None
        PB = np.ascontiguousarray(PB if uhf else PA, dtype=np.float64)
        GA = np.zeros(no2)
        GB = np.zeros(no2)
        lib().patref_gmat(1 if uhf else 0, _p(PA), _p(PB), _p(GA), _p(GB), start)
        return (GA, GB) if uhf else GA

    def oneints(self):
        no2 = self.basis.norb * (self.basis.norb + 1) // 2
        S, T, H = np.zeros(no2), np.zeros(no2), np.zeros(no2)
        lib().patref_oneints(_p(S), _p(T), _p(H))
        return S, T, H

    def dpm(self, H):
        H = np.array(H, dtype=np.float64)
        lib().patref_dpm(_p(H))
        return H

    def enuc(self):
        return lib().patref_enuc()


# ---------------------------------------------------------------- reference
def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_harness"))


def run_ref(basis, cmd, inputs=None, posgrid=None, outputs=(), timeout=3600):
    """Run _ref/ref_harness <cmd...> in a fresh directory holding the basis's
    patin.dat; returns (stdout, {name: array}) for the binary outputs."""
    with tempfile.TemporaryDirectory(prefix="patref_") as d:
        basis.write_patin(os.path.join(d, "patin.dat"))
        if posgrid is not None:
            with open(os.path.join(d, "posgrid.dat"), "w") as f:
                f.write(f"{len(posgrid)}\n")
                for p in posgrid:
                    f.write(f"{p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
        for name, arr in (inputs or {}).items():
            np.ascontiguousarray(arr, dtype=np.float64).tofile(os.path.join(d, name))
        r = subprocess.run([os.path.join(REF_DIR, "ref_harness")] + list(cmd), cwd=d,
                           capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_harness {cmd} failed: {r.stderr[-2000:]}")
        outs = {}
        for name in outputs:
            path = os.path.join(d, name)
            if name == "eri.bin":
                dt = np.dtype([("val", "<f8"), ("i", "<u2"), ("j", "<u2"), ("k", "<u2"), ("l", "<u2")])
                outs[name] = np.fromfile(path, dtype=dt)
            elif name.endswith(".txt"):
                outs[name] = open(path).read()
            else:
                outs[name] = np.fromfile(path, dtype=np.float64)
        return r.stdout, outs


def ref_scf(basis, posgrid=None):
    out, _ = run_ref(basis, ["scf"], posgrid=posgrid)
    return json.loads(out.strip().splitlines()[-1])
