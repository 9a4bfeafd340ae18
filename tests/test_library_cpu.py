"""Host-side checks that need no GPU: the C-ABI library loads and exports
every entry point include/patgpu.h declares, refuses to run without a
device (no CPU fallback), its Rys tables match the quad-precision oracle,
and the quartet bookkeeping matches the workload's published sizes."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from patmol_b200 import configs, workload
from patmol_b200.basis import Basis, pack, unpack, packed_index
import patref

HEADER = os.path.join(ROOT, "include", "patgpu.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ \*]*?\b([a-z_][a-z0-9_]*)\s*\(",
                                 txt, flags=re.M)) - {"if", "while"})


def test_library_exports_every_declared_symbol():
    from patmol_b200 import gpu
    L = gpu.lib()
    names = declared_functions()
    assert "two_electron_ints" in names and "patgpu_rhf_gmatrix" in names
    for n in names:
        assert hasattr(L, n), n


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-device path")
def test_no_cpu_fallback_without_device():
    from patmol_b200 import gpu
    with pytest.raises(gpu.PatgpuError) as e:
        gpu.GpuBasis(configs.water_spd())
    assert "no CUDA device" in str(e.value)


def test_rys_tables_match_oracle():
    from patmol_b200 import gpu
    rng = np.random.default_rng(3)
    worst = 0.0
    for n in range(1, 10):
        Ts = np.concatenate([rng.uniform(0, 100, 60), [0.0, 1e-9, 0.999999, 41.99, 42.0, 90.5, 91.0, 500.0, 1e6]])
        for T in Ts:
            x, w = gpu.rys_host(n, T)
            xo, wo = patref.Oracle.rys(n, float(T))
            worst = max(worst, np.max(np.abs(x - xo) / xo), np.max(np.abs(w - wo) / wo))
    assert worst < 1e-14, worst


def test_rys_rejects_bad_requests():
    from patmol_b200 import gpu
    with pytest.raises(gpu.PatgpuError):
        gpu.rys_host(0, 1.0)
    with pytest.raises(gpu.PatgpuError):
        gpu.rys_host(10, 1.0)


def test_quartet_counts_match_workload_tables():
    c0 = workload.quartet_class_counts(configs.water_spd())
    assert sum(c0.values()) == 879801 and len(c0) == 21
    assert workload.roots_histogram(c0) == {1: 174750, 2: 425412, 3: 240696, 4: 37908, 5: 1035}
    c1 = workload.quartet_class_counts(configs.water_spdf_positron())
    assert sum(c1.values()) == 7328706 and len(c1) == 55
    assert workload.roots_histogram(c1) == {1: 743750, 2: 2518992, 3: 2650478, 4: 1172263, 5: 226525,
                                           6: 16467, 7: 231}


def test_basis_shapes():
    b = configs.water_spdf_positron()
    assert (b.nshell, b.norb, b.ncen) == (87, 292, 4)
    aug = b.dpm_augmented(configs.water_centroid())
    assert aug.nshell == 94 and aug.norb == 292 and aug.skipcen == 4 and aug.charges[-1] == 1.0


def test_patin_roundtrip(tmp_path):
    b = configs.water_spd()
    b.write_patin(str(tmp_path / "patin.dat"))
    c = Basis.read_patin(str(tmp_path / "patin.dat"))
    assert c.norb == b.norb and np.allclose(np.concatenate([s.coef for s in c.shells]),
                                            np.concatenate([s.coef for s in b.shells]), rtol=1e-15)


def test_packing():
    n = 7
    m = np.random.default_rng(0).normal(size=(n, n))
    m = m + m.T
    assert np.allclose(unpack(pack(m), n), m)
    assert packed_index(3, 5) == 5 * 6 // 2 + 3


def test_flop_model_positive_and_monotone():
    f = [workload.flops_per_quartet(c) for c in [(0, 0, 0, 0), (1, 1, 1, 1), (2, 2, 2, 2), (3, 3, 3, 3)]]
    assert all(a < b for a, b in zip(f, f[1:]))
