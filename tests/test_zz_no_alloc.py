"""The allocation-free Fock build (patgpu_rhf_gmatrix_device_noalloc).

Some callers cannot allocate GPU memory while they run: a host program that
hands out all device memory from its own pool, or a loop where a cudaMalloc
would stall the device. For them the library keeps the build's two working
matrices in a fixed array compiled into the library. This file checks,
through the C ABI, that two calls in a row give the same G as the
allocating entry point patgpu_rhf_gmatrix_device, and that bases beyond the
array's 512-function limit are refused. The file is named to run last, so a
run that stops at its first failure has already run every other test.
"""
import numpy as np
import pytest

from patmol_b200 import configs
from patmol_b200.basis import Basis

from golden.make_golden import seeded_density  # noqa: E402

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")


def _device_build(G, fn, P_np):
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    dP = torch.from_numpy(np.ascontiguousarray(P_np)).to(dev)
    dG = torch.full((G.no2,), float("nan"), dtype=torch.float64, device=dev)
    fn(dP.data_ptr(), dG.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize(dev)
    return dG.cpu().numpy()


def test_noalloc_matches_allocating_build_two_calls():
    b = configs.water_spd()
    G = gpu.GpuBasis(b)
    P1, P2 = seeded_density(b.norb, 31), seeded_density(b.norb, 32)
    # two calls in a row through the allocation-free entry point: the second
    # must not see the first call's sums, which stay in the shared scratch
    n1 = _device_build(G, G.rhf_gmatrix_device_noalloc, P1)
    n2 = _device_build(G, G.rhf_gmatrix_device_noalloc, P2)
    r1 = _device_build(G, G.rhf_gmatrix_device, P1)
    r2 = _device_build(G, G.rhf_gmatrix_device, P2)
    assert np.all(np.isfinite(n1)) and np.all(np.isfinite(n2))
    assert np.abs(n1 - r1).max() < 1e-11
    assert np.abs(n2 - r2).max() < 1e-11
    assert np.abs(n1 - n2).max() > 1e-3          # the densities differ, so must G


def test_noalloc_matches_allocating_build_mixed_precision():
    """With the mixed-precision window on, the class launches take their
    two-window and one-launch forms; the allocation-free build must follow
    them exactly like the allocating one."""
    b = configs.water_spd()
    G = gpu.GpuBasis(b)
    assert G.set_mixed_precision(1e-8) >= 0
    P = seeded_density(b.norb, 33)
    n1 = _device_build(G, G.rhf_gmatrix_device_noalloc, P)
    r1 = _device_build(G, G.rhf_gmatrix_device, P)
    n2 = _device_build(G, G.rhf_gmatrix_device_noalloc, P)
    assert np.all(np.isfinite(n1))
    assert np.abs(n1 - r1).max() < 1e-11
    assert n1.tobytes() == n2.tobytes()


def test_noalloc_rejects_bases_beyond_its_scratch():
    # 52 f shells = 520 functions, above the 512 the fixed scratch holds
    specs = [(3, k % 2, [0.3 * 1.5 ** (k // 2)], [1.0]) for k in range(52)]
    b = Basis.from_shell_list([1.0, 1.0], [[0, 0, 0], [0, 0, 2.0]], specs, nelec=2, mult=1)
    assert b.norb == 520
    G = gpu.GpuBasis(b)
    with pytest.raises(gpu.PatgpuError) as e:
        _device_build(G, G.rhf_gmatrix_device_noalloc, np.zeros(G.no2))
    assert "at most 512" in str(e.value)
