"""Test-only torch.autograd.Function over the SCF energy: forward runs the GPU
SCF at the given centre coordinates, backward returns patgpu_rhf_gradient.
Checked against a central difference (h = 1e-4 bohr) of the forward and by
a steepest-descent step lowering the energy."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
scf = pytest.importorskip("patmol_b200.scf")

from test_gpu_gradient import small_water  # noqa: E402


class SCFEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, template, dpm):
        b = template.with_coords(coords.detach().cpu().numpy())
        res = scf.rhf(b, dpm=dpm)
        if not res.converged:
            raise RuntimeError("SCF did not converge")
        ctx.save_for_backward(torch.from_numpy(scf.rhf_gradient(b, res, dpm=dpm)))
        return torch.tensor(res.energy, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gout):
        (g,) = ctx.saved_tensors
        return gout * g, None, None


def test_autograd_matches_difference_and_descends():
    template = small_water(f_on_o=False).dpm_augmented([0.1, 0.3, 2.8])
    x = torch.tensor(template.coords, dtype=torch.float64, requires_grad=True)
    e = SCFEnergy.apply(x, template, True)
    (g,) = torch.autograd.grad(e, x)
    h = 1e-4
    for c, d in [(0, 2), (3, 2)]:
        xp = x.detach().clone()
        xm = x.detach().clone()
        xp[c, d] += h
        xm[c, d] -= h
        fd = (SCFEnergy.apply(xp, template, True) - SCFEnergy.apply(xm, template, True)).item() / (2 * h)
        assert abs(g[c, d].item() - fd) < 2e-6
    step = 0.02 * g / g.norm()
    e2 = SCFEnergy.apply((x - step).detach(), template, True)
    assert e2.item() < e.item()
    assert np.isfinite(g.numpy()).all()
