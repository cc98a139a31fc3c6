"""Differentiable compliance (torch.autograd.Function over the GPU solve).

The backward is the hand-written sensitivity kernel; it is checked against
central finite differences of the compliance (step 1e-4, relative tolerance
1e-4) on seeded random cells, and against the
oracle's restatement of the reference's sensitivity (minimal_compliance.cpp:86-146).
"""
import numpy as np
import pytest

from oracle import oracle as orc
from spgrid_topo_opt_b200 import configs, native

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def model(native_lib):
    import torch
    from spgrid_topo_opt_b200.compliance import Compliance

    torch.cuda.set_device(0)
    prob = configs.cantilever_box(24, density=(0.05, 1.0), bottom_size=6)
    inp = configs.to_inputs(prob)
    m = Compliance(inp, precision=native.PRECISION_FP64, tolerance=1e-14)
    yield inp, m
    m.close()


def test_gradient_matches_finite_differences(model):
    import torch

    inp, m = model
    rho0 = torch.tensor(inp.density.data, dtype=torch.float64, requires_grad=True)
    c = m(rho0)
    c.backward()
    grad = rho0.grad.numpy()
    rng = np.random.default_rng(2018)
    cells = np.argwhere(inp.density.data > 0)
    h = 1e-4
    for b, e in cells[rng.choice(len(cells), 12, replace=False)]:
        rp = inp.density.data.copy()
        rm = inp.density.data.copy()
        rp[b, e] += h
        rm[b, e] -= h
        with torch.no_grad():
            cp = float(m(torch.tensor(rp)))
            cm = float(m(torch.tensor(rm)))
        fd = (cp - cm) / (2 * h)
        assert grad[b, e] == pytest.approx(fd, rel=1e-4, abs=1e-9 * abs(float(c))), (b, e)
    assert np.all(grad[inp.density.data <= 0] == 0)
    # more material, less compliance; cells of the fixed layer have u = 0 and zero gradient
    assert np.all(grad[inp.density.data > 0] <= 0)
    assert np.mean(grad[inp.density.data > 0] < 0) > 0.9


def test_gradient_matches_oracle_sensitivity(model):
    import torch

    inp, m = model
    rho = torch.tensor(inp.density.data, dtype=torch.float64, requires_grad=True)
    m(rho).backward()
    o = orc.Oracle(inp, mode=orc.MODE_FP64, tolerance=1e-12)
    o.solve()
    _, dc, _ = o.sensitivity()
    ref = -inp.dx * dc
    assert np.abs(rho.grad.numpy() - ref).max() <= 1e-7 * np.abs(ref).max()


def test_set_density_keeps_material_pattern(model):
    inp, m = model
    bad = inp.density.data.copy()
    bad[bad > 0][:1] = 0
    idx = np.argwhere(inp.density.data > 0)[0]
    bad[idx[0], idx[1]] = 0.0
    with pytest.raises(native.SolverError):
        m.session.set_density(bad)
    m.session.set_density(inp.density.data)


def test_forward_and_backward_stay_on_the_device(model):
    """With the densities on the GPU, neither pass copies a field to the host:
    the library's device-to-host byte count grows only by the solver's
    per-iteration convergence scalars, far below one copy of u."""
    import torch

    inp, m = model
    rho_host = torch.tensor(inp.density.data, dtype=torch.float64, requires_grad=True)
    m(rho_host).backward()
    rho = torch.tensor(inp.density.data, dtype=torch.float64, device="cuda", requires_grad=True)
    with torch.no_grad():
        m(rho)
    before = m.last_stats["d2h_bytes"]
    c = m(rho)
    c.backward()
    with torch.no_grad():
        m(rho)  # its solve reports the bytes moved since the previous one, backward included
    moved = m.last_stats["d2h_bytes"] - before
    field_bytes = 8 * m.session.solution_size()
    assert moved < field_bytes / 20, (moved, field_bytes)
    assert rho.grad.is_cuda and rho.grad.shape == rho.shape
    assert torch.allclose(rho.grad.cpu(), rho_host.grad, rtol=1e-10, atol=0)
