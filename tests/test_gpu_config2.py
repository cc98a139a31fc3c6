"""Differentiable compliance at the size of the reference's dense-box
sensitivity case: a 128^3 cantilever (E = 1e6, nu = 0.3, p = 3, density seeded
uniform in [0.05, 1], x-min layer fixed, unit load at the x-max face centre),
backward sensitivity against central finite differences (step 1e-4) on 64
seeded cells: relative tolerance 1e-4, with an absolute floor of 1e-9 |C| for
cells whose sensitivity is too small for a finite difference of the compliance
to resolve (the same convention as the 24^3 test)."""
import numpy as np
import pytest

from spgrid_topo_opt_b200 import configs, native

pytestmark = pytest.mark.gpu


def test_compliance_gradient_128_matches_finite_differences(native_lib):
    import torch
    from spgrid_topo_opt_b200.compliance import Compliance

    torch.cuda.set_device(0)
    inp = configs.to_inputs(configs.cantilever_box(128, density=(0.05, 1.0), seed=2018, bottom_size=16))
    m = Compliance(inp, precision=native.PRECISION_FP64, tolerance=1e-15)
    rho0 = torch.tensor(inp.density.data, dtype=torch.float64, requires_grad=True)
    c = m(rho0)
    c.backward()
    grad = rho0.grad.numpy()
    cells = np.argwhere(inp.density.data > 0)
    rng = np.random.default_rng(64)
    h = 1e-4
    worst, strict, worst_abs, worst_rel = 0.0, 0, 0.0, 0.0
    for b, e in cells[rng.choice(len(cells), 64, replace=False)]:
        rp = inp.density.data.copy()
        rm = inp.density.data.copy()
        rp[b, e] += h
        rm[b, e] -= h
        with torch.no_grad():
            fd = (float(m(torch.tensor(rp))) - float(m(torch.tensor(rm)))) / (2 * h)
        worst_abs = max(worst_abs, abs(grad[b, e] - fd) / abs(float(c)))
        worst_rel = max(worst_rel, abs(grad[b, e] - fd) / abs(fd))
        if 1e-4 * abs(fd) >= 1e-9 * abs(float(c)):
            strict += 1
            worst = max(worst, abs(grad[b, e] - fd) / abs(fd))
        assert grad[b, e] == pytest.approx(fd, rel=1e-4, abs=1e-9 * abs(float(c))), (b, e, grad[b, e], fd)
    m.close()
    print(f"{strict} of 64 cells held to the relative bound (largest difference there {worst:.2e}); over all "
          f"64: largest |grad - fd|/|C| {worst_abs:.2e}, largest |grad - fd|/|fd| {worst_rel:.2e}")
