"""Isentropic vortex advected by the free stream: the GPU scheme converges at
high order against the exact translated vortex — the rate between 32^2 and
64^2 elements must exceed N + 0.3 (measured on a B200: N = 2: 2.4, N = 3: 4.2,
blending off).

Periodic [-5, 5]^2, free stream rho = u = v = p = 1, strength 5, t = 1.
Errors: L2 (quadrature) of density; the periodic copy's mismatch at the box
edge (e^-12) is far below the errors measured."""
import numpy as np
import pytest

import prandtl_b200 as pb
from prandtl_b200 import adjoint, cases

pytestmark = pytest.mark.gpu


class Shifted:
    """A mesh whose node coordinates are moved back by (t, t), wrapped into the box."""

    def __init__(self, mesh, t):
        self.mesh, self.t = mesh, t

    def node_coords(self):
        x, y = self.mesh.node_coords()
        return (((x - self.t) + 5.0) % 10.0) - 5.0, (((y - self.t) + 5.0) % 10.0) - 5.0


def density_error(n, order, t_end, blending, cuda_device):
    import torch
    m = cases.vortex_mesh(n, order)
    u0 = cases.isentropic_vortex(m)
    op = pb.DGSEMOperator(m, blending=blending)
    x = torch.from_numpy(u0).to(cuda_device)
    tmp = torch.empty_like(x)
    op.Mult(x, tmp)
    dt = op.cfl_dt(0.1)
    steps = int(np.ceil(t_end / dt))
    dt = t_end / steps
    for _ in range(steps):
        op.rk3_step(x, dt)
    exact = cases.isentropic_vortex(Shifted(m, t_end))
    nn = m.num_nodes
    w = adjoint.node_weights(m)
    err = x.cpu().numpy()[:nn] - exact[:nn]
    assert op.check() == 0
    return float(np.sqrt(np.sum(w * err * err)))


@pytest.mark.parametrize("order", [2, 3])
def test_vortex_converges_at_high_order(order, cuda_device):
    errs = [density_error(n, order, 1.0, 0, cuda_device) for n in (16, 32, 64)]
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    print("order", order, "errors", errs, "rates", rates)
    assert errs[-1] < errs[0]
    assert rates[-1] > order + 0.3, (errs, rates)
