"""ElasticForce (torch.autograd.Function): forward = assembled gradient, backward =
the adjoint kernels, checked against the CPU oracle and central finite differences."""
import numpy as np
import pytest

from polyfem_b200 import NeoHookeanAssembler
from polyfem_b200 import mesh as M

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("et", [M.P1_TET, M.P2_TET, M.Q1_HEX], ids=["P1", "P2", "Q1"])
def test_backward_equals_oracle_adjoint_terms(require_gpu, et):
    import torch

    from oracle.binding import Oracle
    from polyfem_b200.autograd import elastic_force

    mesh, lam, mu, u, p = make_case(et, 2, seed=21, jitter=0.1)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    orc = Oracle(mesh, lam, mu)
    t = lambda a, g=True: torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=g)
    ut, lt, mt, Xt = t(u), t(lam), t(mu), t(mesh.X)
    pt = t(p, False)
    f = elastic_force(ut, lt, mt, Xt, asm)
    assert rel_err(f.detach().cpu().numpy(), orc.gradient(u)) <= 1e-12
    (f * pt).sum().backward()
    E = mesh.n_elements
    term = orc.material_vjp(u, p)
    assert rel_err(lt.grad.cpu().numpy(), -term[:E]) <= 1e-12
    assert rel_err(mt.grad.cpu().numpy(), -term[E:]) <= 1e-12
    assert rel_err(Xt.grad.cpu().numpy().ravel(), orc.shape_vjp(u, p)) <= 1e-12
    outer, inner, vals = orc.hessian(u)
    import scipy.sparse as sp
    Hp = sp.csc_matrix((vals, inner, outer), shape=(mesh.n_dofs, mesh.n_dofs)) @ p
    assert rel_err(ut.grad.cpu().numpy(), Hp) <= 1e-12
    asm.close()


def test_backward_matches_central_differences(require_gpu):
    import torch

    from polyfem_b200.autograd import elastic_force

    mesh, lam, mu, u, p = make_case(M.P2_TET, 2, seed=23, jitter=0.1)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    dev = "cuda"
    base = [torch.tensor(a, dtype=torch.float64, device=dev) for a in (u, lam, mu, mesh.X)]
    pt = torch.tensor(p, dtype=torch.float64, device=dev)
    leaves = [b.clone().requires_grad_(True) for b in base]
    (elastic_force(*leaves, asm) * pt).sum().backward()

    def phi(args):
        with torch.no_grad():
            return float((elastic_force(*args, asm) * pt).sum())

    rng = np.random.default_rng(4)
    steps = [1e-6 * mesh.h, 1e-6 * float(np.median(lam)), 1e-6 * float(np.median(mu)), 1e-6 * mesh.h]
    for k in range(4):
        g = leaves[k].grad.cpu().numpy().ravel()
        for idx in rng.choice(g.size, 4, replace=False):
            plus = [b.clone() for b in base]
            minus = [b.clone() for b in base]
            plus[k].view(-1)[idx] += steps[k]
            minus[k].view(-1)[idx] -= steps[k]
            fd = (phi(plus) - phi(minus)) / (2 * steps[k])
            scale = max(abs(fd), 1e-3 * np.abs(g).max())
            assert abs(g[idx] - fd) <= 1e-5 * scale, (k, idx, g[idx], fd)
    asm.close()
