"""Dense assembly (pfg_dense_matrix; DenseMatrixCache) against the oracle's
restatement, which sums every element matrix into a dense array directly."""
import numpy as np
import pytest

from oracle.binding import Oracle, dense_hessian
from polyfem_b200 import NeoHookeanAssembler, PfgError
from polyfem_b200 import mesh as M

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("et,g", [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)], ids=["P1", "P2", "Q1"])
def test_dense_hessian_matches_oracle(require_gpu, et, g):
    import torch
    mesh, lam, mu, u, _ = make_case(et, g, seed=21, jitter=0.1 if et != M.P1_TET else 0.0)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    orc = Oracle(mesh, lam, mu)
    ref = dense_hessian(orc, mesh, u).mat
    D = asm.assemble_hessian_dense(u)
    assert D.shape == (mesh.n_dofs, mesh.n_dofs)
    assert rel_err(D, ref) <= 1e-12
    # every pattern entry placed bit-exact, zeros elsewhere
    outer, inner = asm.hessian_pattern()
    vals = asm.assemble_hessian_values(u)
    cols = np.repeat(np.arange(mesh.n_dofs), np.diff(outer))
    expect = np.zeros_like(D)
    expect[inner, cols] = vals
    assert np.array_equal(D, expect)
    # device mode gives the same array
    Dd = asm.assemble_hessian_dense(torch.tensor(u, device="cuda")).cpu().numpy()
    assert np.array_equal(Dd, D)
    # the sparseView of the dense cache: the pattern minus exact zeros
    sv = dense_hessian(orc, mesh, u).get_matrix()
    assert set(zip(*sv.nonzero())) <= set(zip(inner, cols))
    # the mass matrix through the same entry point
    Md = asm.dense_matrix(asm.assemble_mass_matrix_values())
    assert np.array_equal(Md, asm.assemble_mass_matrix().toarray())
    asm.close()


def test_dense_matrix_size_limit(require_gpu):
    mesh = M.structured_tet_mesh(20, 1)  # 27,783 dofs: 7.7e8 entries > 2^29
    lam, mu = M.homogeneous_lame(mesh.n_elements)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    with pytest.raises(PfgError):
        asm.dense_matrix(np.zeros(asm.hessian_nnz()))
    asm.close()
