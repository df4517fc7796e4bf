"""The tensor-core element Hessians of the split mode (tcgen05, TF32 pairs, FP32
accumulation in TMEM) against the FP64 oracle.

For P2 and Q1, PFG_SPLIT32 computes every element block as one GEMM row block
D[(e, r, c), (a, b)] = W_e[(r, c), :] . Phi[(a, b), :], with Phi the products of
the reference-element gradients (one table per element type).  These cases cover
partial last tiles (element counts that are not multiples of the 14-element
tile), CTAs that loop over many tiles, non-affine (jittered) hexahedra, both
CTA roles' hand-off of the two kinematics buffers, NaN propagation from an
inverted element, and agreement with the CUDA-core variant of the same split.
Bound: <= 1e-6 relative Frobenius error against the FP64 oracle.
"""
import numpy as np
import pytest

from oracle.binding import Oracle
from polyfem_b200 import NeoHookeanAssembler
from polyfem_b200 import mesh as M

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("et,g,jit", [(M.P2_TET, 1, 0.0), (M.P2_TET, 3, 0.1), (M.P2_TET, 5, 0.0),
                                      (M.Q1_HEX, 3, 0.1), (M.Q1_HEX, 7, 0.1)],
                         ids=["P2-1", "P2-3j", "P2-5", "Q1-3j", "Q1-7j"])
def test_tensor_core_blocks_against_oracle(require_gpu, et, g, jit):
    mesh, lam, mu, u, _ = make_case(et, g, seed=51, jitter=jit)
    assert mesh.n_elements % 14 != 0 or g == 7  # partial last tile in most cases
    orc = Oracle(mesh, lam, mu, n_threads=4, fast_pattern=True)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    _, _, v = orc.hessian(u)
    h = asm.assemble_hessian_values(u, "split32")
    assert rel_err(h, v) <= 1e-6
    # the CUDA-core split agrees with the tensor-core one to the same order
    assert rel_err(asm.assemble_hessian_values(u, "split32_simt"), h) <= 1e-6
    asm.close()


@pytest.mark.parametrize("et,g", [(M.P2_TET, 16), (M.Q1_HEX, 24)], ids=["P2-16", "Q1-24"])
def test_tensor_core_many_tiles_per_cta(require_gpu, et, g):
    """24,576 P2 / 13,824 Q1 elements: more tiles than resident CTAs, so every CTA
    runs its tile loop (and the kinematics double buffer) several times."""
    mesh, lam, mu, u, _ = make_case(et, g, seed=52, jitter=0.1)
    orc = Oracle(mesh, lam, mu, n_threads=8, fast_pattern=True)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    _, _, v = orc.hessian(u)
    h = asm.assemble_hessian_values(u, "split32")
    assert rel_err(h, v) <= 1e-6
    assert np.array_equal(h, asm.assemble_hessian_values(u, "split32"))  # deterministic
    asm.close()


@pytest.mark.parametrize("et", [M.P2_TET, M.Q1_HEX])
def test_tensor_core_inverted_element_gives_nan(require_gpu, et):
    """ln J of an inverted element is NaN in the reference; the NaN reaches exactly
    the CSC entries of that element's node blocks and no others."""
    mesh, lam, mu, u, _ = make_case(et, 3, seed=53)
    orc = Oracle(mesh, lam, mu, fast_pattern=True)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    u = u.copy()
    nodes = mesh.conn[17]
    u.reshape(-1, 3)[nodes] = -3.0 * mesh.node_pos[nodes]  # turns element 17 inside out
    _, _, v = orc.hessian(u)
    assert np.isnan(v).any()
    for prec in ("fp64", "split32", "split32_simt"):
        h = asm.assemble_hessian_values(u, prec)
        assert np.array_equal(np.isnan(h), np.isnan(v)), prec
    ok = ~np.isnan(v)
    assert ok.any() and rel_err(asm.assemble_hessian_values(u, "split32")[ok], v[ok]) <= 1e-6
    asm.close()
