"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the GPU product never does.  The oracle restates the reference's
CPU algorithm (see oracle/pf_oracle.cpp for the file:line map).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "pf_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _i, ctypes.c_int, _i, _d, _d, _d,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_project_psd.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_material.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_material_params.argtypes = [ctypes.c_void_p, _d, ctypes.c_int]
        L.orc_set_elasticity_tensor.argtypes = [ctypes.c_void_p, _d]
        L.orc_basis_value.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_basis_value.restype = ctypes.c_double
        L.orc_mass.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_mass.restype = ctypes.c_longlong
        L.orc_mass_copy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_project_psd.argtypes = [_d, ctypes.c_int]
        L.orc_energy.restype = ctypes.c_double
        L.orc_energy.argtypes = [ctypes.c_void_p, _d]
        L.orc_energy_per_element.argtypes = [ctypes.c_void_p, _d, _d]
        L.orc_gradient.argtypes = [ctypes.c_void_p, _d, _d]
        L.orc_hessian.restype = ctypes.c_longlong
        L.orc_hessian.argtypes = [ctypes.c_void_p, _d]
        L.orc_hessian_copy.argtypes = [ctypes.c_void_p, _i, _i, _d]
        L.orc_slot.restype = ctypes.c_int
        L.orc_slot.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_material_vjp.argtypes = [ctypes.c_void_p, _d, _d, _d]
        L.orc_shape_vjp.argtypes = [ctypes.c_void_p, _d, _d, _d]
        L.orc_element.restype = ctypes.c_int
        L.orc_element.argtypes = [ctypes.c_void_p, ctypes.c_int, _d, _d, _d, _d]
        L.orc_tables.restype = ctypes.c_int
        L.orc_tables.argtypes = [ctypes.c_int, _d, _d, _d, _d]
        L.orc_smc_new.restype = ctypes.c_void_p
        L.orc_smc_new.argtypes = [ctypes.c_int]
        L.orc_smc_copy.restype = ctypes.c_void_p
        L.orc_smc_copy.argtypes = [ctypes.c_void_p]
        L.orc_smc_add.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_smc_prune.argtypes = [ctypes.c_void_p]
        L.orc_smc_get_matrix.restype = ctypes.c_longlong
        L.orc_smc_get_matrix.argtypes = [ctypes.c_void_p]
        L.orc_smc_coeff.restype = ctypes.c_double
        L.orc_smc_coeff.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_smc_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_d)


def _ip(a):
    return a.ctypes.data_as(_i)


class Oracle:
    """CPU restatement of NLAssembler + ElasticForm + ElasticForceDerivative."""

    MATERIALS = {"NeoHookean": 0, "IsochoricNeoHookean": 1, "SaintVenant": 2, "LinearElasticity": 3,
                 "MooneyRivlin": 4, "MooneyRivlin3Param": 5, "VolumePenalty": 6, "HookeLinearElasticity": 7,
                 "SaintVenantTensor": 8, "UnconstrainedOgden": 9, "IncompressibleOgden": 10,
                 "MooneyRivlin3ParamSymbolic": 11}
    # lists of one value per term (alphas, mus, Ds; c, m), then IncompressibleOgden's k
    OGDEN_PARAMS = {"UnconstrainedOgden": ("alphas", "mus", "Ds"), "IncompressibleOgden": ("c", "m", "k")}
    MATERIAL_PARAMS = {"MooneyRivlin": ("c1", "c2", "k"), "MooneyRivlin3Param": ("c1", "c2", "c3", "d1"),
                       "VolumePenalty": ("k",), "MooneyRivlin3ParamSymbolic": ("c1", "c2", "c3", "d1")}

    def __init__(self, mesh, lam, mu, n_threads: int = 1, cache_size: int = 900000,
                 fast_pattern: bool = False, material: str = "NeoHookean", params=None):
        """params: the GenericMatParam values of a parameterised material, a dict of
        name -> scalar or per-element array (MATERIAL_PARAMS names)."""
        L = lib()
        self.mesh = mesh
        self._conn = np.ascontiguousarray(mesh.conn, dtype=np.int32)
        self._gconn = np.ascontiguousarray(mesh.gconn, dtype=np.int32)
        self._X = np.ascontiguousarray(mesh.X, dtype=np.float64)
        self._lam = np.ascontiguousarray(lam, dtype=np.float64)
        self._mu = np.ascontiguousarray(mu, dtype=np.float64)
        self.h = L.orc_create(mesh.elem_type, mesh.n_elements, mesh.n_nodes, _ip(self._conn),
                              mesh.n_geom_nodes, _ip(self._gconn), _dp(self._X), _dp(self._lam),
                              _dp(self._mu), int(n_threads), int(cache_size), int(fast_pattern))
        if not self.h:
            raise RuntimeError("oracle creation failed")
        self.n_dofs = mesh.n_dofs
        if material in ("HookeLinearElasticity", "SaintVenantTensor"):
            if set(params or {}) != {"elasticity_tensor"}:
                raise ValueError(f"{material} takes the parameter elasticity_tensor (21 entries)")
            self._hooke = np.ascontiguousarray(np.asarray(params["elasticity_tensor"], dtype=np.float64).ravel())
            if self._hooke.size != 21:
                raise ValueError("the elasticity tensor takes 21 entries")
            L.orc_set_elasticity_tensor(self.h, _dp(self._hooke))
            params = None
        if material in self.OGDEN_PARAMS:
            keys = self.OGDEN_PARAMS[material]
            if set(params or {}) != set(keys):
                raise ValueError(f"{material} takes the parameters {list(keys)}")
            flat = [v for k in keys for v in (params[k] if isinstance(params[k], (list, tuple)) else [params[k]])]
            params = {f"p{i}": v for i, v in enumerate(flat)}
            names = tuple(params)
        else:
            names = self.MATERIAL_PARAMS.get(material, ())
        if set(params or {}) != set(names):
            raise ValueError(f"{material} takes the parameters {list(names)}")
        if names:
            E = mesh.n_elements
            self._mparams = np.ascontiguousarray(
                np.stack([np.broadcast_to(np.asarray(params[n], dtype=np.float64), (E,)) for n in names]))
            L.orc_set_material_params(self.h, _dp(self._mparams), len(names))
        L.orc_set_material(self.h, self.MATERIALS[material])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def mass_matrix(self, rho=None):
        """MassMatrixAssembler's CSC (outer, inner, values); rho per element or None for 1."""
        r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
        nnz = lib().orc_mass(self.h, None if r is None else ctypes.c_void_p(r.ctypes.data))
        outer = np.empty(self.n_dofs + 1, dtype=np.int32)
        inner = np.empty(nnz, dtype=np.int32)
        vals = np.empty(nnz)
        lib().orc_mass_copy(self.h, ctypes.c_void_p(outer.ctypes.data), ctypes.c_void_p(inner.ctypes.data),
                            ctypes.c_void_p(vals.ctypes.data))
        return outer, inner, vals

    def set_threads(self, n: int):
        lib().orc_set_threads(self.h, int(n))

    def energy(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        return lib().orc_energy(self.h, _dp(u))

    def energy_per_element(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty(self.mesh.n_elements)
        lib().orc_energy_per_element(self.h, _dp(u), _dp(out))
        return out

    def gradient(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        g = np.empty(self.n_dofs)
        lib().orc_gradient(self.h, _dp(u), _dp(g))
        return g

    def hessian(self, u, project_psd: bool = False):
        """Returns (outer, inner, values) of the CSC Hessian; with project_psd every
        element matrix is projected onto the PSD cone before the scatter
        (Assembler.cpp:693-694)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        lib().orc_set_project_psd(self.h, int(bool(project_psd)))
        nnz = lib().orc_hessian(self.h, _dp(u))
        if nnz < 0:
            raise RuntimeError("oracle hessian failed")
        outer = np.empty(self.n_dofs + 1, dtype=np.int32)
        inner = np.empty(nnz, dtype=np.int32)
        vals = np.empty(nnz)
        lib().orc_hessian_copy(self.h, _ip(outer), _ip(inner), _dp(vals))
        return outer, inner, vals

    def slot(self, e: int, k: int) -> int:
        return lib().orc_slot(self.h, int(e), int(k))

    def material_vjp(self, u, p):
        u = np.ascontiguousarray(u, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        out = np.empty(2 * self.mesh.n_elements)
        lib().orc_material_vjp(self.h, _dp(u), _dp(p), _dp(out))
        return out

    def shape_vjp(self, u, p):
        u = np.ascontiguousarray(u, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        out = np.empty(3 * self.mesh.n_geom_nodes)
        lib().orc_shape_vjp(self.h, _dp(u), _dp(p), _dp(out))
        return out

    def element(self, e: int, u):
        n = self.mesh.conn.shape[1]
        u = np.ascontiguousarray(u, dtype=np.float64)
        en = np.zeros(1)
        g = np.zeros(3 * n)
        H = np.zeros((3 * n, 3 * n))
        lib().orc_element(self.h, int(e), _dp(u), _dp(en), _dp(g), _dp(H))
        return en[0], g, H


def project_psd(H):
    """ipc::project_to_psd (CLAMP) of one symmetric matrix, restated in the oracle."""
    A = np.array(H, dtype=np.float64, order="C", copy=True)
    lib().orc_project_psd(_dp(A), A.shape[0])
    return A


def tables(elem_type: int):
    n = {1: 4, 2: 10, 3: 8}[elem_type]
    ng = {1: 4, 2: 4, 3: 8}[elem_type]
    qp = np.zeros((8, 3))
    qw = np.zeros(8)
    gr = np.zeros((8, n, 3))
    gg = np.zeros((8, ng, 3))
    nq = lib().orc_tables(elem_type, _dp(qp), _dp(qw), _dp(gr), _dp(gg))
    return qp[:nq], qw[:nq], gr[:nq], gg[:nq]


class SparseMatrixCache:
    """Bare restated SparseMatrixCache, for the reference's 'cache' known-answer test."""

    def __init__(self, size: int = 0, other: "SparseMatrixCache | None" = None):
        L = lib()
        self.h = L.orc_smc_copy(other.h) if other is not None else L.orc_smc_new(int(size))

    def add_value(self, e, i, j, v):
        lib().orc_smc_add(self.h, int(e), int(i), int(j), float(v))

    def prune(self):
        lib().orc_smc_prune(self.h)

    def get_matrix(self):
        return lib().orc_smc_get_matrix(self.h)

    def coeff(self, i, j):
        return lib().orc_smc_coeff(self.h, int(i), int(j))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_smc_free(self.h)
            self.h = None


class DenseMatrixCache:
    """DenseMatrixCache restated (utils/MatrixCache.cpp:326-403): add_value sums into a
    dense matrix (MatrixCache.cpp:371-374); get_matrix is its sparseView(), which keeps
    the nonzero entries only (MatrixCache.cpp:378-381)."""

    def __init__(self, rows: int, cols: int | None = None):
        self.mat = np.zeros((rows, rows if cols is None else cols))

    def add_value(self, e, i, j, v):
        self.mat[i, j] += v

    def get_matrix(self):
        import scipy.sparse as sp
        return sp.csc_matrix(self.mat)  # stores the nonzeros only, like Eigen's sparseView()


def dense_hessian(orc, mesh, u):
    """The global Hessian through DenseMatrixCache: every element matrix of the oracle
    added entry by entry at its global dofs, elements in order (the serial order of
    Assembler.cpp:306-316's merge of one thread's cache)."""
    n = mesh.conn.shape[1]
    cache = DenseMatrixCache(mesh.n_dofs)
    for e in range(mesh.n_elements):
        H = orc.element(e, u)[2]
        dofs = (3 * mesh.conn[e][:, None] + np.arange(3)[None, :]).ravel()
        cache.mat[np.ix_(dofs, dofs)] += H
    return cache


def composite_reference(mesh, components, element_component, u, project=False):
    """MaterialSum (SumModel.cpp:43-78) and MultiModels (MultiModel.cpp:35-58) restated
    from the oracle's element quantities: per element the sum over the components (or
    only the element's own component) of energy, gradient and Hessian, the Hessian
    projected after the sum (NLAssembler projects the element matrix the composition
    returns), then assembled.  components: (oracle material name, lam, mu, params) per
    component.  Returns (per-element energies, gradient, dense Hessian)."""
    orcs = [Oracle(mesh, lam, mu, material=mat, params=prm) for mat, lam, mu, prm in components]
    n = mesh.conn.shape[1]
    E = mesh.n_elements
    per = np.zeros(E)
    g = np.zeros(mesh.n_dofs)
    H = np.zeros((mesh.n_dofs, mesh.n_dofs))
    for e in range(E):
        ks = range(len(orcs)) if element_component is None else [int(element_component[e])]
        en, ge, He = 0.0, np.zeros(3 * n), np.zeros((3 * n, 3 * n))
        for k in ks:
            a, b, c = orcs[k].element(e, u)
            en, ge, He = en + a, ge + b, He + c
        if project:
            He = project_psd(He)
        dofs = (3 * mesh.conn[e][:, None] + np.arange(3)[None, :]).ravel()
        per[e] = en
        g[dofs] += ge
        H[np.ix_(dofs, dofs)] += He
    return per, g, H


def free_dofs(ndof: int, constrained):
    """not_constraints_ / old_to_new_ of BCLagrangianForm (BCLagrangianForm.cpp:122-137)."""
    is_c = np.zeros(ndof, dtype=bool)
    is_c[np.asarray(constrained, dtype=np.int64)] = True
    free = np.flatnonzero(~is_c).astype(np.int64)
    old_to_new = np.full(ndof, -1, dtype=np.int64)
    old_to_new[free] = np.arange(free.size)
    return free, old_to_new


def project_hessian(outer, inner, values, constrained):
    """BCLagrangianForm::project_hessian (BCLagrangianForm.cpp:165-212), restated:
    drop the constrained rows and columns of a ColMajor CSC matrix in one scan,
    renumbering the free dofs in ascending order.  Returns (outer, inner, values)."""
    ndof = len(outer) - 1
    free, old_to_new = free_dofs(ndof, constrained)
    r_outer = [0]
    r_inner, r_vals = [], []
    for k in free:
        rows = inner[outer[k]:outer[k + 1]]
        keep = old_to_new[rows] >= 0
        r_inner.append(old_to_new[rows[keep]])
        r_vals.append(values[outer[k]:outer[k + 1]][keep])
        r_outer.append(r_outer[-1] + int(keep.sum()))
    cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dtype=dt)
    return np.asarray(r_outer, dtype=np.int32), cat(r_inner, np.int32), cat(r_vals, np.float64)


def project_gradient(grad, constrained):
    """BCLagrangianForm::project_gradient (BCLagrangianForm.cpp:149-155)."""
    free, _ = free_dofs(len(grad), constrained)
    return np.asarray(grad)[free]


def reduced_to_full(y, x_bc, constrained):
    """NLProblem::reduced_to_full for the projecting Dirichlet form (NLProblem.cpp:713-735):
    free dofs from y, constrained dofs from the boundary values."""
    x = np.array(x_bc, dtype=np.float64, copy=True)
    free, _ = free_dofs(len(x), constrained)
    x[free] = y
    return x


def lump_matrix(outer, inner, values):
    """polyfem::utils::lump_matrix (utils/MatrixUtils.cpp:84-101), restated: every
    stored (row, value) of the ColMajor CSC matrix, column by column, becomes the
    triplet (row, row, value), and Eigen's setFromTriplets sums the duplicates of
    one (row, row) in insertion order starting from the first value (ascending
    column).  Returns the diagonal (0 where a row has no entry)."""
    outer = np.asarray(outer, dtype=np.int64)
    inner = np.asarray(inner, dtype=np.int64)
    values = np.asarray(values, dtype=np.float64)
    n = len(outer) - 1
    diag = np.zeros(n, dtype=np.float64)
    seen = np.zeros(n, dtype=bool)
    for k in range(n):
        rows = inner[outer[k]:outer[k + 1]]  # unique within a column
        v = values[outer[k]:outer[k + 1]]
        diag[rows] = np.where(seen[rows], diag[rows] + v, v)
        seen[rows] = True
    return diag


def conjugate_gradient(outer, inner, values, b, tol, max_iter, x0=None):
    """Eigen 3.4's ConjugateGradient<SparseMatrix, Lower|Upper, DiagonalPreconditioner>
    (the "Eigen::ConjugateGradient" choice of polysolve's linear::Solver, which
    the Newton step of polysolve@47dc48d (external) applies to the Hessian NLProblem::hessian returns, solver/NLProblem.cpp:615-621),
    restated on a ColMajor CSC matrix.  Eigen is a dependency absent from the
    reference tree (cmake/recipes/eigen.cmake pins 3.4.0); its published iteration:
    r = b - A x, stop when |r|^2 < max(tol^2 |b|^2, smallest normal double),
    p = D^-1 r, then per iteration q = A p, alpha = r.z / p.q, x += alpha p,
    r -= alpha q, check, z = D^-1 r, beta = r.z' / r.z, p = z + beta p.
    D^-1 = 1 / diag(A) where the diagonal entry is non-zero, else 1.
    Returns (x, iterations, relative residual) as Eigen's solve / iterations() /
    error() report them."""
    import scipy.sparse as sp

    n = len(outer) - 1
    A = sp.csc_matrix((np.asarray(values, dtype=np.float64), inner, outer), shape=(n, n))
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    d = A.diagonal()
    invd = np.where(d != 0.0, 1.0 / np.where(d != 0.0, d, 1.0), 1.0)
    rhs2 = float(b @ b)
    if rhs2 == 0.0:
        return np.zeros(n), 0, 0.0
    r = b - A @ x
    thr = max(tol * tol * rhs2, np.finfo(np.float64).tiny)
    rr = float(r @ r)
    if rr < thr:
        return x, 0, float(np.sqrt(rr / rhs2))
    p = invd * r
    rz = float(r @ p)
    i = 0
    while i < max_iter:
        q = A @ p
        alpha = rz / float(p @ q)
        x += alpha * p
        r -= alpha * q
        rr = float(r @ r)
        if rr < thr:
            break
        z = invd * r
        rz_new = float(r @ z)
        p = z + (rz_new / rz) * p
        rz = rz_new
        i += 1
    return x, i, float(np.sqrt(rr / rhs2))
