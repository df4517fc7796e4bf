"""Host-side mirror of PolyFEM's NeoHookean assembly interface, backed by libpfgpu.

``NeoHookeanAssembler`` plays the part of ``NLAssembler`` + ``NeoHookeanElasticity``
(assembler/Assembler.hpp:238-299) together with the ``AssemblyValsCache`` and the
``SparseMatrixCache`` that ``ElasticForm`` owns.  ``ElasticForm`` mirrors
solver/forms/ElasticForm.cpp and solver/forms/Form.hpp (value, first_derivative,
second_derivative with weight()/scale), and ``ElasticForceDerivative`` mirrors
optimization/force_derivatives/ElasticForceDerivative.cpp.

Vectors may be numpy arrays (host memory: the call copies to the device and back)
or CUDA float64 torch tensors (device memory: the call enqueues on torch's current
stream and returns device tensors).  Every computation runs in libpfgpu's CUDA
kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PFG_FP32, PFG_FP64, PFG_MEM_DEVICE, PFG_MEM_HOST, PFG_SPLIT32, PFG_SPLIT32_SIMT, check, lib

PRECISIONS = {"fp64": PFG_FP64, "fp32": PFG_FP32, "split32": PFG_SPLIT32, "split32_simt": PFG_SPLIT32_SIMT}


def _prec(p) -> int:
    if isinstance(p, str):
        if p not in PRECISIONS:
            raise ValueError(f"unknown precision {p!r}; expected one of {sorted(PRECISIONS)}")
        return PRECISIONS[p]
    return int(p)


def _is_device(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


class NeoHookeanAssembler:
    """NeoHookean energy / gradient / Hessian / adjoint terms on one GPU.

    Parameters mirror what NLAssembler reads from ElementBases and LameParameters:
    ``conn`` (E x n FE node ids), ``gconn`` (E x n_g geometric node ids, or None
    when isoparametric), ``X`` (N_g x 3 rest positions), per-element ``lam``/``mu``.
    """

    def __init__(self, elem_type: int, conn, X, lam, mu, n_nodes: int | None = None,
                 gconn=None, device: int = 0):
        L = lib()
        self.elem_type = int(elem_type)
        self._conn = np.ascontiguousarray(conn, dtype=np.int32)
        self._gconn = None if gconn is None else np.ascontiguousarray(gconn, dtype=np.int32)
        self._X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
        self.n_elements = int(self._conn.shape[0])
        self.n_nodes = int(n_nodes if n_nodes is not None else (self._conn.max() + 1 if self._conn.size else 0))
        self.n_geom_nodes = int(self._X.shape[0])
        self.n_dofs = 3 * self.n_nodes
        self.material = "NeoHookean"
        lam = np.ascontiguousarray(np.broadcast_to(np.asarray(lam, dtype=np.float64), (self.n_elements,)))
        mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu, dtype=np.float64), (self.n_elements,)))
        self.device = int(device)
        desc = _lib.MeshDesc(
            self.elem_type, self.n_elements, self.n_nodes, self.n_geom_nodes,
            self._conn.ctypes.data, None if self._gconn is None else self._gconn.ctypes.data,
            self._X.ctypes.data, lam.ctypes.data, mu.ctypes.data, self.device)
        h = ctypes.c_void_p()
        st = L.pfg_create(ctypes.byref(desc), ctypes.byref(h))
        check(st, None, "pfg_create")
        self._h = h
        self._nnz = None

    @classmethod
    def from_mesh(cls, mesh, lam, mu, device: int = 0):
        gconn = None if mesh.gconn is mesh.conn else mesh.gconn
        return cls(mesh.elem_type, mesh.conn, mesh.X, lam, mu, n_nodes=mesh.n_nodes, gconn=gconn, device=device)

    # -- lifecycle -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().pfg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- helpers -------------------------------------------------------------
    def _prepare(self, *xs):
        dev = [_is_device(x) for x in xs if x is not None]
        if any(dev) and not all(dev):
            raise ValueError("mix of host and device arrays")
        if dev and dev[0]:
            import torch
            for x in xs:
                if x is not None and (x.dtype != torch.float64 or not x.is_contiguous()):
                    raise ValueError("device inputs must be contiguous float64 CUDA tensors")
            check(lib().pfg_set_stream(self._h, ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)),
                  self._h, "pfg_set_stream")
            return PFG_MEM_DEVICE, [x if x is None else ctypes.c_void_p(x.data_ptr()) for x in xs], xs
        check(lib().pfg_set_stream(self._h, None), self._h, "pfg_set_stream")
        arrs = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in xs]
        return PFG_MEM_HOST, [None if a is None else ctypes.c_void_p(a.ctypes.data) for a in arrs], arrs

    def _alloc(self, mem, n):
        if mem == PFG_MEM_DEVICE:
            import torch
            t = torch.empty(n, dtype=torch.float64, device=f"cuda:{self.device}")
            return t, ctypes.c_void_p(t.data_ptr())
        a = np.empty(n, dtype=np.float64)
        return a, ctypes.c_void_p(a.ctypes.data)

    def _check_len(self, x, n, name):
        if x is not None and int(x.numel() if hasattr(x, "numel") else np.size(x)) != n:
            raise ValueError(f"{name} must have {n} entries")

    # -- material / geometry updates -------------------------------------------
    def set_lame(self, lam, mu):
        """LameParameters per-element override (lambda_mat_/mu_mat_)."""
        mem, ptrs, keep = self._prepare(lam, mu)
        self._check_len(lam, self.n_elements, "lambda")
        self._check_len(mu, self.n_elements, "mu")
        check(lib().pfg_set_lame(self._h, ptrs[0], ptrs[1], mem), self._h, "pfg_set_lame")

    def set_rest_positions(self, X):
        mem, ptrs, keep = self._prepare(X)
        self._check_len(X, 3 * self.n_geom_nodes, "X")
        check(lib().pfg_set_rest_positions(self._h, ptrs[0], mem), self._h, "pfg_set_rest_positions")

    # -- NLAssembler interface ---------------------------------------------------
    def assemble_energy(self, u, precision="fp64"):
        """NLAssembler::assemble_energy (assembler/Assembler.cpp:495-531)."""
        self._check_len(u, self.n_dofs, "u")
        mem, ptrs, keep = self._prepare(u)
        out, optr = self._alloc(mem, 1)
        check(lib().pfg_energy(self._h, ptrs[0], mem, _prec(precision), optr), self._h, "pfg_energy")
        return float(out[0]) if mem == PFG_MEM_HOST else out[0]

    def assemble_energy_per_element(self, u, precision="fp64"):
        """NLAssembler::assemble_energy_per_element (assembler/Assembler.cpp:533-572)."""
        self._check_len(u, self.n_dofs, "u")
        mem, ptrs, keep = self._prepare(u)
        out, optr = self._alloc(mem, self.n_elements)
        check(lib().pfg_energy_per_element(self._h, ptrs[0], mem, _prec(precision), optr), self._h,
              "pfg_energy_per_element")
        return out

    def assemble_gradient(self, u, precision="fp64"):
        """NLAssembler::assemble_gradient (assembler/Assembler.cpp:574-643)."""
        self._check_len(u, self.n_dofs, "u")
        mem, ptrs, keep = self._prepare(u)
        out, optr = self._alloc(mem, self.n_dofs)
        check(lib().pfg_gradient(self._h, ptrs[0], mem, _prec(precision), optr), self._h, "pfg_gradient")
        return out

    def hessian_nnz(self) -> int:
        if self._nnz is None:
            nnz = ctypes.c_longlong()
            check(lib().pfg_hessian_pattern(self._h, ctypes.byref(nnz)), self._h, "pfg_hessian_pattern")
            self._nnz = int(nnz.value)
        return self._nnz

    def hessian_pattern(self, device: bool = False):
        """CSC (outer, inner) of the Hessian; int32, Eigen ColMajor layout."""
        nnz = self.hessian_nnz()
        if device:
            import torch
            outer = torch.empty(self.n_dofs + 1, dtype=torch.int32, device=f"cuda:{self.device}")
            inner = torch.empty(nnz, dtype=torch.int32, device=f"cuda:{self.device}")
            check(lib().pfg_set_stream(self._h, ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)),
                  self._h, "pfg_set_stream")
            check(lib().pfg_hessian_pattern_copy(self._h, ctypes.c_void_p(outer.data_ptr()),
                                                 ctypes.c_void_p(inner.data_ptr()), PFG_MEM_DEVICE),
                  self._h, "pfg_hessian_pattern_copy")
            return outer, inner
        outer = np.empty(self.n_dofs + 1, dtype=np.int32)
        inner = np.empty(nnz, dtype=np.int32)
        check(lib().pfg_set_stream(self._h, None), self._h, "pfg_set_stream")
        check(lib().pfg_hessian_pattern_copy(self._h, ctypes.c_void_p(outer.ctypes.data),
                                             ctypes.c_void_p(inner.ctypes.data), PFG_MEM_HOST),
              self._h, "pfg_hessian_pattern_copy")
        return outer, inner

    def assemble_hessian_values(self, u, precision="fp64", project_to_psd: bool = False):
        """CSC values of the Hessian (numpy for host u, torch CUDA tensor for device u)."""
        self._check_len(u, self.n_dofs, "u")
        nnz = self.hessian_nnz()
        mem, ptrs, keep = self._prepare(u)
        out, optr = self._alloc(mem, nnz)
        check(lib().pfg_hessian(self._h, ptrs[0], mem, _prec(precision), int(bool(project_to_psd)), optr),
              self._h, "pfg_hessian")
        return out

    def assemble_hessian(self, u, precision="fp64", project_to_psd: bool = False):
        """NLAssembler::assemble_hessian (assembler/Assembler.cpp:645-771).

        Host input -> scipy.sparse.csc_matrix; device input -> torch sparse CSR
        tensor of H^T (= H: the pattern is structurally symmetric).
        """
        vals = self.assemble_hessian_values(u, precision, project_to_psd)
        if _is_device(vals):
            import torch
            outer, inner = self.hessian_pattern(device=True)
            return torch.sparse_csr_tensor(outer.long(), inner.long(), vals, size=(self.n_dofs, self.n_dofs))
        import scipy.sparse as sp
        outer, inner = self.hessian_pattern()
        return sp.csc_matrix((vals, inner, outer), shape=(self.n_dofs, self.n_dofs))

    def hessian_apply(self, p, values=None):
        """q = H p with the library's SpMV (pfg_hessian_apply): H from `values` (a CUDA
        float64 tensor of nnz entries) or, when None, the last Hessian assembled into
        the context (assemble_hessian_into_context).  Deterministic."""
        self._check_len(p, self.n_dofs, "p")
        mem, ptrs, keep = self._prepare(p)
        vptr = None
        if values is not None:
            if not _is_device(values):
                raise ValueError("values must be a CUDA tensor")
            vptr = ctypes.c_void_p(values.data_ptr())
        out, optr = self._alloc(mem, self.n_dofs)
        check(lib().pfg_hessian_apply(self._h, vptr, ptrs[0], mem, optr), self._h, "pfg_hessian_apply")
        return out

    def assemble_hessian_into_context(self, u, precision="fp64", project_to_psd: bool = False):
        """Assemble the Hessian into the context's own device buffer (no copy out)."""
        self._check_len(u, self.n_dofs, "u")
        self.hessian_nnz()
        mem, ptrs, keep = self._prepare(u)
        check(lib().pfg_hessian(self._h, ptrs[0], mem, _prec(precision), int(bool(project_to_psd)), None),
              self._h, "pfg_hessian")

    def inverted_count(self) -> int:
        c = ctypes.c_longlong()
        check(lib().pfg_inverted_count(self._h, ctypes.byref(c)), self._h, "pfg_inverted_count")
        return int(c.value)

    # -- adjoint terms (ElasticForceDerivative) ------------------------------------
    def force_material_derivative(self, u, adjoint):
        """term = [-sum da (lnJ F^-T):grad p ; -sum da (F - F^-T):grad p], 2E entries."""
        self._check_len(u, self.n_dofs, "u")
        self._check_len(adjoint, self.n_dofs, "adjoint")
        mem, ptrs, keep = self._prepare(u, adjoint)
        out, optr = self._alloc(mem, 2 * self.n_elements)
        check(lib().pfg_material_vjp(self._h, ptrs[0], ptrs[1], mem, optr), self._h, "pfg_material_vjp")
        return out

    def force_shape_derivative(self, u, adjoint, precision="fp64"):
        """Adjoint shape term indexed by geometric node (3 N_g entries)."""
        self._check_len(u, self.n_dofs, "u")
        self._check_len(adjoint, self.n_dofs, "adjoint")
        mem, ptrs, keep = self._prepare(u, adjoint)
        out, optr = self._alloc(mem, 3 * self.n_geom_nodes)
        check(lib().pfg_shape_vjp(self._h, ptrs[0], ptrs[1], mem, _prec(precision), optr), self._h,
              "pfg_shape_vjp")
        return out

    def assemble_mass_matrix_values(self, rho=None):
        """MassMatrixAssembler's mass matrix values (nnz doubles, the Hessian pattern):
        sum_e rho_e int phi_a phi_b I; rho per element, None for 1.  Host arrays in,
        numpy out; a CUDA tensor rho gives a CUDA tensor."""
        mem, ptrs, keep = self._prepare(rho) if rho is not None else self._prepare()
        if rho is not None:
            self._check_len(rho, self.n_elements, "rho")
        out, optr = self._alloc(mem, self.hessian_nnz())
        check(lib().pfg_mass_matrix(self._h, ptrs[0] if rho is not None else None, mem, optr), self._h,
              "pfg_mass_matrix")
        return out

    def lump_matrix(self, values):
        """utils::lump_matrix (utils/MatrixUtils.cpp:84-101) of a matrix in the Hessian
        pattern: the dense diagonal of its row sums (3N doubles), each summed in
        ascending column order.  numpy in, numpy out; a CUDA tensor gives a CUDA tensor."""
        self._check_len(values, self.hessian_nnz(), "values")
        mem, ptrs, keep = self._prepare(values)
        out, optr = self._alloc(mem, self.n_dofs)
        check(lib().pfg_lump_matrix(self._h, ptrs[0], mem, optr), self._h, "pfg_lump_matrix")
        return out

    def dense_matrix(self, values):
        """DenseMatrixCache::mat() (utils/MatrixCache.hpp:136-177) of a matrix in the
        Hessian pattern: the dense ndof x ndof array, zeros outside the pattern.
        numpy in, numpy out (C-contiguous, element [row, col]); a CUDA tensor gives a
        CUDA tensor."""
        self._check_len(values, self.hessian_nnz(), "values")
        mem, ptrs, keep = self._prepare(values)
        out, optr = self._alloc(mem, self.n_dofs * self.n_dofs)
        check(lib().pfg_dense_matrix(self._h, ptrs[0], mem, optr), self._h, "pfg_dense_matrix")
        # the library writes column-major: the flat array is the transpose's rows
        return out.reshape(self.n_dofs, self.n_dofs).T

    def assemble_hessian_dense(self, u, precision="fp64", project_to_psd=False):
        """assemble_hessian with a DenseMatrixCache: the Hessian as a dense array
        (Assembler.cpp:306-316 merges the dense caches before its sparseView())."""
        return self.dense_matrix(self.assemble_hessian_values(u, precision, project_to_psd=project_to_psd))

    def assemble_lumped_mass(self, rho=None):
        """The lumped mass matrix's diagonal, lump_matrix(mass), as BCLagrangianForm
        builds it (BCLagrangianForm.cpp:68) and State does for
        solver.advanced.lump_mass_matrix (State.cpp:1542-1544)."""
        return self.lump_matrix(self.assemble_mass_matrix_values(rho))

    def assemble_mass_matrix(self, rho=None):
        """The mass matrix as scipy CSC (host)."""
        import scipy.sparse as sp
        vals = self.assemble_mass_matrix_values(None if rho is None else np.asarray(rho, dtype=np.float64))
        outer, inner = self.hessian_pattern()
        return sp.csc_matrix((vals, inner, outer), shape=(self.n_dofs, self.n_dofs))

    # -- material (AssemblerUtils::make_assembler's formulation name) ------------------
    MATERIALS = {"NeoHookean": 0, "IsochoricNeoHookean": 1, "SaintVenant": 2, "LinearElasticity": 3,
                 "MooneyRivlin": 4, "MooneyRivlin3Param": 5, "VolumePenalty": 6, "HookeLinearElasticity": 7,
                 "UnconstrainedOgden": 9, "IncompressibleOgden": 10, "MooneyRivlin3ParamSymbolic": 11}
    SAINT_VENANT_TENSOR = 8  # "SaintVenant" with an elasticity_tensor
    # the GenericMatParam names of the parameterised formulations, in pfg_set_material_params order
    MATERIAL_PARAMS = {"MooneyRivlin": ("c1", "c2", "k"), "MooneyRivlin3Param": ("c1", "c2", "c3", "d1"),
                       "VolumePenalty": ("k",), "MooneyRivlin3ParamSymbolic": ("c1", "c2", "c3", "d1")}
    # the Ogden formulations' GenericMatParams (OgdenElasticity.cpp:7-10, 48-51): one value
    # per term for each list; IncompressibleOgden's k is one GenericMatParam
    OGDEN_PARAMS = {"UnconstrainedOgden": ("alphas", "mus", "Ds"), "IncompressibleOgden": ("c", "m", "k")}
    OGDEN_MAX_TERMS = {"UnconstrainedOgden": 2, "IncompressibleOgden": 3}

    def set_material(self, formulation: str, **params):
        """Switch the elastic formulation (AssemblerUtils::make_assembler's name).

        "NeoHookean" (default), "IsochoricNeoHookean", "SaintVenant" (isotropic) and
        "LinearElasticity" use the per-element lambda/mu.  "MooneyRivlin" (c1, c2, k),
        "MooneyRivlin3Param" and "MooneyRivlin3ParamSymbolic" (c1, c2, c3, d1) and "VolumePenalty" (k) take their
        parameters as keywords, each a scalar or one value per element (host arrays
        or CUDA tensors).  "UnconstrainedOgden" takes alphas, mus, Ds (lists of one
        entry per term, 1 or 2 terms) and "IncompressibleOgden" c, m (1 to 3 terms)
        and k, each entry again a scalar or one value per element.  "HookeLinearElasticity" takes ``elasticity_tensor``: the 21
        entries C(i, j), i <= j, of its 6 x 6 Voigt tensor, row by row (the reference's
        material key; ``isotropic_elasticity_tensor`` gives the lambda/mu one); so does
        "SaintVenant" given ``elasticity_tensor``, which is then anisotropic.  Every
        formulation but NeoHookean is assembled in FP64.  The material derivative exists
        for NeoHookean and LinearElasticity, the shape derivative for all but SaintVenant
        and HookeLinearElasticity (as in the reference's assemblers)."""
        if formulation not in self.MATERIALS:
            raise ValueError(f"unknown formulation {formulation!r}; one of {sorted(self.MATERIALS)}")
        mat_id = self.MATERIALS[formulation]
        if formulation == "HookeLinearElasticity" or (formulation == "SaintVenant" and params):
            # SaintVenant with elasticity_tensor: the anisotropic form (PFG_MAT_SAINT_VENANT_TENSOR)
            if set(params) != {"elasticity_tensor"}:
                raise ValueError(f"{formulation} takes the parameter elasticity_tensor, got {sorted(params)}")
            self.set_elasticity_tensor(params["elasticity_tensor"])
            params = {}
            if formulation == "SaintVenant":
                mat_id = self.SAINT_VENANT_TENSOR
        if formulation in self.OGDEN_PARAMS:
            self.set_material_params(*self._ogden_params(formulation, params))
            check(lib().pfg_set_material(self._h, mat_id), self._h, "pfg_set_material")
            self.material = formulation
            return
        names = self.MATERIAL_PARAMS.get(formulation, ())
        if set(params) != set(names):
            raise ValueError(f"{formulation} takes the parameters {list(names)}, got {sorted(params)}")
        if names:
            self.set_material_params(*(params[n] for n in names))
        check(lib().pfg_set_material(self._h, mat_id), self._h, "pfg_set_material")
        self.material = formulation

    def set_composite(self, components, element_component=None):
        """MaterialSum (SumModel.cpp:43-78) or MultiModels (MultiModel.cpp:35-58).

        components: a list (at most 4) of dicts, each {"formulation": name, ...} with the
        formulation's parameters as set_material takes them, and optionally "lam" / "mu"
        (per-element or scalar Lame parameters of that component; default: the
        assembler's).  element_component: None adds all components on every element
        (MaterialSum); else one component index per element (MultiModels).  Assembled
        in FP64; set_material leaves the composition."""
        E = self.n_elements
        if not 1 <= len(components) <= 4:
            raise ValueError("1 to 4 components")
        for k, comp in enumerate(components):
            comp = dict(comp)
            name = comp.pop("formulation")
            lam = comp.pop("lam", None)
            mu = comp.pop("mu", None)
            if (lam is None) != (mu is None):
                raise ValueError("give both lam and mu of a component, or neither")
            mat = self.MATERIALS.get(name)
            if mat is None and name != "NeoHookean":
                raise ValueError(f"unknown formulation {name!r}")
            c21 = None
            if name == "HookeLinearElasticity" or (name == "SaintVenant" and "elasticity_tensor" in comp):
                c21 = np.ascontiguousarray(np.asarray(comp.pop("elasticity_tensor"), dtype=np.float64).ravel())
                if c21.size != 21:
                    raise ValueError("the elasticity tensor takes 21 entries")
                if name == "SaintVenant":
                    mat = self.SAINT_VENANT_TENSOR
            if name in self.OGDEN_PARAMS:
                vals = self._ogden_params(name, comp)
            else:
                names = self.MATERIAL_PARAMS.get(name, ())
                if set(comp) != set(names):
                    raise ValueError(f"{name} takes the parameters {list(names)}, got {sorted(comp)}")
                vals = [comp[n] for n in names]
            packed = (np.ascontiguousarray(np.stack([np.broadcast_to(np.asarray(v, dtype=np.float64), (E,))
                                                     for v in vals])) if vals else None)
            lv = None if lam is None else np.ascontiguousarray(np.broadcast_to(np.asarray(lam, dtype=np.float64), (E,)))
            mv = None if mu is None else np.ascontiguousarray(np.broadcast_to(np.asarray(mu, dtype=np.float64), (E,)))
            ptr = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)
            check(lib().pfg_set_component(self._h, k, mat, ptr(lv), ptr(mv), ptr(packed), len(vals), ptr(c21),
                                          PFG_MEM_HOST), self._h, "pfg_set_component")
        sel = None
        if element_component is not None:
            sel = np.ascontiguousarray(np.asarray(element_component, dtype=np.int32).ravel())
            if sel.size != E:
                raise ValueError(f"element_component must have {E} entries")
        check(lib().pfg_set_composite(self._h, len(components), None if sel is None else ctypes.c_void_p(sel.ctypes.data)),
              self._h, "pfg_set_composite")
        self.material = "MultiModels" if sel is not None else "MaterialSum"

    def _ogden_params(self, formulation, params):
        """The flat pfg_set_material_params list of an Ogden formulation: alphas, mus, Ds
        (three lists of K terms), or c, m (two lists of K terms) and k."""
        keys = self.OGDEN_PARAMS[formulation]
        if set(params) != set(keys):
            raise ValueError(f"{formulation} takes the parameters {list(keys)}, got {sorted(params)}")
        lists = [list(params[k]) if isinstance(params[k], (list, tuple)) else [params[k]] for k in keys]
        if formulation == "IncompressibleOgden":
            if len(lists[2]) != 1:
                raise ValueError("IncompressibleOgden takes one k")
            terms = lists[:2]
        else:
            terms = lists
        K = len(terms[0])
        if any(len(t) != K for t in terms) or not 1 <= K <= self.OGDEN_MAX_TERMS[formulation]:
            raise ValueError(f"{formulation} takes 1 to {self.OGDEN_MAX_TERMS[formulation]} terms, "
                             f"the same number in {list(keys[:len(terms)])}")
        return [v for lst in lists for v in lst]

    def set_elasticity_tensor(self, c21):
        """ElasticityTensor::set_from_entries with 21 entries (MatParams.cpp:180-205):
        C(i, j), i <= j, row by row, over the Voigt strain (e00, e11, e22, 2e12, 2e02, 2e01)."""
        c = np.ascontiguousarray(np.asarray(c21, dtype=np.float64).ravel())
        if c.size != 21:
            raise ValueError("the elasticity tensor takes 21 entries")
        check(lib().pfg_set_elasticity_tensor(self._h, ctypes.c_void_p(c.ctypes.data)), self._h,
              "pfg_set_elasticity_tensor")

    @staticmethod
    def isotropic_elasticity_tensor(lam: float, mu: float):
        """The 21 entries ElasticityTensor::set_from_lambda_mu sets (MatParams.cpp:211-260)."""
        C = np.zeros((6, 6))
        C[:3, :3] = lam
        C[[0, 1, 2], [0, 1, 2]] = 2 * mu + lam
        C[[3, 4, 5], [3, 4, 5]] = mu
        return C[np.triu_indices(6)]

    def set_material_params(self, *params):
        """Per-element parameters of the current or next parameterised formulation, in
        MATERIAL_PARAMS order (pfg_set_material_params)."""
        E = self.n_elements
        if not 1 <= len(params) <= 8:
            raise ValueError("1 to 8 parameters")
        if any(_is_device(p) for p in params):
            import torch
            cols = [p if _is_device(p) else torch.tensor(p, dtype=torch.float64) for p in params]
            packed = torch.stack([torch.broadcast_to(c.to(device=f"cuda:{self.device}", dtype=torch.float64), (E,))
                                  for c in cols]).contiguous()
        else:
            packed = np.ascontiguousarray(
                np.stack([np.broadcast_to(np.asarray(p, dtype=np.float64), (E,)) for p in params]))
        mem, ptrs, keep = self._prepare(packed)
        check(lib().pfg_set_material_params(self._h, ptrs[0], len(params), mem), self._h, "pfg_set_material_params")

    # -- Dirichlet reduction (NLProblem + BCLagrangianForm projection) ---------------
    def set_dirichlet(self, dofs):
        """Constrained dofs (BCLagrangianForm boundary_nodes_); builds the reduced pattern."""
        d = np.ascontiguousarray(np.asarray(dofs, dtype=np.int32).ravel())
        check(lib().pfg_set_dirichlet(self._h, ctypes.c_void_p(d.ctypes.data) if d.size else None, int(d.size)),
              self._h, "pfg_set_dirichlet")
        n = ctypes.c_int()
        nnz = ctypes.c_longlong()
        check(lib().pfg_reduced_pattern(self._h, ctypes.byref(n), ctypes.byref(nnz)), self._h, "pfg_reduced_pattern")
        self.n_free = int(n.value)
        self._red_nnz = int(nnz.value)

    def reduced_pattern(self):
        """CSC (outer, inner) of the reduced Hessian (BCLagrangianForm::project_hessian)."""
        outer = np.empty(self.n_free + 1, dtype=np.int32)
        inner = np.empty(self._red_nnz, dtype=np.int32)
        check(lib().pfg_set_stream(self._h, None), self._h, "pfg_set_stream")
        check(lib().pfg_reduced_pattern_copy(self._h, ctypes.c_void_p(outer.ctypes.data),
                                             ctypes.c_void_p(inner.ctypes.data), PFG_MEM_HOST),
              self._h, "pfg_reduced_pattern_copy")
        return outer, inner

    def assemble_hessian_reduced_values(self, u, precision="fp64", project_to_psd: bool = False):
        """Values of the reduced Hessian at the full displacement u."""
        self._check_len(u, self.n_dofs, "u")
        mem, ptrs, keep = self._prepare(u)
        out, optr = self._alloc(mem, self._red_nnz)
        check(lib().pfg_hessian_reduced(self._h, ptrs[0], mem, _prec(precision), int(bool(project_to_psd)), optr),
              self._h, "pfg_hessian_reduced")
        return out

    def assemble_hessian_reduced(self, u, precision="fp64", project_to_psd: bool = False):
        """NLProblem::hessian's reduction: scipy CSC (host u) of size n_free."""
        import scipy.sparse as sp
        vals = self.assemble_hessian_reduced_values(u, precision, project_to_psd)
        outer, inner = self.reduced_pattern()
        if _is_device(vals):
            vals = vals.cpu().numpy()
        return sp.csc_matrix((vals, inner, outer), shape=(self.n_free, self.n_free))

    def assemble_gradient_reduced(self, u, precision="fp64"):
        """Gradient at the full u restricted to the free dofs (project_gradient)."""
        self._check_len(u, self.n_dofs, "u")
        mem, ptrs, keep = self._prepare(u)
        out, optr = self._alloc(mem, self.n_free)
        check(lib().pfg_gradient_reduced(self._h, ptrs[0], mem, _prec(precision), optr), self._h,
              "pfg_gradient_reduced")
        return out

    def reduced_to_full(self, y, x_bc=None):
        """Full x from the free-dof vector y and the boundary values x_bc (full size)."""
        self._check_len(y, self.n_free, "y")
        if x_bc is not None:
            self._check_len(x_bc, self.n_dofs, "x_bc")
        mem, ptrs, keep = self._prepare(y, x_bc)
        out, optr = self._alloc(mem, self.n_dofs)
        check(lib().pfg_reduced_to_full(self._h, ptrs[0], ptrs[1], mem, optr), self._h, "pfg_reduced_to_full")
        return out

    def synchronize(self):
        check(lib().pfg_synchronize(self._h), self._h, "pfg_synchronize")


class ElasticForm:
    """Mirror of solver::ElasticForm (solver/forms/ElasticForm.cpp) over the GPU assembler.

    Like Form (solver/forms/Form.hpp:26-56), the public derivatives are the
    unweighted ones times ``weight() / scale``.
    """

    def __init__(self, assembler: NeoHookeanAssembler, precision: str = "fp64"):
        self.assembler = assembler
        self.precision = precision
        self._weight = 1.0
        self._scale = 1.0
        self.project_to_psd = False
        self.enabled = True

    def name(self) -> str:
        return "elastic"

    def weight(self) -> float:
        return self._weight

    def set_weight(self, w: float):
        self._weight = float(w)

    def set_scale(self, s: float):
        self._scale = float(s)

    def set_project_to_psd(self, v: bool):
        self.project_to_psd = bool(v)

    # unweighted ------------------------------------------------------------
    def value_unweighted(self, x):
        return self.assembler.assemble_energy(x, self.precision)

    def value_per_element_unweighted(self, x):
        return self.assembler.assemble_energy_per_element(x, self.precision)

    def first_derivative_unweighted(self, x):
        return self.assembler.assemble_gradient(x, self.precision)

    def second_derivative_unweighted(self, x):
        return self.assembler.assemble_hessian(x, self.precision, self.project_to_psd)

    # weighted (Form.hpp) -----------------------------------------------------
    def value(self, x):
        return (self.weight() / self._scale) * self.value_unweighted(x)

    def value_per_element(self, x):
        return (self.weight() / self._scale) * self.value_per_element_unweighted(x)

    def first_derivative(self, x):
        return self.first_derivative_unweighted(x) * (self.weight() / self._scale)

    def second_derivative(self, x):
        return self.second_derivative_unweighted(x) * (self.weight() / self._scale)

    def is_step_valid(self, x0, x1) -> bool:
        """ElasticForm::is_step_valid (ElasticForm.cpp:388-396): reject NaN gradients."""
        g = self.first_derivative(x1)
        if _is_device(g):
            import torch
            return not bool(torch.isnan(g).any())
        return not bool(np.isnan(g).any())


class ElasticForceDerivative:
    """Static adjoint terms, as optimization/force_derivatives/ElasticForceDerivative.hpp:11-26."""

    @staticmethod
    def force_material_derivative(form: ElasticForm, t: float, x, x_prev, adjoint):
        return form.assembler.force_material_derivative(x, adjoint)

    @staticmethod
    def force_shape_derivative(form: ElasticForm, t: float, n_verts: int, x, x_prev, adjoint):
        if n_verts != form.assembler.n_geom_nodes:
            raise ValueError("n_verts must equal the number of geometric nodes")
        return form.assembler.force_shape_derivative(x, adjoint, "fp64")
