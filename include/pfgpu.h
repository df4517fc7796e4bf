/*
 * pfgpu.h — C ABI of the B200 NeoHookean assembly library (libpfgpu.so).
 *
 * Drop-in for PolyFEM's nonlinear-elasticity assembly path (iiiian/polyfem):
 * the NLAssembler virtuals that ElasticForm calls, the SparseMatrixCache that
 * ElasticForm owns, and the two ElasticForceDerivative adjoint terms.  Every
 * entry point takes plain pointers and sizes; no C++ or torch types cross it.
 *
 * Conventions (identical to the reference):
 *  - displacement / adjoint / gradient vectors are node-major: x[node*3 + d];
 *  - conn is the host's Basis::global() table, E x n int32 (row-major);
 *  - the Hessian is Eigen's ColMajor CSC (int32 outer/inner, sorted inner
 *    indices, structural entries stored even when zero); because the pattern
 *    is structurally symmetric these arrays are also the CSR arrays of H^T;
 *  - values are unweighted: the caller applies Form::weight()/scale.
 *  - NaN/inf from inverted elements (J <= 0) propagate exactly as in the
 *    reference; they are not an error status.
 *
 * Memory spaces: every call takes `mem`.  With PFG_MEM_HOST the pointers are
 * host memory, the call copies inputs to the device, runs, copies results
 * back and returns after the stream has synchronised.  With PFG_MEM_DEVICE
 * the pointers are device memory on the context's device and the call only
 * enqueues work on the context's stream (pfg_set_stream), returning at once.
 *
 * Calls on one context are not re-entrant and must be serialised by the
 * caller (as ElasticForm's mutable mat_cache_ requires in the reference).
 */
#ifndef PFGPU_H
#define PFGPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pfg_context pfg_context;

enum pfg_status
{
	PFG_OK = 0,
	PFG_ERR_INVALID = 1,     /* bad argument (null pointer, index out of range, bad enum) */
	PFG_ERR_CUDA = 2,        /* a CUDA runtime call failed; see pfg_last_error */
	PFG_ERR_OOM = 3,         /* device or host allocation failed */
	PFG_ERR_UNSUPPORTED = 4, /* beyond an implementation limit (e.g. the 32-bit reduction plan) */
	PFG_ERR_STATE = 5,       /* call made in the wrong state (e.g. pattern not built) */
	PFG_ERR_NUMERIC = 6      /* the matrix is not positive definite (pfg_direct_factorize) */
};

enum pfg_elem_type
{
	PFG_P1_TET = 1, /* 4-node tetrahedron, 1-point quadrature */
	PFG_P2_TET = 2, /* 10-node tetrahedron on P1 geometry, 4-point quadrature */
	PFG_Q1_HEX = 3  /* 8-node hexahedron, 2x2x2 Gauss quadrature */
};

enum pfg_precision
{
	PFG_FP64 = 0,    /* all arithmetic in FP64 (the drop-in) */
	PFG_FP32 = 1,    /* FP32 arithmetic; det(F)/log J and reductions in FP64 */
	PFG_SPLIT32 = 2, /* Hessian: kinematics (J^-T, F, det/log J, F^-T, basis
	                    gradients) in FP64; for P2 and Q1 the element contraction
	                    on the tensor cores (tcgen05, each FP32 operand split into
	                    two TF32 halves, 3 products, FP32 accumulation), for P1 on
	                    CUDA cores in FP32; staged element blocks in FP32, every
	                    CSC entry summed in FP64.
	                    Relative Frobenius error vs PFG_FP64 <= 1e-6.
	                    Energy/gradient/shape VJP treat it as PFG_FP32. */
	PFG_SPLIT32_SIMT = 3 /* PFG_SPLIT32 with the contraction on CUDA cores (FP32
	                        FMA) for every element type; same bound. */
};

enum pfg_mem
{
	PFG_MEM_HOST = 0,
	PFG_MEM_DEVICE = 1
};

/* Mesh and material description consumed by pfg_create.
 * Replaces the inputs NLAssembler reads through ElementBases / AssemblyValsCache
 * (assembler/Assembler.hpp:244-291, assembler/AssemblyValsCache.hpp) and
 * LameParameters (assembler/MatParams.cpp:368-401). */
typedef struct pfg_mesh_desc
{
	int elem_type;        /* enum pfg_elem_type */
	int n_elements;       /* E >= 0 */
	int n_nodes;          /* N: FE nodes (n_bases); dofs = 3N */
	int n_geom_nodes;     /* N_g: geometric nodes (rows of X) */
	const int *conn;      /* E x n FE node ids (Basis::global()[0].index), host */
	const int *gconn;     /* E x n_g geometric node ids, host; NULL = conn (isoparametric) */
	const double *X;      /* N_g x 3 rest positions of the geometric nodes, host */
	const double *lambda; /* E per-element Lame lambda, host */
	const double *mu;     /* E per-element Lame mu, host */
	int device;           /* CUDA device ordinal */
} pfg_mesh_desc;

/* Creates a context: uploads the mesh in the device layout and validates
 * every index.  Replaces AssemblyValsCache::init (assembler/AssemblyValsCache.cpp:11-32)
 * and ElasticForm's constructor (solver/forms/ElasticForm.cpp:238-280). */
int pfg_create(const pfg_mesh_desc *desc, pfg_context **out);
int pfg_destroy(pfg_context *ctx);

/* cudaStream_t as void*; NULL selects the legacy default stream. */
int pfg_set_stream(pfg_context *ctx, void *stream);

/* Per-element Lame parameters; replaces LameParameters::lambda_mat_/mu_mat_
 * updates (NeoHookeanElasticity.hpp:58-62, update_lame_params). */
int pfg_set_lame(pfg_context *ctx, const double *lambda, const double *mu, int mem);

/* Rest positions of the geometric nodes (N_g x 3); shape optimisation moves them. */
int pfg_set_rest_positions(pfg_context *ctx, const double *X, int mem);

/* Total energy.  Replaces NLAssembler::assemble_energy (assembler/Assembler.cpp:495-531).
 * `out` is one double in the `mem` space.  Deterministic for a fixed mesh. */
int pfg_energy(pfg_context *ctx, const double *u, int mem, int prec, double *out);

/* Energy of every element.  Replaces NLAssembler::assemble_energy_per_element
 * (assembler/Assembler.cpp:533-572).  `out` holds E doubles. */
int pfg_energy_per_element(pfg_context *ctx, const double *u, int mem, int prec, double *out);

/* Gradient (3N doubles).  Replaces NLAssembler::assemble_gradient
 * (assembler/Assembler.cpp:574-643).  Deterministic for a fixed mesh. */
int pfg_gradient(pfg_context *ctx, const double *u, int mem, int prec, double *g);

/* Builds the Hessian sparsity pattern and the element->slot map if they do not
 * exist yet, and returns nnz.  Replaces the first-call branch of
 * SparseMatrixCache::get_matrix (utils/MatrixCache.cpp:134-212). */
int pfg_hessian_pattern(pfg_context *ctx, long long *nnz);

/* Copies the CSC index arrays: outer (3N+1) and inner (nnz) int32. */
int pfg_hessian_pattern_copy(pfg_context *ctx, int *outer, int *inner, int mem);

/* Assembles the Hessian values (nnz doubles, CSC order) into `values` (device
 * memory: written in place, no extra copy); with values == NULL they go to the
 * context's device buffer (pfg_hessian_device_csc), which keeps the result of
 * the last such call.
 * Builds the pattern on the first call.  Replaces NLAssembler::assemble_hessian
 * (assembler/Assembler.cpp:645-771) and the later-call branch of
 * SparseMatrixCache (utils/MatrixCache.cpp:88-113, 214-225).
 * project_psd != 0 projects every element matrix onto the PSD cone before the
 * scatter, as ipc::project_to_psd (CLAMP) does at Assembler.cpp:693-694: an
 * element whose smallest eigenvalue is > 0 is kept as it is, otherwise it
 * becomes V max(l, 0) V^T (eigendecomposition in FP64 on the device). */
int pfg_hessian(pfg_context *ctx, const double *u, int mem, int prec, int project_psd, double *values);

/* q = H p (3N doubles each, in `mem`) with the Hessian in the full pattern:
 * `values` (device memory, nnz doubles) or, when NULL, the values of the last
 * pfg_hessian call that wrote into the context.  H is symmetric, so this is also
 * H^T p, the product the reference's adjoint terms form with Eigen's sparse
 * matrix-vector product (e.g. `term = -hessian.transpose() * adjoint_zeroed`,
 * optimization/force_derivatives/PressureForceDerivative.cpp:24).  One warp per
 * node, each entry summed in a fixed order: bitwise deterministic.  Requires the
 * pattern (any pfg_hessian or pfg_hessian_pattern call builds it). */
int pfg_hessian_apply(pfg_context *ctx, const double *values, const double *p, int mem, double *q);

/* Device pointers of the context-owned CSC arrays (valid until pfg_destroy). */
int pfg_hessian_device_csc(pfg_context *ctx, const int **outer, const int **inner, double **values);

/* Adjoint material term, 2E doubles [d/dlambda per element ; d/dmu per element]:
 * term[e] = -sum_q da (lnJ F^-T):grad p, term[E+e] = -sum_q da (F - F^-T):grad p.
 * Replaces ElasticForceDerivative::force_material_derivative
 * (optimization/force_derivatives/ElasticForceDerivative.cpp:35-133). */
int pfg_material_vjp(pfg_context *ctx, const double *u, const double *p, int mem, double *out);

/* Adjoint shape term, 3*N_g doubles indexed by geometric node.  Replaces
 * ElasticForceDerivative::force_shape_derivative
 * (optimization/force_derivatives/ElasticForceDerivative.cpp:135-264). */
int pfg_shape_vjp(pfg_context *ctx, const double *u, const double *p, int mem, int prec, double *out);

/* Elements whose det(F) was <= 0 (or NaN) in the last energy/gradient call. */
int pfg_inverted_count(pfg_context *ctx, long long *count);

/* Waits for all work enqueued on the context's stream. */
int pfg_synchronize(pfg_context *ctx);

/* Human-readable detail of the last failing call on this context (never NULL). */
const char *pfg_last_error(const pfg_context *ctx);
const char *pfg_status_string(int status);

/* Library version, e.g. 100 for 0.1.0. */
int pfg_version(void);

/* ---------------------------------------------------------------------------
 * Other materials.  AssemblerUtils::make_assembler picks the elastic formulation by
 * name (assembler/AssemblerUtils.cpp:69-93); NeoHookean is this library's default
 * and its fully tuned path.  pfg_set_material switches a context to
 *   PFG_MAT_ISOCHORIC_NEOHOOKEAN: IsochoricNeoHookean (IsochoricNeoHookean.hpp:19-33),
 *                                 psi = mu/2 (tr(F^T F) / J^(2/3) - 3);
 *   PFG_MAT_SAINT_VENANT        : SaintVenantElasticity (SaintVenantElasticity.cpp:
 *                                 209-267) with the isotropic elasticity tensor of
 *                                 (lambda, mu) (ElasticityTensor::set_from_lambda_mu),
 *                                 psi = lambda/2 tr(E)^2 + mu |E|^2, E = (F^T F - I)/2;
 * both with the per-element (lambda, mu) of pfg_set_lame, and the formulations
 * defined by their energy density alone, differentiated automatically as the
 * reference does (GenericElastic AutodiffType::STRESS, GenericElastic.cpp:493-611):
 *   PFG_MAT_LINEAR_ELASTICITY   : LinearElasticity (LinearElasticity.cpp:113-139),
 *                                 psi = mu eps:eps + lambda/2 tr(eps)^2,
 *                                 eps = (grad u + grad u^T)/2; (lambda, mu) of pfg_set_lame;
 *   PFG_MAT_MOONEY_RIVLIN       : MooneyRivlinElasticity (MooneyRivlinElasticity.hpp:25-46),
 *                                 parameters (c1, c2, k);
 *   PFG_MAT_MOONEY_RIVLIN_3PARAM: MooneyRivlin3ParamElasticity
 *                                 (MooneyRivlin3ParamElasticity.hpp:26-49), (c1, c2, c3, d1);
 *   PFG_MAT_VOLUME_PENALTY      : VolumePenalty (VolumePenalty.hpp:20-34), (k);
 *   PFG_MAT_HOOKE               : HookeLinearElasticity (HookeLinearElasticity.cpp:
 *                                 332-423), psi = 1/2 sigma:eps with the Voigt stress
 *                                 sigma = C eps of one anisotropic elasticity tensor C
 *                                 (pfg_set_elasticity_tensor), eps the small strain;
 *   PFG_MAT_SAINT_VENANT_TENSOR : SaintVenantElasticity with that anisotropic tensor
 *                                 (SaintVenantElasticity.cpp:209-267), psi = 1/2 S:E,
 *                                 S = C E in Voigt form, E = (F^T F - I)/2;
 *   PFG_MAT_UNCONSTRAINED_OGDEN : UnconstrainedOgdenElasticity (OgdenElasticity.tpp:8-57),
 *                                 psi = sum_t 2 mu_t/alpha_t^2 (sum_i s_i^alpha_t - 3)
 *                                       + sum_t (J - 1)^(2(t+1)) / D_t,
 *                                 s_i = J^(-1/3) x the principal stretches of F;
 *                                 parameters (alpha_0.., mu_0.., D_0..), 1 or 2 terms;
 *   PFG_MAT_INCOMPRESSIBLE_OGDEN: IncompressibleOgdenElasticity (OgdenElasticity.tpp:
 *                                 59-94), psi = sum_t c_t/m_t^2 (sum_i s_i^m_t - 3)
 *                                 + k/2 ln^2 J; parameters (c_0.., m_0.., k), 1 to 3 terms;
 *   PFG_MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC: MooneyRivlin3ParamSymbolic (MooneyRivlin3ParamSymbolic.cpp:
 *                                 317-340), psi = c1 (I1~ - 3) + c2 (I2~ - 3)
 *                                 + c3 (I1~ - 3)(I2~ - 3) + d1 ln^2 J, (c1, c2, c3, d1).
 * Energy, gradient and Hessian (with project_psd and the Dirichlet reduction) then
 * follow the chosen material in PFG_FP64 (other precisions return
 * PFG_ERR_UNSUPPORTED).  The adjoint terms follow the reference's assemblers:
 * pfg_material_vjp (compute_dstress_dmu_dlambda) exists for NeoHookean and
 * LinearElasticity (dP/dmu = grad u + grad u^T, dP/dlambda = tr(grad u) I,
 * LinearElasticity.cpp:290-299); pfg_shape_vjp (compute_stress_grad_multiply_mat)
 * for every formulation here but the two SaintVenant ones and HookeLinearElasticity,
 * in PFG_FP64 for all but NeoHookean;
 * the others return PFG_ERR_UNSUPPORTED, where the reference throws "Not
 * implemented" (Assembler.hpp:147-156).  Takes effect for the calls that follow;
 * the pattern is unchanged.
 * ------------------------------------------------------------------------- */
enum pfg_material
{
	PFG_MAT_NEOHOOKEAN = 0,
	PFG_MAT_ISOCHORIC_NEOHOOKEAN = 1,
	PFG_MAT_SAINT_VENANT = 2,
	PFG_MAT_LINEAR_ELASTICITY = 3,
	PFG_MAT_MOONEY_RIVLIN = 4,
	PFG_MAT_MOONEY_RIVLIN_3PARAM = 5,
	PFG_MAT_VOLUME_PENALTY = 6,
	PFG_MAT_HOOKE = 7,
	PFG_MAT_SAINT_VENANT_TENSOR = 8,
	PFG_MAT_UNCONSTRAINED_OGDEN = 9,
	PFG_MAT_INCOMPRESSIBLE_OGDEN = 10,
	PFG_MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC = 11
};
int pfg_set_material(pfg_context *ctx, int material);

/* The elasticity tensor of PFG_MAT_HOOKE and PFG_MAT_SAINT_VENANT_TENSOR: ElasticityTensor (assembler/MatParams.cpp:
 * 91-123, 336-344), a symmetric 6 x 6 matrix over the Voigt strain
 * (e00, e11, e22, 2 e12, 2 e02, 2 e01), given as its 21 entries C(i, j), i <= j,
 * row by row: C00 C01 .. C05 C11 .. C15 .. C55 (the order of
 * ElasticityTensor::set_from_entries with 21 entries).  Host memory; one tensor
 * per context, as the reference's assembler holds one.  The calls of these two
 * materials return PFG_ERR_STATE until it is set. */
int pfg_set_elasticity_tensor(pfg_context *ctx, const double *c21);

/* Per-element parameters of PFG_MAT_MOONEY_RIVLIN (n_params 3: c1, c2, k),
 * PFG_MAT_MOONEY_RIVLIN_3PARAM and PFG_MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC (4: c1, c2,
 * c3, d1), PFG_MAT_VOLUME_PENALTY
 * (1: k), PFG_MAT_UNCONSTRAINED_OGDEN (3 K: alpha_0..alpha_K-1, mu_0.., D_0.., with
 * K = 1 or 2 terms, as GenericMatParams alphas, mus, Ds, OgdenElasticity.cpp:12-20)
 * and PFG_MAT_INCOMPRESSIBLE_OGDEN (2 K + 1: c_0.., m_0.., k, K = 1 to 3,
 * OgdenElasticity.cpp:53-60): the reference's GenericMatParam values (MatParams.cpp),
 * one per element, parameter-major: params[k * n_elements + e] is parameter k of
 * element e.  1 <= n_params <= 8.  The energy, gradient and Hessian calls of these
 * materials return PFG_ERR_STATE until parameters of a count the material takes
 * are set; the parameters stay with the context when the material changes. */
int pfg_set_material_params(pfg_context *ctx, const double *params, int n_params, int mem);

/* ---------------------------------------------------------------------------
 * Compositions of formulations.  MaterialSum (SumModel.cpp:43-78) adds the element
 * energies, gradients and Hessians of several formulations, each with its own
 * parameters; MultiModels (MultiModel.cpp:35-58) assembles every element with the
 * formulation of its body.  pfg_set_component sets component k (< PFG_MAX_COMPONENTS):
 * its material (any PFG_MAT_*), its per-element (lambda, mu) (NULL: the context's
 * pfg_set_lame values), its per-element parameters as pfg_set_material_params takes
 * them (params[q * n_elements + e], NULL / 0 for materials without), and the 21
 * tensor entries of PFG_MAT_HOOKE / PFG_MAT_SAINT_VENANT_TENSOR (host memory; NULL
 * otherwise); arrays in `mem`.  pfg_set_composite then switches the context to the
 * composition of components 0 .. n_components-1: element_component (host, n_elements
 * entries in [0, n_components)) gives each element's component (MultiModels), NULL
 * adds all components on every element (MaterialSum).  The element blocks are
 * combined per element before the PSD projection, as the reference projects the
 * composed element matrix.  Energy, per-element energy, gradient and Hessian, full
 * and Dirichlet-reduced, in PFG_FP64; the adjoint terms return PFG_ERR_UNSUPPORTED
 * (SumModel and MultiModel have none).  pfg_set_material leaves the composition.
 * ------------------------------------------------------------------------- */
#define PFG_MAX_COMPONENTS 4
int pfg_set_component(pfg_context *ctx, int k, int material, const double *lambda, const double *mu,
                      const double *params, int n_params, const double *c21, int mem);
int pfg_set_composite(pfg_context *ctx, int n_components, const int *element_component);

/* ---------------------------------------------------------------------------
 * Dirichlet reduction.  When the only constraint form of the nonlinear problem
 * is the Dirichlet one (BCLagrangianForm::can_project), NLProblem reduces the
 * full quantities by dropping the constrained dofs:
 *   Hessian:  BCLagrangianForm::project_hessian (BCLagrangianForm.cpp:165-212),
 *             called from NLProblem::full_hessian_to_reduced_hessian
 *             (solver/NLProblem.cpp:735-740);
 *   gradient: BCLagrangianForm::project_gradient (BCLagrangianForm.cpp:149-155),
 *             called from NLProblem::gradient (NLProblem.cpp:596-611);
 *   x:        NLProblem::reduced_to_full (NLProblem.cpp:713-735): free dofs from
 *             the reduced vector, constrained dofs from the boundary values.
 * Free dofs keep their order (old_to_new is increasing).  The reduced Hessian is
 * assembled directly in its reduced CSC (the full matrix is never written).
 * ------------------------------------------------------------------------- */

/* Constrained dof indices (host memory, any order, duplicates ignored); builds the
 * reduced pattern (and the full one if needed).  n = 0: no dof constrained. */
int pfg_set_dirichlet(pfg_context *ctx, const int *dofs, int n);

/* Number of free dofs and nonzeros of the reduced Hessian. */
int pfg_reduced_pattern(pfg_context *ctx, int *n_free, long long *nnz);

/* Reduced CSC index arrays: outer (n_free+1) and inner (nnz) int32. */
int pfg_reduced_pattern_copy(pfg_context *ctx, int *outer, int *inner, int mem);

/* Reduced Hessian values (nnz doubles) at the full displacement u (3N doubles);
 * values == NULL keeps them in the context.  project_psd as in pfg_hessian. */
int pfg_hessian_reduced(pfg_context *ctx, const double *u, int mem, int prec, int project_psd, double *values);

/* Gradient at the full displacement u, restricted to the free dofs (n_free doubles). */
int pfg_gradient_reduced(pfg_context *ctx, const double *u, int mem, int prec, double *g);

/* x (3N) from y (n_free) and x_bc (3N, read at the constrained dofs; NULL = 0). */
int pfg_reduced_to_full(pfg_context *ctx, const double *y, const double *x_bc, int mem, double *x);

/* ---------------------------------------------------------------------------
 * Mass matrix: MassMatrixAssembler's M = sum_e rho_e int phi_a phi_b I dV
 * (LinearAssembler::assemble with the Mass term, assembler/Assembler.cpp:157-260,
 * assembler/Mass.cpp:5-24), in the Hessian's CSC pattern (the linear assembler adds
 * all nine entries of every node block: the off-diagonal ones are stored zeros).
 * rho: per-element density (E doubles in `mem`) or NULL for 1.  values: nnz
 * doubles in `mem` (required).  Quadrature of order 2p as the reference's mass
 * quadrature (AssemblerUtils::quadrature_order("Mass")): the exact integral on the
 * affine tets, the 2x2x2 Gauss rule on Q1.  FP64; the context's Hessian values are
 * not touched. */
int pfg_mass_matrix(pfg_context *ctx, const double *rho, int mem, double *values);

/* ---------------------------------------------------------------------------
 * Row-sum lumping: polyfem::utils::lump_matrix (utils/MatrixUtils.cpp:84-101),
 * which BCLagrangianForm applies to the mass matrix (solver/forms/lagrangian/
 * BCLagrangianForm.cpp:68) and State to the mass matrix when
 * solver.advanced.lump_mass_matrix is set (State.cpp:1542-1544).
 * diag[r] = sum_k M(r, k), summed in ascending column order as the reference's
 * setFromTriplets sums the duplicates of (r, r): the diagonal of the lumped
 * matrix (every row has an entry, so the diagonal is dense).
 * values: nnz doubles in the Hessian pattern (e.g. pfg_mass_matrix output) in
 * `mem`; diag: 3N doubles in `mem`.  FP64.  Host-mode calls stage the values
 * in the buffer host-mode pfg_mass_matrix calls use. */
int pfg_lump_matrix(pfg_context *ctx, const double *values, int mem, double *diag);

/* ---------------------------------------------------------------------------
 * Dense assembly: polyfem::utils::DenseMatrixCache (utils/MatrixCache.hpp:136-177,
 * MatrixCache.cpp:326-403), whose mat() the assembler merges densely
 * (assembler/Assembler.cpp:306-316) before taking its sparseView().
 * dense[col * ndof + row] (column-major, ndof = 3 N, Eigen's default storage) =
 * the value of (row, col) in `values` (nnz doubles in the Hessian pattern, e.g.
 * pfg_hessian or pfg_mass_matrix output) and 0 outside the pattern.  values and
 * dense in `mem`; PFG_ERR_UNSUPPORTED when ndof^2 > PFG_DENSE_MAX_ENTRIES.  A
 * host-mode call allocates device staging for the values and the dense matrix
 * for the duration of the call. */
#define PFG_DENSE_MAX_ENTRIES (1LL << 29)
int pfg_dense_matrix(pfg_context *ctx, const double *values, int mem, double *dense);

/* ---------------------------------------------------------------------------
 * Linear solve on the device.  After every assembly the Newton step hands the
 * Hessian that NLProblem::hessian returns (solver/NLProblem.cpp:615-621) to its
 * linear solver through polysolve's linear::Solver (analyze_pattern, factorize,
 * solve; called inside the Newton solver of polysolve@47dc48d, external).  pfg_cg_solve is that hand-off without a host round trip: the
 * conjugate gradient of Eigen's ConjugateGradient<..., Lower|Upper,
 * DiagonalPreconditioner>, the "Eigen::ConjugateGradient" choice of polysolve,
 * run on the context's assembled Hessian:
 *   system = PFG_SYS_FULL   : the 3N x 3N Hessian of the last pfg_hessian call
 *                             that wrote into the context (values == NULL there);
 *   system = PFG_SYS_REDUCED: the n_free x n_free Hessian of the last
 *                             pfg_hessian_reduced call into the context.
 * `values` (device memory, nnz doubles of that pattern) replaces the context's
 * values when not NULL.  b and x have the system's size; x is the starting guess
 * when `guess` is non-zero, else the iteration starts at x = 0.  The iteration
 * stops when |b - H x| < tol |b| or after max_iter iterations; *iters and
 * *rel_res (host pointers, NULL allowed) receive the iteration count and
 * |b - H x| / |b| as Eigen's iterations() and error() report them.  Reaching
 * max_iter is not an error (Eigen reports it through info()): check *rel_res.
 * H must be symmetric positive definite for the iteration to converge (the
 * Dirichlet-reduced Hessian with project_psd, for instance).  The result is
 * bitwise deterministic. */
enum pfg_system
{
	PFG_SYS_FULL = 0,
	PFG_SYS_REDUCED = 1
};
int pfg_cg_solve(pfg_context *ctx, int system, const double *values, const double *b, int mem, double tol,
                 int max_iter, int guess, double *x, int *iters, double *rel_res);

/* Sparse direct solve on the device: the factorisation polysolve's direct choices
 * compute for the Newton step's SPD system (Eigen::SimplicialLDLT, Cholmod or
 * Pardiso at the reference's call sites: mesh/remesh/L2Projection.cpp:25-29,
 * State.cpp:1562-1565), as a multifrontal Cholesky P A P^T = L L^T with a nested
 * dissection ordering, in the three calls of polysolve's linear::Solver:
 *   pfg_direct_analyze   (analyzePattern): orders and analyses the pattern of
 *       `system` (PFG_SYS_FULL after pfg_hessian, PFG_SYS_REDUCED after
 *       pfg_set_dirichlet; host work, then the maps go to the device).  Repeat it
 *       when the pattern changes: pfg_set_dirichlet discards the reduced system's
 *       analysis.  PFG_ERR_OOM when the dense fronts do not fit in device memory,
 *       PFG_ERR_UNSUPPORTED beyond 65,535 fronts at one height of the tree;
 *   pfg_direct_factorize (factorize): factorises `values` (device memory, nnz
 *       doubles of the analysed pattern, both triangles stored; the lower one is
 *       read) or, with values == NULL, the system's values the last assembly left
 *       in the context.  PFG_ERR_NUMERIC when the matrix is not positive definite
 *       (Eigen's NumericalIssue): a non-positive or non-finite pivot.  The call
 *       waits for the factorisation to finish (it reads the pivot check);
 *   pfg_direct_solve     (solve): x = A^-1 b for b and x in `mem` (x may be b);
 *       with PFG_MEM_DEVICE it is asynchronous on the context's stream.
 * pfg_direct_free releases the analysis and the factor (pfg_destroy does too).
 * Every sum is taken in a fixed order, so factor and solution are bitwise
 * deterministic.  pfg_direct_stats (after analyze) and pfg_direct_symbolic (any
 * host pattern: full symmetric CSC of n columns with sorted rows; host only, no
 * device) write seven values: n, fronts, tree levels, doubles of the dense
 * fronts, entries of L, largest front order, flops of the factorisation. */
int pfg_direct_analyze(pfg_context *ctx, int system);
int pfg_direct_factorize(pfg_context *ctx, int system, const double *values);
int pfg_direct_solve(pfg_context *ctx, int system, const double *b, int mem, double *x);
int pfg_direct_free(pfg_context *ctx);
int pfg_direct_stats(const pfg_context *ctx, long long *stats);
int pfg_direct_symbolic(int n, const int *outer, const int *inner, long long *stats);

/* ---------------------------------------------------------------------------
 * Allocation-free energy.  No counterpart in the reference: PolyFEM always
 * owns its memory.  It exists for callers that must not allocate device
 * memory at all (a host that pre-plans every byte, or runs inside a pool it
 * does not own), for whom pfg_create is not an option because it allocates.
 *
 * Same result as pfg_energy for the same inputs.  Every pointer is device
 * memory on the current device and is owned by the caller:
 *   conn_soa  : [n][E] int32, local node a of element e at conn_soa[a*E + e]
 *   gconn_soa : [n_g][E] int32 (required for P2; NULL = conn_soa otherwise)
 *   X         : [N_g][3] float64 rest positions
 *   lame      : [E][2] float64 (lambda, mu) per element, 16-byte aligned (each
 *               pair is read as one 16-byte load; a misaligned pointer is
 *               refused with PFG_ERR_INVALID before anything is launched)
 *   u         : [3N] float64 displacement, node-major
 *   out       : 1 float64 (the energy)
 * The connectivity is trusted: every conn_soa entry must lie in [0, n_nodes)
 * and every gconn_soa entry in [0, n_geom_nodes).  pfg_create checks each index
 * on the host; this call cannot, because the tables are already on the device
 * and reading them back would need a host buffer, so an index out of range
 * reads out of bounds on the device.  The sizes are checked as pfg_create
 * checks them (3 n_nodes and E n below 2^31).
 * The call enqueues work on `stream` (cudaStream_t as void*, NULL = default
 * stream) and returns without synchronising.  It allocates nothing: the
 * reduction scratch is a fixed array inside the library's device image
 * (512 KiB, held by every GPU that loads the library until exit), which
 * limits n_elements to 256 * PFG_NOALLOC_MAX_BLOCKS = 16,777,216 (the energy
 * kernel takes 256 elements per block); larger meshes return
 * PFG_ERR_UNSUPPORTED with the limit in pfg_last_error(NULL).  All calls
 * share that array, so calls that overlap on the GPU race.  The first call on
 * a device looks up the array's address; make it before any stream capture.
 * Errors are reported through pfg_last_error(NULL).
 * ------------------------------------------------------------------------- */
#define PFG_NOALLOC_MAX_BLOCKS 65536
int pfg_energy_noalloc(int elem_type, int n_elements, int n_nodes, int n_geom_nodes, const int *conn_soa,
                       const int *gconn_soa, const double *X, const double *lame, const double *u, int prec,
                       double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PFGPU_H */
