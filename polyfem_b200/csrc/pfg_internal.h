// Internal declarations shared by the host API (pfg_api.cu) and the kernel
// launchers (pfg_kernels.cu, pfg_tc.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace pfg
{

// Device-resident mesh in the layout the kernels read.
//  conn     : [n][E] int32 (structure of arrays: local node a of all elements is contiguous)
//  gconn    : [n_g][E] int32 (aliases conn for isoparametric elements)
//  X        : [N_g][3] float64 rest positions
//  lame     : [E] (lambda, mu) float64 pairs
//  inc_off  : [N+1] offsets of each FE node's incidences ("strips") in inc_eb
//  inc_eb   : [E*n] e*n + b for every incidence (element e holds the node at local b),
//             grouped by node, elements ascending
//  eb_inc   : [E*n] the incidence index of (e, b), i.e. the inverse permutation of inc_eb
//  ginc_off / ginc_eb : the same for the geometric nodes (alias inc_* when isoparametric)
struct DevMesh
{
	int et = 0, E = 0, N = 0, Ng = 0;
	int mat = 0; // pfg_material: 0 NeoHookean, 1 IsochoricNeoHookean, 2 SaintVenant, 3 LinearElasticity,
	             // 4 MooneyRivlin, 5 MooneyRivlin3Param, 6 VolumePenalty, 7 HookeLinearElasticity,
	             // 8 SaintVenant with an anisotropic tensor, 9 UnconstrainedOgden, 10 IncompressibleOgden,
	             // 11 MooneyRivlin3ParamSymbolic (pfg_set_material)
	const int *conn = nullptr;
	const int *gconn = nullptr;
	const double *X = nullptr;
	const double2 *lame = nullptr;
	const double4 *mpar = nullptr; // per-element parameters of materials 4..6, 9..11 (pfg_set_material_params):
	                               // eight zero-padded values (two double4) per element
	int mterms = 0;                // number of terms of the Ogden formulations (9, 10)
	const double *hooke = nullptr; // materials 7, 8: the full symmetric 6 x 6 Voigt elasticity tensor, row-major
	const int *inc_off = nullptr;
	const int *inc_eb = nullptr;
	const int *eb_inc = nullptr; // [E*n] inverse of inc_eb: incidence index of (e, b)
	const int *ginc_off = nullptr;
	const int *ginc_eb = nullptr;
	const int *g_eb_inc = nullptr; // [E*n_g] inverse of ginc_eb (aliases eb_inc when isoparametric)
	int *err = nullptr; // set to 1 by a kernel whose bounded wait gave up (the context reports it)
	int *work = nullptr; // element counter of the PSD projection's persistent warps (cleared before each launch)
};

// Element Hessian staging: element e's symmetric node blocks (a, b), a <= b, as one
// packed upper triangle of n(n+1)/2 blocks at stage[e * tri_pad(n)], block (a, b)
// at 9 * tri_index(n, a, b) holding H_e(3a+r, 3b+c) at [c][r]; tri_pad rounds the
// 9 n(n+1)/2 values up to a multiple of 8 so that a triangle is whole 32-byte
// sectors in FP32 and FP64 alike.
__host__ __device__ constexpr int tri_index(int n, int a, int b) { return a * n - a * (a - 1) / 2 + (b - a); }
__host__ __device__ constexpr int tri_pad(int n) { return ((9 * (n * (n + 1) / 2) + 7) / 8) * 8; }
constexpr unsigned TRI_TRANSPOSED = 0x80000000u;

// Device-resident Hessian pattern (Eigen ColMajor CSC, int32 indices) and its
// reduction plan.  Node B's column block has deg(B) row nodes (rank 0..deg-1 in
// ascending node order); entry (3A+r, 3B+c) lives at
//   outer[3B] + c*3*deg(B) + 3*rank_B(A) + r,
// and B's node blocks are numbered from outer[3B] / 9.  For node B with
// incidences s0..s1-1 (inc_off), element e holding B at local b:
//   contrib[s0*n + k], k < (s1-s0)*n : the staged block that gives column node B
//       its rows of local row node a, grouped by the rank of a, incidences
//       ascending inside a group: e * tri_pad(n) + 9 * tri_index(n, min(a,b), max(a,b)),
//       with TRI_TRANSPOSED set when a > b (the block is (b, a), read transposed);
//   blk_rel[outer[3B]/9 + rank]     : start of the rank's group, relative to s0*n.
struct DevPattern
{
	long long nnz = 0;
	int max_deg = 0; // largest number of neighbour nodes of a node

	const int *outer = nullptr;
	const int *inner = nullptr;
	const unsigned int *contrib = nullptr;
	const unsigned short *blk_rel = nullptr;
	double *values = nullptr;
	// Dirichlet-reduced output (BCLagrangianForm::project_hessian): when red_col_start
	// is set the reduction writes only entries whose row and column are free, at
	//   values[red_col_start[col] + red_row_off[outer[3B]/3 + 3*rank + r]]
	// (red_col_start < 0: constrained column; red_row_off == 0xFFFF: constrained row)
	const int *red_col_start = nullptr;
	const unsigned short *red_row_off = nullptr;
};

struct Scratch
{
	double *partials = nullptr;       // per-block energy partial sums
	unsigned int *ticket = nullptr;   // last-block-done counter (returns to 0 after each launch)
	unsigned long long *inverted = nullptr;
	int max_blocks = 0;
	double *vec_stage = nullptr;      // one 32-byte slot per incidence, in incidence (node) order: element gradient / shape contributions
	void *hess_stage = nullptr;       // one packed block triangle per element (tri_pad values, FP64 or FP32)
};

constexpr int PREC_FP64 = 0;
constexpr int PREC_FP32 = 1;
constexpr int PREC_SPLIT32 = 2;      // tensor cores (P2, Q1); CUDA cores for P1
constexpr int PREC_SPLIT32_SIMT = 3; // the same split with the contraction on CUDA cores

// Elements per thread block of the total-energy kernel for an element type (the
// number of per-block partial sums is ceil(E / this)).
int energy_elems_per_block(int et);

// All launchers return cudaGetLastError() after enqueueing on `s`.
cudaError_t launch_energy(const DevMesh &m, const double *u, int prec, bool per_element, double *out,
						  const Scratch &sc, cudaStream_t s);
cudaError_t launch_gradient(const DevMesh &m, const double *u, int prec, double *g, const Scratch &sc,
							cudaStream_t s);
// vec_stage must hold E*max(n, n_g)*4 doubles
// project_psd != 0: every element matrix is projected onto the PSD cone (ipc::project_to_psd, CLAMP) before the scatter
cudaError_t launch_hessian(const DevMesh &m, const DevPattern &p, const double *u, int prec, int project_psd,
						   void *stage, cudaStream_t s);
// Mass matrix values (nnz of the Hessian pattern) into p.values; rho = per-element
// density (device, E doubles) or NULL for 1; stage as for the FP64 Hessian
cudaError_t launch_mass(const DevMesh &m, const DevPattern &p, const double *rho, void *stage, cudaStream_t s);
// utils::lump_matrix: diag (3 * n_nodes) = row sums of the values in the Hessian
// pattern (outer, inner), each summed in ascending column order
cudaError_t launch_lump_rows(int n_nodes, const int *outer, const int *inner, const double *vals, double *diag,
							 cudaStream_t s);
// Compositions of formulations (MaterialSum, MultiModels): FP64 pass 1 alone and the
// projection + scatter alone; the gradient's slots alone and their gather; per-element
// and per-slot combination of a component's buffer into the accumulated one (sel:
// component of every element, NULL = all elements; first: start from zero); the
// deterministic sum of an array (Scratch partials and ticket)
cudaError_t launch_fp64_blocks(const DevMesh &m, const double *u, double *stage, cudaStream_t s);
cudaError_t launch_fp64_finish(const DevMesh &m, const DevPattern &p, double *stage, bool project_psd, cudaStream_t s);
cudaError_t launch_gradient_stage(const DevMesh &m, const double *u, const Scratch &sc, cudaStream_t s);
cudaError_t launch_gradient_gather(const DevMesh &m, const double *stage, double *g, cudaStream_t s);
cudaError_t launch_combine_elements(double *acc, const double *src, long long per, int E, const int *sel, int comp,
									bool first, cudaStream_t s);
cudaError_t launch_combine_slots(double *acc, const double *src, long long n_inc, int n, const int *inc_eb, const int *sel,
								 int comp, bool first, cudaStream_t s);
cudaError_t launch_sum_array(const double *x, int n, double *out, const Scratch &sc, cudaStream_t s);
// DenseMatrixCache: the values of the Hessian pattern into a dense column-major
// ndof x ndof array (zeros outside the pattern)
cudaError_t launch_csc_to_dense(int ndof, const int *outer, const int *inner, const double *vals, double *dense,
								cudaStream_t s);
// Dirichlet reduction helpers: dof maps of the free dofs (old_to_new[dof] = index
// among the free dofs or -1, free[i] = dof of the i-th free dof)
cudaError_t launch_gather_free(const double *full, const int *free, int n_free, double *out, cudaStream_t s);
cudaError_t launch_reduced_to_full(const double *y, const double *x_bc, const int *old_to_new, int ndof, double *x,
								   cudaStream_t s);
// Materials from MAT_FIRST_AD on are differentiated automatically (pfg_materials.cu):
// the energy, the element gradients into sc.vec_stage (one slot per incidence, as
// the other gradient kernels), and the FP64 element block triangles into stage.
constexpr int MAT_FIRST_AD = 3;
cudaError_t launch_ad_energy(const DevMesh &m, const double *u, bool per_element, double *out, const Scratch &sc,
							 cudaStream_t s);
cudaError_t launch_ad_gradient_stage(const DevMesh &m, const double *u, const Scratch &sc, cudaStream_t s);
cudaError_t launch_ad_blocks(const DevMesh &m, const double *u, double *stage, cudaStream_t s);
// adjoint terms of the other materials: LinearElasticity's material derivative, and the
// shape derivative's element contributions (one slot per geometric incidence) of
// IsochoricNeoHookean and materials MAT_FIRST_AD.. (SaintVenant has none in the reference)
cudaError_t launch_ad_material_vjp(const DevMesh &m, const double *u, const double *adj, double *out, cudaStream_t s);
cudaError_t launch_ad_shape_vjp_stage(const DevMesh &m, const double *u, const double *adj, const Scratch &sc,
									  cudaStream_t s);
cudaError_t launch_material_vjp(const DevMesh &m, const double *u, const double *adj, double *out, cudaStream_t s);
cudaError_t launch_shape_vjp(const DevMesh &m, const double *u, const double *adj, int prec, double *out,
							 const Scratch &sc, cudaStream_t s);
cudaError_t hessian_kernel_setup(int device);
// Tensor-core element blocks of the split mode (pfg_tc.cu): the Phi tables of the
// current device and the kernels' shared-memory limits (called by hessian_kernel_setup);
// the packed FP32 block triangles of all elements into `stage` (P2 and Q1 only)
cudaError_t tc_tables_setup(int device);
cudaError_t launch_hessian_blocks_tc(const DevMesh &m, const double *u, float *stage, cudaStream_t s);
size_t tc_smem_bytes(int et);

// Device conjugate gradient (pfg_solve.cu).  Work vectors of n doubles (r, z, p, q,
// invd), cg_partials_doubles() per-block partial sums and the scalars sc[CG_NSC].
enum
{
	CG_RZ = 0,    // r.z of the current iterate
	CG_ALPHA = 1, // step length of the last iteration
	CG_BETA = 2,  // direction update factor of the last iteration
	CG_RR = 3,    // |r|^2 of the current iterate
	CG_RHS2 = 4,  // |b|^2
	CG_THR = 5,   // stopping threshold on |r|^2
	CG_DONE = 6,  // 1 once |r|^2 < threshold: every later kernel of the iteration returns at once
	CG_ITER = 7,  // iterations counted as Eigen counts them (not the one that stopped)
	CG_NSC = 8
};
struct CgWork
{
	double *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *invd = nullptr, *part = nullptr, *sc = nullptr;
};
size_t cg_partials_doubles();
// invd[j] = 1 / H(j, j), or 1 where the diagonal is zero or structurally absent
cudaError_t launch_cg_diag_inv(int n, const int *outer, const int *inner, const double *vals, double *invd,
							   cudaStream_t s);
// The SpMV takes the columns in groups of m <= 3 consecutive columns with the same
// rows (a node's dofs): groups[g] = first column * 4 + m, or, with groups == NULL,
// group g = columns 3g .. 3g+2.
// q = H p over the full pattern (a node's three columns share their rows), one warp
// per node, every entry summed in a fixed order (bitwise deterministic)
cudaError_t launch_hessian_apply(int n_nodes, const int *outer, const int *inner, const double *vals, const double *p,
								 double *q, cudaStream_t s);
// r = b - H x (x = 0 unless guess), p = D^-1 r; sc: r.z, |r|^2, |b|^2, the threshold
// max(tol^2 |b|^2, smallest normal), done (|b| = 0 or |r|^2 below it), 0 iterations
cudaError_t launch_cg_start(int n, int ngroups, const int *groups, const int *outer, const int *inner,
							const double *vals, const double *b, bool guess, double tol, double *x, const CgWork &w,
							cudaStream_t s);
// `count` iterations unless done: q = H p, alpha, x += alpha p, r -= alpha q, stop
// test, z = D^-1 r, beta, p = z + beta p, iteration count + 1
cudaError_t launch_cg_iterations(int n, int count, int ngroups, const int *groups, const int *outer,
								 const int *inner, const double *vals, double *x, const CgWork &w, cudaStream_t s);

// Sets the message pfg_last_error(NULL) returns on this host thread.
void set_global_error(const std::string &msg);

// Sparse direct solve (pfg_direct.cu): multifrontal Cholesky of an SPD matrix in a
// CSC pattern.  direct_symbolic analyses a host pattern (0 or a PFG error code),
// direct_upload moves its maps to the device, direct_factorize factorises device
// values (0 ok, 1 not positive definite, 2 CUDA error in *ce), direct_solve
// solves for device vectors (x may alias b).  direct_stats: n, fronts, levels,
// front doubles, entries of L, largest front, flops of the factorisation.
struct DirectFactor;
int direct_symbolic(int n, const int *outer, const int *inner, DirectFactor **out, std::string &msg);
int direct_upload(DirectFactor *f, std::string &msg);
int direct_factorize(DirectFactor *f, const double *vals, cudaStream_t s, cudaError_t *ce);
cudaError_t direct_solve(DirectFactor *f, const double *b, double *x, cudaStream_t s);
void direct_destroy(DirectFactor *f);
void direct_stats(const DirectFactor *f, long long *st);
int direct_n(const DirectFactor *f);
long long direct_nnz(const DirectFactor *f);
bool direct_factorized(const DirectFactor *f);
double *direct_io(DirectFactor *f);

} // namespace pfg
