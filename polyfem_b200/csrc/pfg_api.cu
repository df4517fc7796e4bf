// Host side of the C ABI declared in include/pfgpu.h.
//
// Ownership and lifecycle mirror the reference: the context plays the role of
// ElasticForm (solver/forms/ElasticForm.cpp) holding the AssemblyValsCache
// inputs and the mutable SparseMatrixCache; the pattern and the assembly plan
// (which element incidences feed which CSC column block, and at which row) are
// built once (first pfg_hessian / pfg_hessian_pattern call) and then stay on
// the device, like SparseMatrixCache's mapping_/second_cache_
// (utils/MatrixCache.cpp:134-212).
#include "../../include/pfgpu.h"
#include "pfg_internal.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

using namespace pfg;

struct pfg_context
{
	int device = 0;
	cudaStream_t stream = nullptr;
	int n = 0, ng = 0; // nodes / geometric nodes per element
	DevMesh m;
	// owned device buffers
	int *d_conn = nullptr, *d_gconn = nullptr;
	double *d_X = nullptr;
	double2 *d_lame = nullptr;
	// pattern
	bool has_pattern = false;
	DevPattern pat;
	int *d_outer = nullptr, *d_inner = nullptr;
	double *d_values = nullptr;
	unsigned int *d_contrib = nullptr;
	unsigned short *d_blk_rel = nullptr;
	// Dirichlet reduction (pfg_set_dirichlet)
	bool has_dirichlet = false;
	std::vector<int> h_constrained;      // sorted unique constrained dofs
	int n_free = 0;
	long long red_nnz = 0;
	int *d_old_to_new = nullptr, *d_free = nullptr, *d_red_col_start = nullptr, *d_red_outer = nullptr,
		*d_red_inner = nullptr;
	unsigned short *d_red_row_off = nullptr;
	double *d_red_values = nullptr, *d_full_tmp = nullptr;
	int *d_red_groups = nullptr; // per node with free dofs: first reduced column * 4 + their count
	int n_red_groups = 0;
	int *d_eb_inc = nullptr, *d_g_eb_inc = nullptr;
	// node -> (element, local index) incidences, FE and geometric nodes
	std::vector<long long> h_inc_off; // [N+1]
	std::vector<int> h_inc_e;         // element of each incidence, grouped by node, ascending
	int *d_inc_off = nullptr, *d_inc_eb = nullptr, *d_ginc_off = nullptr, *d_ginc_eb = nullptr;
	// staging buffers (allocated on first use): element contributions / element Hessian blocks
	double *d_vec_stage = nullptr;
	void *d_hess_stage[2] = {nullptr, nullptr}; // [0] FP64, [1] FP32
	std::vector<int> h_conn; // row-major E x n copy for the host pattern build
	// scratch and host-mode staging
	Scratch sc;
	double *d_result = nullptr;
	double *d_u = nullptr, *d_p = nullptr, *d_out = nullptr;
	size_t out_cap = 0;
	// conjugate gradient (pfg_cg_solve): r, z, p, q, invd, b, x (cg_n doubles each),
	// the per-block partials and the scalars; a pinned host copy of the scalars
	double *d_cg = nullptr;
	size_t cg_n = 0;
	// mass matrix (pfg_mass_matrix): values for host-mode calls, staged densities
	double *d_mass = nullptr, *d_rho = nullptr;
	// lumped diagonal for host-mode pfg_lump_matrix calls (3N doubles)
	double *d_lump = nullptr;
	// parameters of the automatically differentiated materials (pfg_set_material_params):
	// eight zero-padded doubles (two double4) per element; n_mpar = the count last set (0: none)
	double4 *d_mpar = nullptr;
	int n_mpar = 0;
	// elasticity tensor of HookeLinearElasticity and the anisotropic SaintVenant
	// (pfg_set_elasticity_tensor): 36 doubles
	double *d_hooke = nullptr;
	double *h_cg_sc = nullptr;
	int *d_err = nullptr; // set by a kernel whose bounded wait gave up (DevMesh::err)
	int *d_work = nullptr; // DevMesh::work
	// compositions of formulations (pfg_set_component / pfg_set_composite): each
	// component's material and parameters; the component of every element (MultiModels)
	// or none (MaterialSum); per-component scratch of the element kernels
	struct Component
	{
		int mat = -1;
		double2 *lame = nullptr; // NULL: the context's Lame parameters
		double4 *mpar = nullptr;
		int n_mpar = 0, terms = 0;
		double *hooke = nullptr;
	};
	Component comps[PFG_MAX_COMPONENTS];
	int n_comps = 0;
	bool composite = false;
	int *d_elem_comp = nullptr;
	double *d_comp_e = nullptr, *d_comp_eacc = nullptr; // per-element energies: one component's, combined
	double *d_comp_vec = nullptr;                       // one component's gradient slots
	double *d_comp_stage = nullptr;                     // one component's FP64 block triangles
	unsigned long long *d_comp_inverted = nullptr;      // inverted counts of components after the first
	// sparse direct solve (pfg_direct_*): the analysed (and factorised) system
	pfg::DirectFactor *direct = nullptr;
	int direct_system = -1;
	std::string err;
};

static thread_local std::string g_create_error;

void pfg::set_global_error(const std::string &msg) { g_create_error = msg; }

namespace
{
int fail(pfg_context *c, int status, const std::string &msg)
{
	if (c)
		c->err = msg;
	else
		g_create_error = msg;
	return status;
}

int cuda_fail(pfg_context *c, cudaError_t e, const char *where)
{
	const int st = (e == cudaErrorMemoryAllocation) ? PFG_ERR_OOM : PFG_ERR_CUDA;
	return fail(c, st, std::string(where) + ": " + cudaGetErrorString(e));
}

#define PFG_CUDA(c, call)                                   \
	do                                                      \
	{                                                       \
		cudaError_t e_ = (call);                            \
		if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
	} while (0)

struct DeviceGuard
{
	int prev = -1;
	explicit DeviceGuard(int dev)
	{
		cudaGetDevice(&prev);
		if (prev != dev) cudaSetDevice(dev);
	}
	~DeviceGuard()
	{
		int cur = -1;
		cudaGetDevice(&cur);
		if (prev >= 0 && cur != prev) cudaSetDevice(prev);
	}
};

int nodes_per_element(int et) { return et == PFG_P1_TET ? 4 : et == PFG_P2_TET ? 10 : et == PFG_Q1_HEX ? 8 : 0; }
int geom_nodes_per_element(int et) { return et == PFG_P1_TET ? 4 : et == PFG_P2_TET ? 4 : et == PFG_Q1_HEX ? 8 : 0; }

template <class F>
void parallel_ranges(long long n, F &&f)
{
	int nt = (int)std::min<long long>(std::max(1u, std::thread::hardware_concurrency()), 32);
	if (n < 4096) nt = 1;
	if (nt <= 1)
	{
		f(0LL, n, 0);
		return;
	}
	std::vector<std::thread> th;
	for (int t = 0; t < nt; ++t)
		th.emplace_back([&, t] { f(n * t / nt, n * (t + 1) / nt, t); });
	for (auto &x : th) x.join();
}

int check_mem(int mem) { return mem == PFG_MEM_HOST || mem == PFG_MEM_DEVICE; }
// Whether a material takes pfg_set_material_params parameters, and whether n of them
// fit it; for the Ogden formulations also the number of terms n gives.
bool material_takes_params(int mat)
{
	return mat == PFG_MAT_MOONEY_RIVLIN || mat == PFG_MAT_MOONEY_RIVLIN_3PARAM || mat == PFG_MAT_VOLUME_PENALTY ||
		   mat == PFG_MAT_UNCONSTRAINED_OGDEN || mat == PFG_MAT_INCOMPRESSIBLE_OGDEN ||
		   mat == PFG_MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC;
}
bool material_params_fit(int mat, int n, int *terms)
{
	*terms = 0;
	switch (mat)
	{
	case PFG_MAT_MOONEY_RIVLIN: return n == 3;
	case PFG_MAT_MOONEY_RIVLIN_3PARAM:
	case PFG_MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC: return n == 4;
	case PFG_MAT_VOLUME_PENALTY: return n == 1;
	case PFG_MAT_UNCONSTRAINED_OGDEN: // alphas, mus, Ds: three per term
		*terms = n / 3;
		return n == 3 || n == 6;
	case PFG_MAT_INCOMPRESSIBLE_OGDEN: // cs, ms: two per term, then k
		*terms = (n - 1) / 2;
		return n == 3 || n == 5 || n == 7;
	default: return true;
	}
}
// The other materials (pfg_set_material) are assembled in FP64 only, and the
// parameterised ones need their parameters.
int check_material_prec(pfg_context *c, int prec)
{
	if (c->composite)
		return prec == PFG_FP64 ? PFG_OK
								: fail(c, PFG_ERR_UNSUPPORTED, "compositions of formulations are assembled in PFG_FP64 only");
	if (c->m.mat != PFG_MAT_NEOHOOKEAN && prec != PFG_FP64)
		return fail(c, PFG_ERR_UNSUPPORTED, "only PFG_FP64 is implemented for materials other than NeoHookean");
	int terms = 0;
	if (material_takes_params(c->m.mat) && c->m.E && !(c->n_mpar > 0 && material_params_fit(c->m.mat, c->n_mpar, &terms)))
		return fail(c, PFG_ERR_STATE, "the material's parameters are not set (pfg_set_material_params)");
	c->m.mterms = terms;
	if ((c->m.mat == PFG_MAT_HOOKE || c->m.mat == PFG_MAT_SAINT_VENANT_TENSOR) && !c->d_hooke)
		return fail(c, PFG_ERR_STATE, "the elasticity tensor is not set (pfg_set_elasticity_tensor)");
	return PFG_OK;
}
int check_prec(int prec) { return prec == PFG_FP64 || prec == PFG_FP32 || prec == PFG_SPLIT32 || prec == PFG_SPLIT32_SIMT; }

int ensure_staging(pfg_context *c, size_t out_doubles)
{
	const size_t ndof = 3 * (size_t)c->m.N;
	if (!c->d_u)
	{
		PFG_CUDA(c, cudaMalloc(&c->d_u, std::max<size_t>(ndof, 1) * sizeof(double)));
		PFG_CUDA(c, cudaMalloc(&c->d_p, std::max<size_t>(ndof, 1) * sizeof(double)));
	}
	if (out_doubles > c->out_cap)
	{
		if (c->d_out) cudaFree(c->d_out);
		c->d_out = nullptr;
		c->out_cap = 0;
		PFG_CUDA(c, cudaMalloc(&c->d_out, out_doubles * sizeof(double)));
		c->out_cap = out_doubles;
	}
	return PFG_OK;
}

// Element-contribution staging of the gradient / shape term (first use allocates).
int ensure_vec_stage(pfg_context *c)
{
	if (!c->d_vec_stage)
	{
		const size_t n = (size_t)std::max(c->m.E, 1) * std::max(c->n, c->ng) * 4;
		PFG_CUDA(c, cudaMalloc(&c->d_vec_stage, n * sizeof(double)));
	}
	c->sc.vec_stage = c->d_vec_stage;
	return PFG_OK;
}

// Element-block staging of the Hessian for one precision (first use allocates).
int ensure_hess_stage(pfg_context *c, int prec)
{
	const int k = prec == PFG_FP64 ? 0 : 1;
	if (!c->d_hess_stage[k])
	{
		const size_t tsz = k == 0 ? sizeof(double) : sizeof(float);
		const size_t n = (size_t)std::max(c->m.E, 1) * tri_pad(c->n) * tsz; // one block triangle per element
		PFG_CUDA(c, cudaMalloc(&c->d_hess_stage[k], n));
	}
	return PFG_OK;
}

// Stage a host input vector of 3N doubles into `dst`; device inputs are used in place.
int stage_in(pfg_context *c, const double *src, int mem, double *dst, size_t n, const double **use)
{
	if (mem == PFG_MEM_DEVICE)
	{
		*use = src;
		return PFG_OK;
	}
	if (n) PFG_CUDA(c, cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
	*use = dst;
	return PFG_OK;
}

// After a stream synchronisation: a kernel that gave up a bounded wait left the
// flag set; report it once and clear it.
int check_kernel_flag(pfg_context *c)
{
	int v = 0;
	PFG_CUDA(c, cudaMemcpy(&v, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
	if (v)
	{
		PFG_CUDA(c, cudaMemset(c->d_err, 0, sizeof(int)));
		return fail(c, PFG_ERR_CUDA, "a tensor-core kernel gave up waiting for its MMA or bulk copy; the results of "
									 "the calls since the last synchronisation are invalid");
	}
	return PFG_OK;
}

int finish_host(pfg_context *c, double *host_dst, const double *dev_src, size_t n)
{
	if (n) PFG_CUDA(c, cudaMemcpyAsync(host_dst, dev_src, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
	PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	return check_kernel_flag(c);
}

// Host build of the CSC pattern (Eigen ColMajor semantics: per column the sorted
// unique rows touched by any element) and the node-owner assembly plans.
int build_pattern(pfg_context *c)
{
	const int N = c->m.N, n = c->n;
	const int *conn = c->h_conn.data();
	const std::vector<long long> &ioff = c->h_inc_off;
	const std::vector<int> &inc = c->h_inc_e;
	// neighbours of every node, sorted and unique, built in parallel node ranges
	std::vector<int> deg(N, 0);
	const int nt_max = 64;
	std::vector<std::vector<int>> part(nt_max);
	std::vector<long long> part_begin(nt_max, 0), part_end(nt_max, 0);
	int used_threads = 0;
	parallel_ranges(N, [&](long long s, long long e, int t) {
		std::vector<int> tmp;
		auto &out = part[t];
		part_begin[t] = s;
		part_end[t] = e;
		for (long long B = s; B < e; ++B)
		{
			tmp.clear();
			for (long long k = ioff[B]; k < ioff[B + 1]; ++k)
			{
				const int el = inc[k];
				for (int a = 0; a < n; ++a) tmp.push_back(conn[(size_t)el * n + a]);
			}
			std::sort(tmp.begin(), tmp.end());
			tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
			deg[B] = (int)tmp.size();
			out.insert(out.end(), tmp.begin(), tmp.end());
		}
	});
	for (int t = 0; t < nt_max; ++t)
		if (part_end[t] > part_begin[t]) used_threads = t + 1;
	std::vector<long long> noff(N + 1, 0);
	for (int i = 0; i < N; ++i) noff[i + 1] = noff[i] + deg[i];
	std::vector<int> nbr(noff[N]);
	for (int t = 0; t < used_threads; ++t)
		if (!part[t].empty()) std::copy(part[t].begin(), part[t].end(), nbr.begin() + noff[part_begin[t]]);
	part.clear();

	const long long nnz = 9 * noff[N];
	if (nnz > 0x7fffffffLL) return fail(c, PFG_ERR_UNSUPPORTED, "Hessian has more than 2^31-1 nonzeros (int32 CSC)");
	int max_deg = 0;
	for (int B = 0; B < N; ++B) max_deg = std::max(max_deg, deg[B]);
	if (max_deg > 65535) return fail(c, PFG_ERR_UNSUPPORTED, "a node has more than 65535 neighbours");
	const int ndof = 3 * N;
	std::vector<int> outer(ndof + 1);
	{
		long long base = 0;
		for (int B = 0; B < N; ++B)
		{
			for (int cc = 0; cc < 3; ++cc) outer[3 * B + cc] = (int)(base + (long long)cc * 3 * deg[B]);
			base += 9LL * deg[B];
		}
		outer[ndof] = (int)base;
	}
	std::vector<int> inner(nnz);
	parallel_ranges(N, [&](long long s, long long e, int) {
		for (long long B = s; B < e; ++B)
			for (int cc = 0; cc < 3; ++cc)
			{
				long long o = outer[3 * B + cc];
				for (long long k = noff[B]; k < noff[B + 1]; ++k)
					for (int m = 0; m < 3; ++m) inner[o++] = 3 * nbr[k] + m;
			}
	});
	// row rank of every (incidence, local row node)
	const long long nstrip = ioff[N];
	std::vector<unsigned short> strip_rank((size_t)nstrip * n);
	parallel_ranges(N, [&](long long s0, long long s1, int) {
		for (long long B = s0; B < s1; ++B)
		{
			const int *lo = nbr.data() + noff[B], *hi = nbr.data() + noff[B + 1];
			for (long long k = ioff[B]; k < ioff[B + 1]; ++k)
			{
				const int *ce = conn + (size_t)inc[k] * n;
				for (int a = 0; a < n; ++a)
					strip_rank[(size_t)k * n + a] = (unsigned short)(std::lower_bound(lo, hi, ce[a]) - lo);
			}
		}
	});

	// Reduction plan of every column node B (the device form of SparseMatrixCache's
	// second_cache_): its n * (#incidences) element blocks, grouped by the row rank
	// they land on, incidences ascending inside a group.  contrib holds each block
	// as its offset in the staged block triangles (transposed flag for a > b);
	// blk_rel[block] is where the block's group starts, relative to B's first
	// contribution, in 16 bits while a node has at most 65535 / n incidences.
	long long max_tot = 0;
	for (int B = 0; B < N; ++B) max_tot = std::max(max_tot, (ioff[B + 1] - ioff[B]) * n);
	if (max_tot > 65535)
		return fail(c, PFG_ERR_UNSUPPORTED,
					"a node has more than 65535 incident (element, local node) pairs; the 16-bit reduction plan cannot hold it");
	const long long tp = tri_pad(n);
	if ((long long)c->m.E * tp > 0x7fffffffLL)
		return fail(c, PFG_ERR_UNSUPPORTED, "E * (9 n(n+1)/2, padded) staged block values exceed 2^31-1 (31-bit plan offsets)");
	std::vector<unsigned int> contrib((size_t)nstrip * n);
	std::vector<unsigned short> blk_rel((size_t)noff[N]);
	parallel_ranges(N, [&](long long s0, long long s1, int) {
		std::vector<int> pos;
		for (long long B = s0; B < s1; ++B)
		{
			const int d = deg[B];
			pos.assign(d + 1, 0);
			const long long k0 = ioff[B], k1 = ioff[B + 1];
			for (long long k = k0; k < k1; ++k)
				for (int a = 0; a < n; ++a) pos[strip_rank[(size_t)k * n + a] + 1]++;
			for (int r = 0; r < d; ++r) pos[r + 1] += pos[r];
			for (int r = 0; r < d; ++r) blk_rel[noff[B] + r] = (unsigned short)pos[r];
			unsigned int *cb = contrib.data() + (size_t)k0 * n;
			for (long long k = k0; k < k1; ++k)
			{
				const int el = inc[k];
				const int *ce = conn + (size_t)el * n;
				int b = 0;
				while (ce[b] != B) ++b;
				for (int a = 0; a < n; ++a)
				{
					const unsigned blk = (unsigned)(el * tp + 9 * tri_index(n, std::min(a, b), std::max(a, b)));
					cb[pos[strip_rank[(size_t)k * n + a]]++] = a > b ? (blk | TRI_TRANSPOSED) : blk;
				}
			}
		}
	});

	PFG_CUDA(c, cudaMalloc(&c->d_outer, sizeof(int) * (ndof + 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_inner, sizeof(int) * std::max<long long>(nnz, 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_values, sizeof(double) * std::max<long long>(nnz, 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_contrib, sizeof(unsigned int) * std::max<size_t>(contrib.size(), 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_blk_rel, sizeof(unsigned short) * std::max<size_t>(blk_rel.size(), 1)));
	PFG_CUDA(c, cudaMemcpy(c->d_outer, outer.data(), sizeof(int) * (ndof + 1), cudaMemcpyHostToDevice));
	if (nnz) PFG_CUDA(c, cudaMemcpy(c->d_inner, inner.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice));
	if (!contrib.empty())
		PFG_CUDA(c, cudaMemcpy(c->d_contrib, contrib.data(), sizeof(unsigned int) * contrib.size(),
							   cudaMemcpyHostToDevice));
	if (!blk_rel.empty())
		PFG_CUDA(c, cudaMemcpy(c->d_blk_rel, blk_rel.data(), sizeof(unsigned short) * blk_rel.size(),
							   cudaMemcpyHostToDevice));
	c->pat.nnz = nnz;
	c->pat.max_deg = max_deg;
	c->pat.outer = c->d_outer;
	c->pat.inner = c->d_inner;
	c->pat.contrib = c->d_contrib;
	c->pat.blk_rel = c->d_blk_rel;
	c->pat.values = c->d_values;
	c->has_pattern = true;
	return PFG_OK;
}

// node -> incidence lists (grouped by node, elements ascending) of a connectivity
void build_incidence(const int *conn, int E, int n, int N, std::vector<long long> &off, std::vector<int> &elem,
					 std::vector<int> &eb)
{
	off.assign(N + 1, 0);
	for (long long i = 0; i < (long long)E * n; ++i) off[conn[i] + 1]++;
	for (int i = 0; i < N; ++i) off[i + 1] += off[i];
	elem.assign(off[N], 0);
	eb.assign(off[N], 0);
	std::vector<long long> pos(off.begin(), off.end() - 1);
	for (int e = 0; e < E; ++e)
		for (int a = 0; a < n; ++a)
		{
			const long long k = pos[conn[(size_t)e * n + a]]++;
			elem[k] = e;
			eb[k] = e * n + a;
		}
}

void free_direct(pfg_context *c)
{
	direct_destroy(c->direct);
	c->direct = nullptr;
	c->direct_system = -1;
}

void free_dirichlet(pfg_context *c)
{
	if (c->direct_system == PFG_SYS_REDUCED) free_direct(c);
	void *rptrs[] = {c->d_old_to_new, c->d_free, c->d_red_col_start, c->d_red_outer, c->d_red_inner, c->d_red_row_off,
					 c->d_red_values, c->d_red_groups};
	for (void *p : rptrs)
		if (p) cudaFree(p);
	c->d_old_to_new = c->d_free = c->d_red_col_start = c->d_red_outer = c->d_red_inner = nullptr;
	c->d_red_row_off = nullptr;
	c->d_red_values = nullptr;
	c->d_red_groups = nullptr;
	c->n_red_groups = 0;
	c->has_dirichlet = false;
	c->n_free = 0;
	c->red_nnz = 0;
}

// Reduced pattern of BCLagrangianForm::project_hessian (BCLagrangianForm.cpp:165-212):
// constrained rows and columns dropped, free dofs renumbered in ascending order
// (old_to_new), each column keeping its free rows in ascending order.  Because a
// node's three columns share one row set, the position of a kept row inside its
// column is one 16-bit offset per (node, row slot).
int build_dirichlet(pfg_context *c)
{
	const int N = c->m.N, ndof = 3 * N;
	std::vector<int> old_to_new(ndof, 0), freev;
	for (int d : c->h_constrained) old_to_new[d] = -1;
	freev.reserve(ndof);
	for (int i = 0; i < ndof; ++i)
		if (old_to_new[i] == 0)
		{
			old_to_new[i] = (int)freev.size();
			freev.push_back(i);
		}
		else
			old_to_new[i] = -1;
	const int n_free = (int)freev.size();
	std::vector<int> outer(ndof + 1), inner((size_t)c->pat.nnz);
	PFG_CUDA(c, cudaMemcpy(outer.data(), c->d_outer, sizeof(int) * (ndof + 1), cudaMemcpyDeviceToHost));
	if (c->pat.nnz) PFG_CUDA(c, cudaMemcpy(inner.data(), c->d_inner, sizeof(int) * c->pat.nnz, cudaMemcpyDeviceToHost));
	// row offsets per (node, row slot) and kept rows per node
	std::vector<unsigned short> row_off((size_t)c->pat.nnz / 3);
	std::vector<int> kept(N, 0);
	for (int B = 0; B < N; ++B)
	{
		const int o0 = outer[3 * B], len = outer[3 * B + 1] - o0; // 3 * deg rows
		int k = 0;
		for (int j = 0; j < len; ++j)
			row_off[(size_t)o0 / 3 + j] = old_to_new[inner[(size_t)o0 + j]] >= 0 ? (unsigned short)k++ : (unsigned short)0xFFFF;
		kept[B] = k;
	}
	std::vector<int> col_start(ndof, -1), red_outer(n_free + 1, 0);
	long long pos = 0;
	for (int i = 0; i < n_free; ++i)
	{
		const int col = freev[i];
		if (pos > 0x7fffffffLL) return fail(c, PFG_ERR_UNSUPPORTED, "reduced Hessian has more than 2^31-1 nonzeros");
		col_start[col] = (int)pos;
		red_outer[i] = (int)pos;
		pos += kept[col / 3];
	}
	red_outer[n_free] = (int)pos;
	std::vector<int> red_inner((size_t)pos);
	for (int i = 0; i < n_free; ++i)
	{
		const int col = freev[i], B = col / 3, o0 = outer[3 * B], len = outer[3 * B + 1] - o0;
		long long q = red_outer[i];
		for (int j = 0; j < len; ++j)
		{
			const int r = old_to_new[inner[(size_t)o0 + j]];
			if (r >= 0) red_inner[(size_t)q++] = r;
		}
	}
	// column groups of the conjugate gradient's SpMV: the free dofs of a node are
	// consecutive reduced columns with the same rows
	std::vector<int> groups;
	for (int B = 0; B < N; ++B)
	{
		int m = 0, c0 = -1;
		for (int d = 0; d < 3; ++d)
			if (old_to_new[3 * B + d] >= 0)
			{
				if (c0 < 0) c0 = old_to_new[3 * B + d];
				++m;
			}
		if (m) groups.push_back(c0 * 4 + m);
	}
	free_dirichlet(c);
	PFG_CUDA(c, cudaMalloc(&c->d_red_groups, sizeof(int) * std::max<size_t>(groups.size(), 1)));
	if (!groups.empty())
		PFG_CUDA(c, cudaMemcpy(c->d_red_groups, groups.data(), sizeof(int) * groups.size(), cudaMemcpyHostToDevice));
	c->n_red_groups = (int)groups.size();
	PFG_CUDA(c, cudaMalloc(&c->d_old_to_new, sizeof(int) * std::max(ndof, 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_free, sizeof(int) * std::max(n_free, 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_red_col_start, sizeof(int) * std::max(ndof, 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_red_outer, sizeof(int) * (n_free + 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_red_inner, sizeof(int) * std::max<long long>(pos, 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_red_row_off, sizeof(unsigned short) * std::max<size_t>(row_off.size(), 1)));
	PFG_CUDA(c, cudaMalloc(&c->d_red_values, sizeof(double) * std::max<long long>(pos, 1)));
	PFG_CUDA(c, cudaMemcpy(c->d_old_to_new, old_to_new.data(), sizeof(int) * ndof, cudaMemcpyHostToDevice));
	if (n_free) PFG_CUDA(c, cudaMemcpy(c->d_free, freev.data(), sizeof(int) * n_free, cudaMemcpyHostToDevice));
	PFG_CUDA(c, cudaMemcpy(c->d_red_col_start, col_start.data(), sizeof(int) * ndof, cudaMemcpyHostToDevice));
	PFG_CUDA(c, cudaMemcpy(c->d_red_outer, red_outer.data(), sizeof(int) * (n_free + 1), cudaMemcpyHostToDevice));
	if (pos) PFG_CUDA(c, cudaMemcpy(c->d_red_inner, red_inner.data(), sizeof(int) * pos, cudaMemcpyHostToDevice));
	if (!row_off.empty())
		PFG_CUDA(c, cudaMemcpy(c->d_red_row_off, row_off.data(), sizeof(unsigned short) * row_off.size(), cudaMemcpyHostToDevice));
	c->n_free = n_free;
	c->red_nnz = pos;
	c->has_dirichlet = true;
	return PFG_OK;
}

// the DevMesh of component k: the context's mesh with the component's material
DevMesh component_mesh(const pfg_context *c, int k)
{
	DevMesh mk = c->m;
	const auto &comp = c->comps[k];
	mk.mat = comp.mat;
	if (comp.lame) mk.lame = comp.lame;
	mk.mpar = comp.mpar;
	mk.mterms = comp.terms;
	mk.hooke = comp.hooke;
	return mk;
}

int ensure_composite_scratch(pfg_context *c, bool energy, bool gradient, bool hessian)
{
	const size_t E = std::max(c->m.E, 1);
	if (!c->d_comp_inverted) PFG_CUDA(c, cudaMalloc(&c->d_comp_inverted, sizeof(unsigned long long)));
	if (energy && !c->d_comp_e)
	{
		PFG_CUDA(c, cudaMalloc(&c->d_comp_e, sizeof(double) * E));
		PFG_CUDA(c, cudaMalloc(&c->d_comp_eacc, sizeof(double) * E));
	}
	if (gradient && !c->d_comp_vec)
		PFG_CUDA(c, cudaMalloc(&c->d_comp_vec, sizeof(double) * E * std::max(c->n, c->ng) * 4));
	if (hessian && !c->d_comp_stage) PFG_CUDA(c, cudaMalloc(&c->d_comp_stage, sizeof(double) * E * tri_pad(c->n)));
	return PFG_OK;
}

// Scratch of component k: components after the first count their inverted elements
// elsewhere (every component evaluates every element)
Scratch component_scratch(const pfg_context *c, int k)
{
	Scratch sk = c->sc;
	if (k > 0) sk.inverted = c->d_comp_inverted;
	return sk;
}

// composite energies: per element (per_element) or their deterministic total, into dst
int composite_energy(pfg_context *c, const double *du, bool per_element, double *dst)
{
	int st;
	if ((st = ensure_composite_scratch(c, true, false, false))) return st;
	double *acc = per_element ? dst : c->d_comp_eacc;
	for (int k = 0; k < c->n_comps; ++k)
	{
		PFG_CUDA(c, launch_energy(component_mesh(c, k), du, PFG_FP64, true, c->d_comp_e, component_scratch(c, k), c->stream));
		PFG_CUDA(c, launch_combine_elements(acc, c->d_comp_e, 1, c->m.E, c->d_elem_comp, k, k == 0, c->stream));
	}
	if (!per_element) PFG_CUDA(c, launch_sum_array(acc, c->m.E, dst, c->sc, c->stream));
	return PFG_OK;
}

// composite gradient (3N) into dst
int composite_gradient(pfg_context *c, const double *du, double *dst)
{
	int st;
	if ((st = ensure_composite_scratch(c, false, true, false))) return st;
	const long long n_inc = (long long)c->m.E * c->n;
	for (int k = 0; k < c->n_comps; ++k)
	{
		Scratch sk = component_scratch(c, k);
		sk.vec_stage = c->d_comp_vec;
		PFG_CUDA(c, launch_gradient_stage(component_mesh(c, k), du, sk, c->stream));
		PFG_CUDA(c, launch_combine_slots(c->d_vec_stage, c->d_comp_vec, n_inc, c->n, c->m.inc_eb, c->d_elem_comp, k, k == 0,
										 c->stream));
	}
	PFG_CUDA(c, launch_gradient_gather(c->m, c->d_vec_stage, dst, c->stream));
	return PFG_OK;
}

// composite Hessian into the pattern p: every component's FP64 block triangles combined
// per element, then projected (optionally) and scattered
int composite_hessian(pfg_context *c, const DevPattern &p, const double *du, int project_psd)
{
	int st;
	if ((st = ensure_composite_scratch(c, false, false, true))) return st;
	double *acc = static_cast<double *>(c->d_hess_stage[0]);
	for (int k = 0; k < c->n_comps; ++k)
	{
		PFG_CUDA(c, launch_fp64_blocks(component_mesh(c, k), du, c->d_comp_stage, c->stream));
		PFG_CUDA(c, launch_combine_elements(acc, c->d_comp_stage, tri_pad(c->n), c->m.E, c->d_elem_comp, k, k == 0, c->stream));
	}
	PFG_CUDA(c, launch_fp64_finish(c->m, p, acc, project_psd != 0, c->stream));
	return PFG_OK;
}

void free_all(pfg_context *c)
{
	void *ptrs[] = {c->d_conn, c->d_gconn, c->d_X, c->d_lame, c->d_outer, c->d_inner, c->d_values, c->d_contrib, c->d_blk_rel, c->d_eb_inc, c->d_g_eb_inc,
					c->d_inc_off, c->d_inc_eb, c->d_ginc_off, c->d_ginc_eb, c->d_vec_stage, c->d_hess_stage[0],
					c->d_hess_stage[1], c->sc.partials, c->sc.ticket, c->sc.inverted, c->d_result, c->d_u, c->d_p, c->d_out};
	for (void *p : ptrs)
		if (p) cudaFree(p);
	void *rptrs[] = {c->d_old_to_new, c->d_free, c->d_red_col_start, c->d_red_outer, c->d_red_inner, c->d_red_row_off,
					 c->d_red_values, c->d_full_tmp, c->d_red_groups};
	for (void *p : rptrs)
		if (p) cudaFree(p);
	if (c->d_cg) cudaFree(c->d_cg);
	free_direct(c);
	if (c->h_cg_sc) cudaFreeHost(c->h_cg_sc);
	if (c->d_mass) cudaFree(c->d_mass);
	if (c->d_lump) cudaFree(c->d_lump);
	if (c->d_hooke) cudaFree(c->d_hooke);
	if (c->d_rho) cudaFree(c->d_rho);
	if (c->d_mpar) cudaFree(c->d_mpar);
	if (c->d_err) cudaFree(c->d_err);
	if (c->d_work) cudaFree(c->d_work);
	for (auto &k : c->comps)
	{
		if (k.lame) cudaFree(k.lame);
		if (k.mpar) cudaFree(k.mpar);
		if (k.hooke) cudaFree(k.hooke);
	}
	void *cptrs[] = {c->d_elem_comp, c->d_comp_e, c->d_comp_eacc, c->d_comp_vec, c->d_comp_stage, c->d_comp_inverted};
	for (void *p : cptrs)
		if (p) cudaFree(p);
}
} // namespace

extern "C" {

int pfg_version(void) { return 100; }

const char *pfg_status_string(int s)
{
	switch (s)
	{
	case PFG_OK: return "ok";
	case PFG_ERR_INVALID: return "invalid argument";
	case PFG_ERR_CUDA: return "CUDA error";
	case PFG_ERR_OOM: return "out of memory";
	case PFG_ERR_UNSUPPORTED: return "unsupported";
	case PFG_ERR_STATE: return "invalid state";
	case PFG_ERR_NUMERIC: return "matrix not positive definite";
	}
	return "unknown status";
}

const char *pfg_last_error(const pfg_context *c) { return c ? c->err.c_str() : g_create_error.c_str(); }

int pfg_create(const pfg_mesh_desc *d, pfg_context **out)
{
	if (!out) return fail(nullptr, PFG_ERR_INVALID, "out is NULL");
	*out = nullptr;
	if (!d) return fail(nullptr, PFG_ERR_INVALID, "desc is NULL");
	const int n = nodes_per_element(d->elem_type), ng = geom_nodes_per_element(d->elem_type);
	if (!n) return fail(nullptr, PFG_ERR_INVALID, "unknown elem_type");
	if (d->n_elements < 0 || d->n_nodes < 0 || d->n_geom_nodes < 0) return fail(nullptr, PFG_ERR_INVALID, "negative size");
	if ((long long)d->n_nodes * 3 > 0x7fffffffLL) return fail(nullptr, PFG_ERR_UNSUPPORTED, "too many nodes");
	if (d->n_elements > 0 && (!d->conn || !d->X || !d->lambda || !d->mu))
		return fail(nullptr, PFG_ERR_INVALID, "conn, X, lambda and mu are required");
	const int *gconn = d->gconn ? d->gconn : d->conn;
	if (!d->gconn && ng != n) return fail(nullptr, PFG_ERR_INVALID, "gconn is required for non-isoparametric elements");
	const size_t E = (size_t)d->n_elements;
	for (size_t i = 0; i < E * n; ++i)
		if (d->conn[i] < 0 || d->conn[i] >= d->n_nodes)
			return fail(nullptr, PFG_ERR_INVALID, "conn[" + std::to_string(i) + "] = " + std::to_string(d->conn[i]) + " out of range");
	for (size_t i = 0; i < E * ng; ++i)
		if (gconn[i] < 0 || gconn[i] >= d->n_geom_nodes)
			return fail(nullptr, PFG_ERR_INVALID, "gconn[" + std::to_string(i) + "] out of range");
	int ndev = 0;
	cudaError_t ce = cudaGetDeviceCount(&ndev);
	if (ce != cudaSuccess) return fail(nullptr, PFG_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(ce));
	if (d->device < 0 || d->device >= ndev) return fail(nullptr, PFG_ERR_INVALID, "bad device ordinal");

	DeviceGuard g(d->device);
	auto *c = new pfg_context();
	c->device = d->device;
	c->n = n;
	c->ng = ng;
	c->m.et = d->elem_type;
	c->m.E = d->n_elements;
	c->m.N = d->n_nodes;
	c->m.Ng = d->n_geom_nodes;
	c->h_conn.assign(d->conn, d->conn + E * n);

	auto bail = [&](int st) {
		g_create_error = c->err;
		free_all(c);
		delete c;
		return st;
	};
#define CREATE_CUDA(call)                                 \
	do                                                    \
	{                                                     \
		cudaError_t e_ = (call);                          \
		if (e_ != cudaSuccess) return bail(cuda_fail(c, e_, #call)); \
	} while (0)

	// structure-of-arrays connectivity
	{
		std::vector<int> soa(E * n);
		for (size_t e = 0; e < E; ++e)
			for (int a = 0; a < n; ++a) soa[(size_t)a * E + e] = d->conn[e * n + a];
		CREATE_CUDA(cudaMalloc(&c->d_conn, sizeof(int) * std::max<size_t>(soa.size(), 1)));
		if (!soa.empty()) CREATE_CUDA(cudaMemcpy(c->d_conn, soa.data(), sizeof(int) * soa.size(), cudaMemcpyHostToDevice));
	}
	if (d->gconn && (d->gconn != d->conn || ng != n))
	{
		std::vector<int> soa(E * ng);
		for (size_t e = 0; e < E; ++e)
			for (int a = 0; a < ng; ++a) soa[(size_t)a * E + e] = gconn[e * ng + a];
		CREATE_CUDA(cudaMalloc(&c->d_gconn, sizeof(int) * std::max<size_t>(soa.size(), 1)));
		if (!soa.empty()) CREATE_CUDA(cudaMemcpy(c->d_gconn, soa.data(), sizeof(int) * soa.size(), cudaMemcpyHostToDevice));
	}
	CREATE_CUDA(cudaMalloc(&c->d_X, sizeof(double) * 3 * std::max(d->n_geom_nodes, 1)));
	if (d->n_geom_nodes)
		CREATE_CUDA(cudaMemcpy(c->d_X, d->X, sizeof(double) * 3 * d->n_geom_nodes, cudaMemcpyHostToDevice));
	{
		std::vector<double2> lm(std::max<size_t>(E, 1));
		for (size_t e = 0; e < E; ++e) lm[e] = make_double2(d->lambda[e], d->mu[e]);
		CREATE_CUDA(cudaMalloc(&c->d_lame, sizeof(double2) * lm.size()));
		CREATE_CUDA(cudaMemcpy(c->d_lame, lm.data(), sizeof(double2) * lm.size(), cudaMemcpyHostToDevice));
	}
	// node -> incidence lists for the deterministic per-node sums
	if ((long long)E * n > 0x7fffffffLL) return bail(fail(c, PFG_ERR_UNSUPPORTED, "E * n exceeds 2^31-1"));
	{
		std::vector<int> eb;
		build_incidence(d->conn, (int)E, n, d->n_nodes, c->h_inc_off, c->h_inc_e, eb);
		std::vector<int> off32(c->h_inc_off.begin(), c->h_inc_off.end());
		CREATE_CUDA(cudaMalloc(&c->d_inc_off, sizeof(int) * off32.size()));
		CREATE_CUDA(cudaMalloc(&c->d_inc_eb, sizeof(int) * std::max<size_t>(eb.size(), 1)));
		CREATE_CUDA(cudaMemcpy(c->d_inc_off, off32.data(), sizeof(int) * off32.size(), cudaMemcpyHostToDevice));
		if (!eb.empty()) CREATE_CUDA(cudaMemcpy(c->d_inc_eb, eb.data(), sizeof(int) * eb.size(), cudaMemcpyHostToDevice));
		std::vector<int> inv(eb.size());
		for (size_t k = 0; k < eb.size(); ++k) inv[eb[k]] = (int)k;
		CREATE_CUDA(cudaMalloc(&c->d_eb_inc, sizeof(int) * std::max<size_t>(inv.size(), 1)));
		if (!inv.empty()) CREATE_CUDA(cudaMemcpy(c->d_eb_inc, inv.data(), sizeof(int) * inv.size(), cudaMemcpyHostToDevice));
		if (d->gconn && (d->gconn != d->conn || ng != n))
		{
			std::vector<long long> goff;
			std::vector<int> gelem, geb;
			build_incidence(gconn, (int)E, ng, d->n_geom_nodes, goff, gelem, geb);
			std::vector<int> goff32(goff.begin(), goff.end());
			CREATE_CUDA(cudaMalloc(&c->d_ginc_off, sizeof(int) * goff32.size()));
			CREATE_CUDA(cudaMalloc(&c->d_ginc_eb, sizeof(int) * std::max<size_t>(geb.size(), 1)));
			CREATE_CUDA(cudaMemcpy(c->d_ginc_off, goff32.data(), sizeof(int) * goff32.size(), cudaMemcpyHostToDevice));
			if (!geb.empty()) CREATE_CUDA(cudaMemcpy(c->d_ginc_eb, geb.data(), sizeof(int) * geb.size(), cudaMemcpyHostToDevice));
			std::vector<int> ginv(geb.size());
			for (size_t k = 0; k < geb.size(); ++k) ginv[geb[k]] = (int)k;
			CREATE_CUDA(cudaMalloc(&c->d_g_eb_inc, sizeof(int) * std::max<size_t>(ginv.size(), 1)));
			if (!ginv.empty())
				CREATE_CUDA(cudaMemcpy(c->d_g_eb_inc, ginv.data(), sizeof(int) * ginv.size(), cudaMemcpyHostToDevice));
		}
	}
	c->sc.max_blocks = (int)(E / 128 + 2);
	CREATE_CUDA(cudaMalloc(&c->sc.partials, sizeof(double) * c->sc.max_blocks));
	CREATE_CUDA(cudaMalloc(&c->sc.ticket, sizeof(unsigned int)));
	CREATE_CUDA(cudaMemset(c->sc.ticket, 0, sizeof(unsigned int)));
	CREATE_CUDA(cudaMalloc(&c->sc.inverted, sizeof(unsigned long long)));
	CREATE_CUDA(cudaMemset(c->sc.inverted, 0, sizeof(unsigned long long)));
	CREATE_CUDA(cudaMalloc(&c->d_result, sizeof(double)));
	CREATE_CUDA(cudaMalloc(&c->d_err, sizeof(int)));
	CREATE_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
	CREATE_CUDA(cudaMalloc(&c->d_work, sizeof(int)));
	CREATE_CUDA(hessian_kernel_setup(c->device));
#undef CREATE_CUDA
	c->m.conn = c->d_conn;
	c->m.gconn = c->d_gconn ? c->d_gconn : c->d_conn;
	c->m.inc_off = c->d_inc_off;
	c->m.inc_eb = c->d_inc_eb;
	c->m.eb_inc = c->d_eb_inc;
	c->m.ginc_off = c->d_ginc_off ? c->d_ginc_off : c->d_inc_off;
	c->m.ginc_eb = c->d_ginc_eb ? c->d_ginc_eb : c->d_inc_eb;
	c->m.g_eb_inc = c->d_g_eb_inc ? c->d_g_eb_inc : c->d_eb_inc;
	c->m.X = c->d_X;
	c->m.lame = c->d_lame;
	c->m.err = c->d_err;
	c->m.work = c->d_work;
	*out = c;
	return PFG_OK;
}

int pfg_destroy(pfg_context *c)
{
	if (!c) return PFG_ERR_INVALID;
	{
		DeviceGuard g(c->device);
		if (c->stream) cudaStreamSynchronize(c->stream);
		free_all(c);
	}
	delete c;
	return PFG_OK;
}

int pfg_set_stream(pfg_context *c, void *stream)
{
	if (!c) return PFG_ERR_INVALID;
	c->stream = (cudaStream_t)stream;
	return PFG_OK;
}

int pfg_set_material(pfg_context *c, int material)
{
	if (!c || material < PFG_MAT_NEOHOOKEAN || material > PFG_MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC)
		return fail(c, PFG_ERR_INVALID, "bad arguments");
	c->m.mat = material;
	c->composite = false;
	return PFG_OK;
}

int pfg_set_elasticity_tensor(pfg_context *c, const double *c21)
{
	if (!c || !c21) return fail(c, PFG_ERR_INVALID, "bad arguments");
	// ElasticityTensor::set_from_entries (MatParams.cpp:180-205): C(i, j), i <= j, row by
	// row; operator() reads C(j, i) for j < i (MatParams.cpp:103-112)
	double full[36];
	for (int i = 0, k = 0; i < 6; ++i)
		for (int j = i; j < 6; ++j, ++k) full[6 * i + j] = full[6 * j + i] = c21[k];
	DeviceGuard g(c->device);
	if (!c->d_hooke) PFG_CUDA(c, cudaMalloc(&c->d_hooke, sizeof(full)));
	PFG_CUDA(c, cudaMemcpyAsync(c->d_hooke, full, sizeof(full), cudaMemcpyHostToDevice, c->stream));
	PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	c->m.hooke = c->d_hooke;
	return PFG_OK;
}

int pfg_set_material_params(pfg_context *c, const double *params, int n_params, int mem)
{
	if (!c || !check_mem(mem) || n_params < 1 || n_params > 8) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (c->m.E && !params) return fail(c, PFG_ERR_INVALID, "params NULL");
	DeviceGuard g(c->device);
	const size_t E = c->m.E;
	constexpr size_t PER = 8; // doubles per element on the device (two double4)
	if (E)
	{
		if (!c->d_mpar)
		{
			PFG_CUDA(c, cudaMalloc(&c->d_mpar, sizeof(double) * PER * E));
			c->m.mpar = c->d_mpar;
		}
		if (mem == PFG_MEM_HOST)
		{
			std::vector<double> pv(PER * E, 0.0);
			for (size_t e = 0; e < E; ++e)
				for (int k = 0; k < n_params; ++k) pv[PER * e + k] = params[(size_t)k * E + e];
			PFG_CUDA(c, cudaMemcpyAsync(c->d_mpar, pv.data(), sizeof(double) * PER * E, cudaMemcpyHostToDevice, c->stream));
			PFG_CUDA(c, cudaStreamSynchronize(c->stream));
		}
		else
		{
			PFG_CUDA(c, cudaMemsetAsync(c->d_mpar, 0, sizeof(double) * PER * E, c->stream));
			for (int k = 0; k < n_params; ++k)
				PFG_CUDA(c, cudaMemcpy2DAsync((char *)c->d_mpar + k * sizeof(double), sizeof(double) * PER,
											  params + (size_t)k * E, sizeof(double), sizeof(double), E,
											  cudaMemcpyDeviceToDevice, c->stream));
		}
	}
	c->n_mpar = n_params;
	return PFG_OK;
}

int pfg_set_component(pfg_context *c, int k, int material, const double *lambda, const double *mu, const double *params,
					  int n_params, const double *c21, int mem)
{
	if (!c || !check_mem(mem) || k < 0 || k >= PFG_MAX_COMPONENTS || material < PFG_MAT_NEOHOOKEAN ||
		material > PFG_MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC || (lambda == nullptr) != (mu == nullptr) || n_params < 0 ||
		n_params > 8)
		return fail(c, PFG_ERR_INVALID, "bad arguments");
	int terms = 0;
	if (material_takes_params(material) && !(n_params > 0 && params && material_params_fit(material, n_params, &terms)))
		return fail(c, PFG_ERR_INVALID, "the component's material takes parameters of another count");
	const bool tensor = material == PFG_MAT_HOOKE || material == PFG_MAT_SAINT_VENANT_TENSOR;
	if (tensor && !c21) return fail(c, PFG_ERR_INVALID, "the component's material takes an elasticity tensor");
	DeviceGuard g(c->device);
	auto &comp = c->comps[k];
	const size_t E = c->m.E;
	comp.mat = material;
	comp.terms = terms;
	comp.n_mpar = material_takes_params(material) ? n_params : 0;
	if (lambda && E)
	{
		if (!comp.lame) PFG_CUDA(c, cudaMalloc(&comp.lame, sizeof(double2) * E));
		std::vector<double2> lm(E);
		std::vector<double> hl, hm;
		const double *pl = lambda, *pm = mu;
		if (mem == PFG_MEM_DEVICE)
		{
			hl.resize(E);
			hm.resize(E);
			PFG_CUDA(c, cudaMemcpy(hl.data(), lambda, sizeof(double) * E, cudaMemcpyDeviceToHost));
			PFG_CUDA(c, cudaMemcpy(hm.data(), mu, sizeof(double) * E, cudaMemcpyDeviceToHost));
			pl = hl.data();
			pm = hm.data();
		}
		for (size_t e = 0; e < E; ++e) lm[e] = make_double2(pl[e], pm[e]);
		PFG_CUDA(c, cudaMemcpy(comp.lame, lm.data(), sizeof(double2) * E, cudaMemcpyHostToDevice));
	}
	else if (comp.lame)
	{
		cudaFree(comp.lame);
		comp.lame = nullptr;
	}
	if (comp.n_mpar && E)
	{
		constexpr size_t PER = 8;
		if (!comp.mpar) PFG_CUDA(c, cudaMalloc(&comp.mpar, sizeof(double) * PER * E));
		std::vector<double> src((size_t)n_params * E), pv(PER * E, 0.0);
		if (mem == PFG_MEM_DEVICE)
			PFG_CUDA(c, cudaMemcpy(src.data(), params, sizeof(double) * src.size(), cudaMemcpyDeviceToHost));
		else
			std::copy(params, params + src.size(), src.begin());
		for (size_t e = 0; e < E; ++e)
			for (int q = 0; q < n_params; ++q) pv[PER * e + q] = src[(size_t)q * E + e];
		PFG_CUDA(c, cudaMemcpy(comp.mpar, pv.data(), sizeof(double) * PER * E, cudaMemcpyHostToDevice));
	}
	if (tensor)
	{
		double full[36];
		for (int i = 0, q = 0; i < 6; ++i)
			for (int j = i; j < 6; ++j, ++q) full[6 * i + j] = full[6 * j + i] = c21[q];
		if (!comp.hooke) PFG_CUDA(c, cudaMalloc(&comp.hooke, sizeof(full)));
		PFG_CUDA(c, cudaMemcpy(comp.hooke, full, sizeof(full), cudaMemcpyHostToDevice));
	}
	return PFG_OK;
}

int pfg_set_composite(pfg_context *c, int n_components, const int *element_component)
{
	if (!c || n_components < 1 || n_components > PFG_MAX_COMPONENTS) return fail(c, PFG_ERR_INVALID, "bad arguments");
	for (int k = 0; k < n_components; ++k)
		if (c->comps[k].mat < 0) return fail(c, PFG_ERR_STATE, "a component is not set (pfg_set_component)");
	DeviceGuard g(c->device);
	const int E = c->m.E;
	if (element_component)
	{
		for (int e = 0; e < E; ++e)
			if (element_component[e] < 0 || element_component[e] >= n_components)
				return fail(c, PFG_ERR_INVALID, "element_component out of range");
		if (!c->d_elem_comp) PFG_CUDA(c, cudaMalloc(&c->d_elem_comp, sizeof(int) * std::max(E, 1)));
		if (E) PFG_CUDA(c, cudaMemcpy(c->d_elem_comp, element_component, sizeof(int) * E, cudaMemcpyHostToDevice));
	}
	else if (c->d_elem_comp)
	{
		cudaFree(c->d_elem_comp);
		c->d_elem_comp = nullptr;
	}
	c->n_comps = n_components;
	c->composite = true;
	return PFG_OK;
}

int pfg_set_lame(pfg_context *c, const double *lambda, const double *mu, int mem)
{
	if (!c || !check_mem(mem)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (c->m.E && (!lambda || !mu)) return fail(c, PFG_ERR_INVALID, "lambda/mu NULL");
	DeviceGuard g(c->device);
	const size_t E = c->m.E;
	if (!E) return PFG_OK;
	if (mem == PFG_MEM_HOST)
	{
		std::vector<double2> lm(E);
		for (size_t e = 0; e < E; ++e) lm[e] = make_double2(lambda[e], mu[e]);
		PFG_CUDA(c, cudaMemcpyAsync(c->d_lame, lm.data(), sizeof(double2) * E, cudaMemcpyHostToDevice, c->stream));
		PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	}
	else
	{
		PFG_CUDA(c, cudaMemcpy2DAsync(c->d_lame, sizeof(double2), lambda, sizeof(double), sizeof(double), E,
									  cudaMemcpyDeviceToDevice, c->stream));
		PFG_CUDA(c, cudaMemcpy2DAsync((char *)c->d_lame + sizeof(double), sizeof(double2), mu, sizeof(double),
									  sizeof(double), E, cudaMemcpyDeviceToDevice, c->stream));
	}
	return PFG_OK;
}

int pfg_set_rest_positions(pfg_context *c, const double *X, int mem)
{
	if (!c || !check_mem(mem)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (c->m.Ng && !X) return fail(c, PFG_ERR_INVALID, "X NULL");
	DeviceGuard g(c->device);
	const size_t bytes = sizeof(double) * 3 * (size_t)c->m.Ng;
	if (!bytes) return PFG_OK;
	PFG_CUDA(c, cudaMemcpyAsync(c->d_X, X, bytes, mem == PFG_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
								c->stream));
	if (mem == PFG_MEM_HOST) PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	return PFG_OK;
}

int pfg_energy(pfg_context *c, const double *u, int mem, int prec, double *out)
{
	if (!c || !check_mem(mem) || !check_prec(prec) || !out) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (c->m.N && !u) return fail(c, PFG_ERR_INVALID, "u NULL");
	if (int st_m = check_material_prec(c, prec)) return st_m;
	DeviceGuard g(c->device);
	int st = ensure_staging(c, 1);
	if (st) return st;
	const double *du;
	if ((st = stage_in(c, u, mem, c->d_u, 3 * (size_t)c->m.N, &du))) return st;
	PFG_CUDA(c, cudaMemsetAsync(c->sc.inverted, 0, sizeof(unsigned long long), c->stream));
	double *dst = mem == PFG_MEM_DEVICE ? out : c->d_result;
	if (c->composite)
	{
		if ((st = composite_energy(c, du, false, dst))) return st;
	}
	else
		PFG_CUDA(c, launch_energy(c->m, du, prec, false, dst, c->sc, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, out, c->d_result, 1);
	return PFG_OK;
}

int pfg_energy_per_element(pfg_context *c, const double *u, int mem, int prec, double *out)
{
	if (!c || !check_mem(mem) || !check_prec(prec) || (c->m.E && !out)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (c->m.N && !u) return fail(c, PFG_ERR_INVALID, "u NULL");
	if (int st_m = check_material_prec(c, prec)) return st_m;
	DeviceGuard g(c->device);
	int st = ensure_staging(c, std::max(c->m.E, 1));
	if (st) return st;
	const double *du;
	if ((st = stage_in(c, u, mem, c->d_u, 3 * (size_t)c->m.N, &du))) return st;
	PFG_CUDA(c, cudaMemsetAsync(c->sc.inverted, 0, sizeof(unsigned long long), c->stream));
	double *dst = mem == PFG_MEM_DEVICE ? out : c->d_out;
	if (c->composite)
	{
		if ((st = composite_energy(c, du, true, dst))) return st;
	}
	else
		PFG_CUDA(c, launch_energy(c->m, du, prec, true, dst, c->sc, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, out, c->d_out, c->m.E);
	return PFG_OK;
}

int pfg_gradient(pfg_context *c, const double *u, int mem, int prec, double *gout)
{
	if (!c || !check_mem(mem) || !check_prec(prec) || (c->m.N && (!gout || !u))) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (int st_m = check_material_prec(c, prec)) return st_m;
	DeviceGuard g(c->device);
	const size_t ndof = 3 * (size_t)c->m.N;
	int st = ensure_staging(c, std::max<size_t>(ndof, 1));
	if (st) return st;
	const double *du;
	if ((st = stage_in(c, u, mem, c->d_u, ndof, &du))) return st;
	PFG_CUDA(c, cudaMemsetAsync(c->sc.inverted, 0, sizeof(unsigned long long), c->stream));
	double *dst = mem == PFG_MEM_DEVICE ? gout : c->d_out;
	if ((st = ensure_vec_stage(c))) return st;
	if (c->composite)
	{
		if ((st = composite_gradient(c, du, dst))) return st;
	}
	else
		PFG_CUDA(c, launch_gradient(c->m, du, prec, dst, c->sc, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, gout, c->d_out, ndof);
	return PFG_OK;
}

int pfg_hessian_pattern(pfg_context *c, long long *nnz)
{
	if (!c) return PFG_ERR_INVALID;
	DeviceGuard g(c->device);
	if (!c->has_pattern)
	{
		const int st = build_pattern(c);
		if (st) return st;
	}
	if (nnz) *nnz = c->pat.nnz;
	return PFG_OK;
}

int pfg_hessian_pattern_copy(pfg_context *c, int *outer, int *inner, int mem)
{
	if (!c || !check_mem(mem)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (!c->has_pattern) return fail(c, PFG_ERR_STATE, "pattern not built");
	DeviceGuard g(c->device);
	const cudaMemcpyKind k = mem == PFG_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
	if (outer) PFG_CUDA(c, cudaMemcpyAsync(outer, c->d_outer, sizeof(int) * (3 * (size_t)c->m.N + 1), k, c->stream));
	if (inner && c->pat.nnz) PFG_CUDA(c, cudaMemcpyAsync(inner, c->d_inner, sizeof(int) * c->pat.nnz, k, c->stream));
	if (mem == PFG_MEM_HOST) PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	return PFG_OK;
}

int pfg_hessian(pfg_context *c, const double *u, int mem, int prec, int project_psd, double *values)
{
	if (!c || !check_mem(mem) || !check_prec(prec)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (c->m.N && !u) return fail(c, PFG_ERR_INVALID, "u NULL");
	if (int st_m = check_material_prec(c, prec)) return st_m;
	DeviceGuard g(c->device);
	int st;
	if (!c->has_pattern && (st = build_pattern(c))) return st;
	if ((st = ensure_staging(c, 1))) return st;
	const double *du;
	if ((st = stage_in(c, u, mem, c->d_u, 3 * (size_t)c->m.N, &du))) return st;
	if ((st = ensure_hess_stage(c, prec))) return st;
	// device output goes straight into the caller's array; otherwise into the context's
	DevPattern p = c->pat;
	if (values && mem == PFG_MEM_DEVICE) p.values = values;
	if (c->composite)
	{
		if ((st = composite_hessian(c, p, du, project_psd))) return st;
	}
	else
		PFG_CUDA(c, launch_hessian(c->m, p, du, prec, project_psd, c->d_hess_stage[prec == PFG_FP64 ? 0 : 1], c->stream));
	if (values && mem == PFG_MEM_HOST) return finish_host(c, values, c->d_values, c->pat.nnz);
	if (mem == PFG_MEM_HOST)
	{
		PFG_CUDA(c, cudaStreamSynchronize(c->stream));
		return check_kernel_flag(c);
	}
	return PFG_OK;
}

int pfg_hessian_apply(pfg_context *c, const double *values, const double *p, int mem, double *q)
{
	if (!c || !check_mem(mem) || (c->m.N && (!p || !q))) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (!c->has_pattern) return fail(c, PFG_ERR_STATE, "no Hessian assembled yet (pattern not built)");
	DeviceGuard g(c->device);
	const size_t ndof = 3 * (size_t)c->m.N;
	int st = ensure_staging(c, std::max<size_t>(ndof, 1));
	if (st) return st;
	const double *dp;
	if ((st = stage_in(c, p, mem, c->d_p, ndof, &dp))) return st;
	double *dq = mem == PFG_MEM_DEVICE ? q : c->d_out;
	PFG_CUDA(c, launch_hessian_apply(c->m.N, c->d_outer, c->d_inner, values ? values : c->d_values, dp, dq, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, q, c->d_out, ndof);
	return PFG_OK;
}

int pfg_hessian_device_csc(pfg_context *c, const int **outer, const int **inner, double **values)
{
	if (!c) return PFG_ERR_INVALID;
	if (!c->has_pattern) return fail(c, PFG_ERR_STATE, "pattern not built");
	if (outer) *outer = c->d_outer;
	if (inner) *inner = c->d_inner;
	if (values) *values = c->d_values;
	return PFG_OK;
}

int pfg_material_vjp(pfg_context *c, const double *u, const double *p, int mem, double *out)
{
	if (!c || !check_mem(mem) || (c->m.E && !out) || (c->m.N && (!u || !p))) return fail(c, PFG_ERR_INVALID, "bad arguments");
	// compute_dstress_dmu_dlambda exists for NeoHookean and LinearElasticity (and
	// FixedCorotational, not built); the reference throws for the others
	if (c->composite || (c->m.mat != PFG_MAT_NEOHOOKEAN && c->m.mat != PFG_MAT_LINEAR_ELASTICITY))
		return fail(c, PFG_ERR_UNSUPPORTED, "the material derivative exists for NeoHookean and LinearElasticity only");
	DeviceGuard g(c->device);
	const size_t ndof = 3 * (size_t)c->m.N;
	int st = ensure_staging(c, std::max<size_t>(2 * (size_t)c->m.E, 1));
	if (st) return st;
	const double *du, *dp;
	if ((st = stage_in(c, u, mem, c->d_u, ndof, &du))) return st;
	if ((st = stage_in(c, p, mem, c->d_p, ndof, &dp))) return st;
	double *dst = mem == PFG_MEM_DEVICE ? out : c->d_out;
	PFG_CUDA(c, launch_material_vjp(c->m, du, dp, dst, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, out, c->d_out, 2 * (size_t)c->m.E);
	return PFG_OK;
}

int pfg_shape_vjp(pfg_context *c, const double *u, const double *p, int mem, int prec, double *out)
{
	if (!c || !check_mem(mem) || !check_prec(prec) || (c->m.Ng && !out) || (c->m.N && (!u || !p)))
		return fail(c, PFG_ERR_INVALID, "bad arguments");
	// compute_stress_grad_multiply_mat exists for every formulation built here but
	// SaintVenant and HookeLinearElasticity, whose reference assemblers throw
	if (c->composite || c->m.mat == PFG_MAT_SAINT_VENANT || c->m.mat == PFG_MAT_SAINT_VENANT_TENSOR ||
		c->m.mat == PFG_MAT_HOOKE)
		return fail(c, PFG_ERR_UNSUPPORTED, "the shape derivative does not exist for SaintVenant and HookeLinearElasticity");
	if (int st_m = check_material_prec(c, prec)) return st_m;
	DeviceGuard g(c->device);
	const size_t ndof = 3 * (size_t)c->m.N;
	int st = ensure_staging(c, std::max<size_t>(3 * (size_t)c->m.Ng, 1));
	if (st) return st;
	const double *du, *dp;
	if ((st = stage_in(c, u, mem, c->d_u, ndof, &du))) return st;
	if ((st = stage_in(c, p, mem, c->d_p, ndof, &dp))) return st;
	double *dst = mem == PFG_MEM_DEVICE ? out : c->d_out;
	if ((st = ensure_vec_stage(c))) return st;
	PFG_CUDA(c, launch_shape_vjp(c->m, du, dp, prec, dst, c->sc, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, out, c->d_out, 3 * (size_t)c->m.Ng);
	return PFG_OK;
}

int pfg_inverted_count(pfg_context *c, long long *count)
{
	if (!c || !count) return PFG_ERR_INVALID;
	DeviceGuard g(c->device);
	unsigned long long v = 0;
	PFG_CUDA(c, cudaMemcpyAsync(&v, c->sc.inverted, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
	PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	*count = (long long)v;
	return PFG_OK;
}

int pfg_synchronize(pfg_context *c)
{
	if (!c) return PFG_ERR_INVALID;
	DeviceGuard g(c->device);
	PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	return check_kernel_flag(c);
}

/* ---------------------------------------------------------------------------
 * Dirichlet reduction (NLProblem with one BCLagrangianForm, which can project)
 * ------------------------------------------------------------------------- */
int pfg_set_dirichlet(pfg_context *c, const int *dofs, int n)
{
	if (!c || n < 0 || (n > 0 && !dofs)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	const int ndof = 3 * c->m.N;
	std::vector<int> d(dofs, dofs + n);
	for (int v : d)
		if (v < 0 || v >= ndof) return fail(c, PFG_ERR_INVALID, "constrained dof out of range");
	std::sort(d.begin(), d.end());
	d.erase(std::unique(d.begin(), d.end()), d.end());
	DeviceGuard g(c->device);
	if (c->stream) PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	int st;
	if (!c->has_pattern && (st = build_pattern(c))) return st;
	c->h_constrained = std::move(d);
	return build_dirichlet(c);
}

int pfg_reduced_pattern(pfg_context *c, int *n_free, long long *nnz)
{
	if (!c) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (!c->has_dirichlet) return fail(c, PFG_ERR_STATE, "no Dirichlet set (pfg_set_dirichlet)");
	if (n_free) *n_free = c->n_free;
	if (nnz) *nnz = c->red_nnz;
	return PFG_OK;
}

int pfg_reduced_pattern_copy(pfg_context *c, int *outer, int *inner, int mem)
{
	if (!c || !check_mem(mem)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (!c->has_dirichlet) return fail(c, PFG_ERR_STATE, "no Dirichlet set (pfg_set_dirichlet)");
	DeviceGuard g(c->device);
	const cudaMemcpyKind k = mem == PFG_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
	if (outer) PFG_CUDA(c, cudaMemcpyAsync(outer, c->d_red_outer, sizeof(int) * ((size_t)c->n_free + 1), k, c->stream));
	if (inner && c->red_nnz) PFG_CUDA(c, cudaMemcpyAsync(inner, c->d_red_inner, sizeof(int) * c->red_nnz, k, c->stream));
	if (mem == PFG_MEM_HOST) PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	return PFG_OK;
}

int pfg_hessian_reduced(pfg_context *c, const double *u, int mem, int prec, int project_psd, double *values)
{
	if (!c || !check_mem(mem) || !check_prec(prec)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (c->m.N && !u) return fail(c, PFG_ERR_INVALID, "u NULL");
	if (!c->has_dirichlet) return fail(c, PFG_ERR_STATE, "no Dirichlet set (pfg_set_dirichlet)");
	if (int st_m = check_material_prec(c, prec)) return st_m;
	DeviceGuard g(c->device);
	int st;
	if ((st = ensure_staging(c, 1))) return st;
	const double *du;
	if ((st = stage_in(c, u, mem, c->d_u, 3 * (size_t)c->m.N, &du))) return st;
	if ((st = ensure_hess_stage(c, prec))) return st;
	DevPattern p = c->pat;
	p.values = (values && mem == PFG_MEM_DEVICE) ? values : c->d_red_values;
	p.red_col_start = c->d_red_col_start;
	p.red_row_off = c->d_red_row_off;
	if (c->composite)
	{
		if ((st = composite_hessian(c, p, du, project_psd))) return st;
	}
	else
		PFG_CUDA(c, launch_hessian(c->m, p, du, prec, project_psd, c->d_hess_stage[prec == PFG_FP64 ? 0 : 1], c->stream));
	if (values && mem == PFG_MEM_HOST) return finish_host(c, values, c->d_red_values, c->red_nnz);
	if (mem == PFG_MEM_HOST) PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	return PFG_OK;
}

int pfg_gradient_reduced(pfg_context *c, const double *u, int mem, int prec, double *g_out)
{
	if (!c || !check_mem(mem) || !check_prec(prec) || (c->m.N && (!g_out || !u))) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (!c->has_dirichlet) return fail(c, PFG_ERR_STATE, "no Dirichlet set (pfg_set_dirichlet)");
	if (int st_m = check_material_prec(c, prec)) return st_m;
	DeviceGuard g(c->device);
	const size_t ndof = 3 * (size_t)c->m.N;
	int st = ensure_staging(c, std::max<size_t>(ndof, 1));
	if (st) return st;
	if (!c->d_full_tmp) PFG_CUDA(c, cudaMalloc(&c->d_full_tmp, sizeof(double) * std::max<size_t>(ndof, 1)));
	const double *du;
	if ((st = stage_in(c, u, mem, c->d_u, ndof, &du))) return st;
	PFG_CUDA(c, cudaMemsetAsync(c->sc.inverted, 0, sizeof(unsigned long long), c->stream));
	if ((st = ensure_vec_stage(c))) return st;
	if (c->composite)
	{
		if ((st = composite_gradient(c, du, c->d_full_tmp))) return st;
	}
	else
		PFG_CUDA(c, launch_gradient(c->m, du, prec, c->d_full_tmp, c->sc, c->stream));
	double *dst = mem == PFG_MEM_DEVICE ? g_out : c->d_out;
	PFG_CUDA(c, launch_gather_free(c->d_full_tmp, c->d_free, c->n_free, dst, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, g_out, c->d_out, c->n_free);
	return PFG_OK;
}

int pfg_mass_matrix(pfg_context *c, const double *rho, int mem, double *values)
{
	if (!c || !check_mem(mem) || !values) return fail(c, PFG_ERR_INVALID, "bad arguments");
	DeviceGuard g(c->device);
	int st;
	if (!c->has_pattern && (st = build_pattern(c))) return st;
	if ((st = ensure_hess_stage(c, PFG_FP64))) return st;
	const double *drho = rho;
	if (rho && mem == PFG_MEM_HOST)
	{
		if (!c->d_rho) PFG_CUDA(c, cudaMalloc(&c->d_rho, sizeof(double) * std::max(c->m.E, 1)));
		if (c->m.E) PFG_CUDA(c, cudaMemcpyAsync(c->d_rho, rho, sizeof(double) * c->m.E, cudaMemcpyHostToDevice, c->stream));
		drho = c->d_rho;
	}
	DevPattern p = c->pat;
	if (mem == PFG_MEM_HOST)
	{
		if (!c->d_mass) PFG_CUDA(c, cudaMalloc(&c->d_mass, sizeof(double) * std::max<long long>(c->pat.nnz, 1)));
		p.values = c->d_mass;
	}
	else
		p.values = values;
	PFG_CUDA(c, launch_mass(c->m, p, drho, c->d_hess_stage[0], c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, values, c->d_mass, c->pat.nnz);
	return PFG_OK;
}

int pfg_lump_matrix(pfg_context *c, const double *values, int mem, double *diag)
{
	if (!c || !check_mem(mem) || !values || !diag) return fail(c, PFG_ERR_INVALID, "bad arguments");
	DeviceGuard g(c->device);
	int st;
	if (!c->has_pattern && (st = build_pattern(c))) return st;
	const long long nnz = c->pat.nnz;
	const int ndof = 3 * c->m.N;
	const double *dv = values;
	double *dd = diag;
	if (mem == PFG_MEM_HOST)
	{
		// host values go through the mass matrix's host staging buffer (nnz doubles)
		if (!c->d_mass) PFG_CUDA(c, cudaMalloc(&c->d_mass, sizeof(double) * std::max<long long>(nnz, 1)));
		if (!c->d_lump) PFG_CUDA(c, cudaMalloc(&c->d_lump, sizeof(double) * std::max(ndof, 1)));
		if (nnz) PFG_CUDA(c, cudaMemcpyAsync(c->d_mass, values, sizeof(double) * nnz, cudaMemcpyHostToDevice, c->stream));
		dv = c->d_mass;
		dd = c->d_lump;
	}
	PFG_CUDA(c, launch_lump_rows(c->m.N, c->d_outer, c->d_inner, dv, dd, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, diag, c->d_lump, ndof);
	return PFG_OK;
}

int pfg_dense_matrix(pfg_context *c, const double *values, int mem, double *dense)
{
	if (!c || !check_mem(mem) || !values || !dense) return fail(c, PFG_ERR_INVALID, "bad arguments");
	DeviceGuard g(c->device);
	int st;
	if (!c->has_pattern && (st = build_pattern(c))) return st;
	const long long nnz = c->pat.nnz;
	const long long ndof = 3LL * c->m.N;
	if (ndof * ndof > PFG_DENSE_MAX_ENTRIES)
		return fail(c, PFG_ERR_UNSUPPORTED, "dense matrix larger than PFG_DENSE_MAX_ENTRIES entries");
	if (mem == PFG_MEM_DEVICE)
	{
		PFG_CUDA(c, launch_csc_to_dense((int)ndof, c->d_outer, c->d_inner, values, dense, c->stream));
		return PFG_OK;
	}
	// host mode: the values and the dense matrix are staged in device buffers of this call
	double *dv = nullptr, *dd = nullptr;
	cudaError_t e = cudaMalloc(&dv, sizeof(double) * std::max<long long>(nnz, 1));
	if (e == cudaSuccess) e = cudaMalloc(&dd, sizeof(double) * std::max<long long>(ndof * ndof, 1));
	if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(dv, values, sizeof(double) * nnz, cudaMemcpyHostToDevice, c->stream);
	if (e == cudaSuccess) e = launch_csc_to_dense((int)ndof, c->d_outer, c->d_inner, dv, dd, c->stream);
	if (e == cudaSuccess && ndof)
		e = cudaMemcpyAsync(dense, dd, sizeof(double) * ndof * ndof, cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
	cudaFree(dv);
	cudaFree(dd);
	if (e != cudaSuccess) return cuda_fail(c, e, "pfg_dense_matrix");
	return PFG_OK;
}

int pfg_cg_solve(pfg_context *c, int system, const double *values, const double *b, int mem, double tol, int max_iter,
				 int guess, double *x, int *iters, double *rel_res)
{
	if (!c || !check_mem(mem) || (system != PFG_SYS_FULL && system != PFG_SYS_REDUCED) || !(tol >= 0.0) || max_iter < 0)
		return fail(c, PFG_ERR_INVALID, "bad arguments");
	const int *outer, *inner, *groups;
	const double *vals;
	int n, ngroups;
	if (system == PFG_SYS_FULL)
	{
		if (!c->has_pattern) return fail(c, PFG_ERR_STATE, "no Hessian assembled (pfg_hessian)");
		outer = c->d_outer;
		inner = c->d_inner;
		vals = values ? values : c->d_values;
		n = 3 * c->m.N;
		groups = nullptr; // node B: columns 3B .. 3B+2
		ngroups = c->m.N;
	}
	else
	{
		if (!c->has_dirichlet) return fail(c, PFG_ERR_STATE, "no Dirichlet set (pfg_set_dirichlet)");
		outer = c->d_red_outer;
		inner = c->d_red_inner;
		vals = values ? values : c->d_red_values;
		n = c->n_free;
		groups = c->d_red_groups;
		ngroups = c->n_red_groups;
	}
	if (n > 0 && (!b || !x)) return fail(c, PFG_ERR_INVALID, "b or x NULL");
	DeviceGuard g(c->device);
	const size_t nn = std::max<size_t>(n, 1);
	if (c->cg_n < nn)
	{
		if (c->d_cg) cudaFree(c->d_cg);
		c->d_cg = nullptr;
		c->cg_n = 0;
		PFG_CUDA(c, cudaMalloc(&c->d_cg, sizeof(double) * (7 * nn + cg_partials_doubles() + CG_NSC)));
		c->cg_n = nn;
	}
	if (!c->h_cg_sc) PFG_CUDA(c, cudaMallocHost(&c->h_cg_sc, sizeof(double) * CG_NSC));
	CgWork w;
	const size_t cn = c->cg_n;
	w.r = c->d_cg;
	w.z = w.r + cn;
	w.p = w.z + cn;
	w.q = w.p + cn;
	w.invd = w.q + cn;
	double *db = w.invd + cn, *dx = db + cn;
	w.part = dx + cn;
	w.sc = w.part + cg_partials_doubles();
	if (mem == PFG_MEM_HOST)
	{
		if (n) PFG_CUDA(c, cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
		if (n && guess) PFG_CUDA(c, cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
	}
	else
	{
		db = const_cast<double *>(b);
		dx = x;
	}
	int it = 0;
	double res = 0.0;
	if (n > 0)
	{
		const auto read_scalars = [&]() -> int {
			PFG_CUDA(c, cudaMemcpyAsync(c->h_cg_sc, w.sc, sizeof(double) * CG_NSC, cudaMemcpyDeviceToHost, c->stream));
			PFG_CUDA(c, cudaStreamSynchronize(c->stream));
			return PFG_OK;
		};
		int st;
		PFG_CUDA(c, launch_cg_diag_inv(n, outer, inner, vals, w.invd, c->stream));
		PFG_CUDA(c, launch_cg_start(n, ngroups, groups, outer, inner, vals, db, guess != 0, tol, dx, w, c->stream));
		// iterations in batches of CG_BATCH; the device stops them at convergence
		constexpr int CG_BATCH = 8;
		int queued = 0;
		for (;;)
		{
			if ((st = read_scalars())) return st;
			if (c->h_cg_sc[CG_DONE] != 0.0 || queued >= max_iter) break;
			const int k = std::min(CG_BATCH, max_iter - queued);
			PFG_CUDA(c, launch_cg_iterations(n, k, ngroups, groups, outer, inner, vals, dx, w, c->stream));
			queued += k;
		}
		const double rhs2 = c->h_cg_sc[CG_RHS2];
		it = (int)c->h_cg_sc[CG_ITER];
		if (rhs2 == 0.0)
			PFG_CUDA(c, cudaMemsetAsync(dx, 0, sizeof(double) * n, c->stream)); // Eigen: x = 0, no iteration
		else
			res = std::sqrt(c->h_cg_sc[CG_RR] / rhs2);
	}
	if (iters) *iters = it;
	if (rel_res) *rel_res = res;
	if (mem == PFG_MEM_HOST) return finish_host(c, x, dx, n);
	return PFG_OK;
}

// the system's device pattern: n, nnz, outer, inner, values; PFG_OK or a state error
static int system_pattern(pfg_context *c, int system, int &n, long long &nnz, const int *&outer, const int *&inner,
						  const double *&vals)
{
	if (system == PFG_SYS_FULL)
	{
		if (!c->has_pattern) return fail(c, PFG_ERR_STATE, "no Hessian assembled (pfg_hessian)");
		n = 3 * c->m.N;
		nnz = c->pat.nnz;
		outer = c->d_outer;
		inner = c->d_inner;
		vals = c->d_values;
		return PFG_OK;
	}
	if (system == PFG_SYS_REDUCED)
	{
		if (!c->has_dirichlet) return fail(c, PFG_ERR_STATE, "no Dirichlet set (pfg_set_dirichlet)");
		n = c->n_free;
		nnz = c->red_nnz;
		outer = c->d_red_outer;
		inner = c->d_red_inner;
		vals = c->d_red_values;
		return PFG_OK;
	}
	return fail(c, PFG_ERR_INVALID, "bad system");
}

int pfg_direct_analyze(pfg_context *c, int system)
{
	if (!c) return fail(c, PFG_ERR_INVALID, "bad arguments");
	int n;
	long long nnz;
	const int *d_outer, *d_inner;
	const double *vals;
	if (int st = system_pattern(c, system, n, nnz, d_outer, d_inner, vals)) return st;
	DeviceGuard g(c->device);
	free_direct(c);
	std::vector<int> outer((size_t)n + 1), inner((size_t)std::max<long long>(nnz, 1));
	PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	PFG_CUDA(c, cudaMemcpy(outer.data(), d_outer, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost));
	if (nnz) PFG_CUDA(c, cudaMemcpy(inner.data(), d_inner, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost));
	pfg::DirectFactor *f = nullptr;
	std::string msg;
	if (int st = direct_symbolic(n, outer.data(), inner.data(), &f, msg)) return fail(c, st, msg);
	if (int st = direct_upload(f, msg))
	{
		direct_destroy(f);
		return fail(c, st, msg);
	}
	c->direct = f;
	c->direct_system = system;
	return PFG_OK;
}

int pfg_direct_factorize(pfg_context *c, int system, const double *values)
{
	if (!c) return fail(c, PFG_ERR_INVALID, "bad arguments");
	int n;
	long long nnz;
	const int *d_outer, *d_inner;
	const double *vals;
	if (int st = system_pattern(c, system, n, nnz, d_outer, d_inner, vals)) return st;
	if (!c->direct || c->direct_system != system || direct_n(c->direct) != n || direct_nnz(c->direct) != nnz)
		return fail(c, PFG_ERR_STATE, "pattern not analysed (pfg_direct_analyze)");
	if (values) vals = values;
	if (nnz && !vals) return fail(c, PFG_ERR_STATE, "no values assembled");
	DeviceGuard g(c->device);
	cudaError_t ce = cudaSuccess;
	const int r = direct_factorize(c->direct, vals, c->stream, &ce);
	if (r == 1) return fail(c, PFG_ERR_NUMERIC, "matrix not positive definite (non-positive pivot)");
	if (r) return cuda_fail(c, ce, "direct_factorize");
	return PFG_OK;
}

int pfg_direct_solve(pfg_context *c, int system, const double *b, int mem, double *x)
{
	if (!c || !check_mem(mem)) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (!c->direct || c->direct_system != system || !direct_factorized(c->direct))
		return fail(c, PFG_ERR_STATE, "not factorised (pfg_direct_factorize)");
	const int n = direct_n(c->direct);
	if (n == 0) return PFG_OK;
	if (!b || !x) return fail(c, PFG_ERR_INVALID, "b or x NULL");
	DeviceGuard g(c->device);
	if (mem == PFG_MEM_HOST)
	{
		double *io = direct_io(c->direct);
		PFG_CUDA(c, cudaMemcpyAsync(io, b, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
		PFG_CUDA(c, direct_solve(c->direct, io, io, c->stream));
		PFG_CUDA(c, cudaMemcpyAsync(x, io, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
		PFG_CUDA(c, cudaStreamSynchronize(c->stream));
		return PFG_OK;
	}
	PFG_CUDA(c, direct_solve(c->direct, b, x, c->stream));
	return PFG_OK;
}

int pfg_direct_free(pfg_context *c)
{
	if (!c) return fail(c, PFG_ERR_INVALID, "bad arguments");
	DeviceGuard g(c->device);
	PFG_CUDA(c, cudaStreamSynchronize(c->stream));
	free_direct(c);
	return PFG_OK;
}

int pfg_direct_stats(const pfg_context *c, long long *stats)
{
	if (!c || !stats) return fail(const_cast<pfg_context *>(c), PFG_ERR_INVALID, "bad arguments");
	if (!c->direct) return fail(const_cast<pfg_context *>(c), PFG_ERR_STATE, "pattern not analysed (pfg_direct_analyze)");
	direct_stats(c->direct, stats);
	return PFG_OK;
}

int pfg_direct_symbolic(int n, const int *outer, const int *inner, long long *stats)
{
	if (n < 0 || !outer || !stats || (n > 0 && outer[n] > 0 && !inner)) return fail(nullptr, PFG_ERR_INVALID, "bad arguments");
	if (outer[0] != 0) return fail(nullptr, PFG_ERR_INVALID, "outer[0] must be 0");
	for (int j = 0; j < n; ++j)
	{
		if (outer[j + 1] < outer[j]) return fail(nullptr, PFG_ERR_INVALID, "outer not monotone");
		for (int t = outer[j]; t < outer[j + 1]; ++t)
			if (inner[t] < 0 || inner[t] >= n || (t > outer[j] && inner[t] <= inner[t - 1]))
				return fail(nullptr, PFG_ERR_INVALID, "rows out of range or not strictly ascending");
	}
	pfg::DirectFactor *f = nullptr;
	std::string msg;
	if (int st = direct_symbolic(n, outer, inner, &f, msg)) return fail(nullptr, st, msg);
	direct_stats(f, stats);
	direct_destroy(f);
	return PFG_OK;
}

int pfg_reduced_to_full(pfg_context *c, const double *y, const double *x_bc, int mem, double *x)
{
	if (!c || !check_mem(mem) || (c->m.N && (!x || (c->n_free && !y)))) return fail(c, PFG_ERR_INVALID, "bad arguments");
	if (!c->has_dirichlet) return fail(c, PFG_ERR_STATE, "no Dirichlet set (pfg_set_dirichlet)");
	DeviceGuard g(c->device);
	const size_t ndof = 3 * (size_t)c->m.N;
	int st = ensure_staging(c, std::max<size_t>(ndof, 1));
	if (st) return st;
	const double *dy = y, *dbc = x_bc;
	if (mem == PFG_MEM_HOST)
	{
		// y -> d_p (n_free <= ndof doubles), x_bc -> d_u
		if (c->n_free) PFG_CUDA(c, cudaMemcpyAsync(c->d_p, y, sizeof(double) * c->n_free, cudaMemcpyHostToDevice, c->stream));
		if (x_bc) PFG_CUDA(c, cudaMemcpyAsync(c->d_u, x_bc, sizeof(double) * ndof, cudaMemcpyHostToDevice, c->stream));
		dy = c->d_p;
		dbc = x_bc ? c->d_u : nullptr;
	}
	double *dst = mem == PFG_MEM_DEVICE ? x : c->d_out;
	PFG_CUDA(c, launch_reduced_to_full(dy, dbc, c->d_old_to_new, (int)ndof, dst, c->stream));
	if (mem == PFG_MEM_HOST) return finish_host(c, x, c->d_out, ndof);
	return PFG_OK;
}

} // extern "C"
