// Linear solve on the device: conjugate gradient with the diagonal (Jacobi)
// preconditioner on the context's assembled Hessian (full or Dirichlet-reduced
// CSC), the hand-off the Newton step makes to its linear solver after every
// assembly: the Hessian NLProblem::hessian returns (solver/NLProblem.cpp:615-621)
// goes to polysolve's linear::Solver (analyze_pattern / factorize / solve),
// called inside the Newton solver of polysolve@47dc48d (external).
//
// The iteration is Eigen's ConjugateGradient with DiagonalPreconditioner (Eigen
// 3.4, the version the reference pins in cmake/recipes/eigen.cmake), restated:
//   r = b - H x, rhs2 = |b|^2;  rhs2 == 0: x = 0, done
//   threshold = max(tol^2 rhs2, smallest normal double)
//   |r|^2 < threshold: done after 0 iterations
//   p = D^-1 r, rz = r.p, i = 0
//   while i < max_iter:
//     q = H p;  alpha = rz / p.q;  x += alpha p;  r -= alpha q
//     |r|^2 < threshold: stop
//     z = D^-1 r;  rz' = r.z;  beta = rz' / rz;  rz = rz';  p = z + beta p;  i += 1
//   iterations = i, relative residual = sqrt(|r|^2 / rhs2)
// with D^-1 = 1 / diag(H) where the diagonal is non-zero, else 1.
// The stop test runs on the device: the reduction that forms |r|^2 sets a done flag
// that makes every later kernel return at once, so the host enqueues iterations in
// batches and reads the flag and the count once per batch.
//
// H is structurally and numerically symmetric (the reduction sums both triangles of
// every block in the same element order), so column j of the CSC is row j and
// q = H p is a gather: one warp per node's columns, no atomics.  Every dot product is a
// fixed-order reduction (warp butterfly, warps in order, blocks in order), so the
// iterates are bitwise deterministic.
#include "pfg_internal.h"

#include <algorithm>

namespace pfg
{

namespace
{

constexpr int CG_NT = 256;      // threads per block of every kernel here
constexpr int CG_MAX_GRID = 1184; // 148 SMs x 8: blocks of the grid-stride kernels
#ifndef PFG_SPMV_MINB
#define PFG_SPMV_MINB 8 // 64 warps per SM at 32 registers (a few spill): measured best
#endif

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// sum over the block's threads in a fixed order; the result is valid in thread 0
__device__ __forceinline__ double block_sum(double v)
{
	__shared__ double ws[CG_NT / 32];
	v = warp_sum(v);
	if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
	__syncthreads();
	double s = 0.0;
	if (threadIdx.x == 0)
#pragma unroll
		for (int w = 0; w < CG_NT / 32; ++w) s += ws[w];
	__syncthreads();
	return s;
}

__global__ void __launch_bounds__(CG_NT) k_diag_inv(int n, const int *__restrict__ outer, const int *__restrict__ inner,
													const double *__restrict__ vals, double *__restrict__ invd)
{
	for (int j = blockIdx.x * CG_NT + threadIdx.x; j < n; j += gridDim.x * CG_NT)
	{
		// rows of a column are sorted: binary search for the diagonal entry
		int lo = __ldg(outer + j), hi = __ldg(outer + j + 1);
		double d = 0.0;
		while (lo < hi)
		{
			const int mid = (lo + hi) >> 1;
			const int r = __ldg(inner + mid);
			if (r == j)
			{
				d = __ldg(vals + mid);
				break;
			}
			if (r < j)
				lo = mid + 1;
			else
				hi = mid;
		}
		invd[j] = d != 0.0 ? 1.0 / d : 1.0;
	}
}

// q = H p, one warp per column group (m <= 3 consecutive columns with the same rows,
// a node's dofs): each row index is loaded and p gathered once for the m columns.
// part[warp] = sum over the warp's columns of p_j q_j when part != nullptr (one
// partial per warp: no block barrier behind the slowest warp).
__global__ void __launch_bounds__(CG_NT, PFG_SPMV_MINB) k_spmv(int ngroups, const int *__restrict__ groups,
												const int *__restrict__ outer, const int *__restrict__ inner,
												const double *__restrict__ vals, const double *__restrict__ p,
												double *__restrict__ q, double *__restrict__ part,
												const double *__restrict__ sc)
{
	if (part && sc[CG_DONE] != 0.0) return; // an iteration after the stopping one
	const int lane = threadIdx.x & 31;
	const int wpb = CG_NT / 32;
	double pq = 0.0;
	for (int g = blockIdx.x * wpb + (threadIdx.x >> 5); g < ngroups; g += gridDim.x * wpb)
	{
		int c0 = 3 * g, m = 3;
		if (groups)
		{
			const int code = __ldg(groups + g);
			c0 = code >> 2;
			m = code & 3;
		}
		const int k0 = __ldg(outer + c0), len = __ldg(outer + c0 + 1) - k0;
		const int o1 = m > 1 ? __ldg(outer + c0 + 1) : k0, o2 = m > 2 ? __ldg(outer + c0 + 2) : k0;
		double s0 = 0.0, s1 = 0.0, s2 = 0.0;
		for (int t = lane; t < len; t += 32)
		{
			const double pv = __ldg(p + __ldg(inner + k0 + t));
			s0 = fma(__ldg(vals + k0 + t), pv, s0);
			if (m > 1) s1 = fma(__ldg(vals + o1 + t), pv, s1);
			if (m > 2) s2 = fma(__ldg(vals + o2 + t), pv, s2);
		}
		s0 = warp_sum(s0);
		if (m > 1) s1 = warp_sum(s1);
		if (m > 2) s2 = warp_sum(s2);
		if (lane == 0)
		{
			q[c0] = s0;
			pq = fma(p[c0], s0, pq);
			if (m > 1)
			{
				q[c0 + 1] = s1;
				pq = fma(p[c0 + 1], s1, pq);
			}
			if (m > 2)
			{
				q[c0 + 2] = s2;
				pq = fma(p[c0 + 2], s2, pq);
			}
		}
	}
	if (part && lane == 0) part[blockIdx.x * wpb + (threadIdx.x >> 5)] = pq;
}

// r = b - q
__global__ void __launch_bounds__(CG_NT) k_resid(int n, const double *__restrict__ b, const double *__restrict__ q,
												 double *__restrict__ r)
{
	for (int j = blockIdx.x * CG_NT + threadIdx.x; j < n; j += gridDim.x * CG_NT) r[j] = b[j] - q[j];
}

// z = D^-1 r, p = z; part = (r.z, r.r, b.b) per block
__global__ void __launch_bounds__(CG_NT) k_cg_start(int n, const double *__restrict__ invd, const double *__restrict__ b,
													const double *__restrict__ r, double *__restrict__ p,
													double *__restrict__ part)
{
	double rz = 0.0, rr = 0.0, bb = 0.0;
	for (int j = blockIdx.x * CG_NT + threadIdx.x; j < n; j += gridDim.x * CG_NT)
	{
		const double rj = r[j], zj = invd[j] * rj, bj = b[j];
		p[j] = zj;
		rz = fma(rj, zj, rz);
		rr = fma(rj, rj, rr);
		bb = fma(bj, bj, bb);
	}
	const double s0 = block_sum(rz), s1 = block_sum(rr), s2 = block_sum(bb);
	if (threadIdx.x == 0)
	{
		part[blockIdx.x] = s0;
		part[gridDim.x + blockIdx.x] = s1;
		part[2 * gridDim.x + blockIdx.x] = s2;
	}
}

// x += alpha p, r -= alpha q, z = D^-1 r; part = (r.r, r.z) per block
__global__ void __launch_bounds__(CG_NT) k_cg_step(int n, const double *__restrict__ sc, const double *__restrict__ p,
												   const double *__restrict__ q, double *__restrict__ x,
												   double *__restrict__ r, const double *__restrict__ invd,
												   double *__restrict__ z, double *__restrict__ part)
{
	if (sc[CG_DONE] != 0.0) return;
	const double alpha = sc[CG_ALPHA];
	double rr = 0.0, rz = 0.0;
	for (int j = blockIdx.x * CG_NT + threadIdx.x; j < n; j += gridDim.x * CG_NT)
	{
		x[j] = fma(alpha, p[j], x[j]);
		const double rj = fma(-alpha, q[j], r[j]);
		r[j] = rj;
		const double zj = invd[j] * rj;
		z[j] = zj;
		rr = fma(rj, rj, rr);
		rz = fma(rj, zj, rz);
	}
	const double s0 = block_sum(rr), s1 = block_sum(rz);
	if (threadIdx.x == 0)
	{
		part[blockIdx.x] = s0;
		part[gridDim.x + blockIdx.x] = s1;
	}
}

// p = z + beta p
__global__ void __launch_bounds__(CG_NT) k_cg_dir(int n, const double *__restrict__ sc, const double *__restrict__ z,
												  double *__restrict__ p)
{
	if (sc[CG_DONE] != 0.0) return;
	const double beta = sc[CG_BETA];
	for (int j = blockIdx.x * CG_NT + threadIdx.x; j < n; j += gridDim.x * CG_NT) p[j] = fma(beta, p[j], z[j]);
}

enum
{
	RED_START = 0, // (r.z, r.r, b.b) -> rz, rr, rhs2
	RED_ALPHA = 1, // p.q -> alpha = rz / p.q
	RED_BETA = 2   // (r.r, r.z') -> rr, beta = rz' / rz, rz = rz'
};

// one block: the per-block partials summed in block order, then the scalars
__global__ void __launch_bounds__(CG_NT) k_cg_reduce(const double *__restrict__ part, int count, int mode, double tol,
													 double *__restrict__ sc)
{
	if (mode != RED_START && sc[CG_DONE] != 0.0) return;
	const int ncomp = mode == RED_START ? 3 : (mode == RED_ALPHA ? 1 : 2);
	double s[3] = {0.0, 0.0, 0.0};
	for (int c = 0; c < ncomp; ++c)
	{
		double v = 0.0;
		for (int i = threadIdx.x; i < count; i += CG_NT) v += part[c * count + i];
		s[c] = block_sum(v);
	}
	if (threadIdx.x != 0) return;
	if (mode == RED_START)
	{
		sc[CG_RZ] = s[0];
		sc[CG_RR] = s[1];
		sc[CG_RHS2] = s[2];
		const double thr = fmax(tol * tol * s[2], 2.2250738585072014e-308);
		sc[CG_THR] = thr;
		sc[CG_DONE] = (s[2] == 0.0 || s[1] < thr) ? 1.0 : 0.0;
		sc[CG_ITER] = 0.0;
	}
	else if (mode == RED_ALPHA)
		sc[CG_ALPHA] = sc[CG_RZ] / s[0];
	else
	{
		sc[CG_RR] = s[0];
		if (s[0] < sc[CG_THR])
			sc[CG_DONE] = 1.0; // converged: x and r stay as they are, the count is not advanced
		else
		{
			sc[CG_BETA] = s[1] / sc[CG_RZ];
			sc[CG_RZ] = s[1];
			sc[CG_ITER] += 1.0;
		}
	}
}

int grid_vec(int n) { return n <= 0 ? 1 : (int)std::min<long long>(CG_MAX_GRID, ((long long)n + CG_NT - 1) / CG_NT); }
int grid_spmv(int ngroups) { return ngroups <= 0 ? 1 : (int)std::min<long long>(CG_MAX_GRID, ((long long)ngroups + 7) / 8); }

} // namespace

size_t cg_partials_doubles() { return (size_t)(CG_NT / 32) * CG_MAX_GRID; } // one per SpMV warp, >= 3 per vector block

cudaError_t launch_hessian_apply(int n_nodes, const int *outer, const int *inner, const double *vals, const double *p,
								 double *q, cudaStream_t s)
{
	if (n_nodes > 0)
		k_spmv<<<grid_spmv(n_nodes), CG_NT, 0, s>>>(n_nodes, nullptr, outer, inner, vals, p, q, nullptr, nullptr);
	return cudaGetLastError();
}

cudaError_t launch_cg_diag_inv(int n, const int *outer, const int *inner, const double *vals, double *invd,
							   cudaStream_t s)
{
	if (n > 0) k_diag_inv<<<grid_vec(n), CG_NT, 0, s>>>(n, outer, inner, vals, invd);
	return cudaGetLastError();
}

cudaError_t launch_cg_start(int n, int ngroups, const int *groups, const int *outer, const int *inner,
							const double *vals, const double *b, bool guess, double tol, double *x, const CgWork &w,
							cudaStream_t s)
{
	const int gv = grid_vec(n);
	if (guess)
	{
		k_spmv<<<grid_spmv(ngroups), CG_NT, 0, s>>>(ngroups, groups, outer, inner, vals, x, w.q, nullptr, w.sc);
		k_resid<<<gv, CG_NT, 0, s>>>(n, b, w.q, w.r);
	}
	else
	{
		cudaError_t e = cudaMemsetAsync(x, 0, sizeof(double) * (size_t)n, s);
		if (e != cudaSuccess) return e;
		e = cudaMemcpyAsync(w.r, b, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, s);
		if (e != cudaSuccess) return e;
	}
	k_cg_start<<<gv, CG_NT, 0, s>>>(n, w.invd, b, w.r, w.p, w.part);
	k_cg_reduce<<<1, CG_NT, 0, s>>>(w.part, gv, RED_START, tol, w.sc);
	return cudaGetLastError();
}

cudaError_t launch_cg_iterations(int n, int count, int ngroups, const int *groups, const int *outer,
								 const int *inner, const double *vals, double *x, const CgWork &w, cudaStream_t s)
{
	const int gs = grid_spmv(ngroups), gv = grid_vec(n);
	for (int i = 0; i < count; ++i)
	{
		k_spmv<<<gs, CG_NT, 0, s>>>(ngroups, groups, outer, inner, vals, w.p, w.q, w.part, w.sc);
		k_cg_reduce<<<1, CG_NT, 0, s>>>(w.part, gs * (CG_NT / 32), RED_ALPHA, 0.0, w.sc);
		k_cg_step<<<gv, CG_NT, 0, s>>>(n, w.sc, w.p, w.q, x, w.r, w.invd, w.z, w.part);
		k_cg_reduce<<<1, CG_NT, 0, s>>>(w.part, gv, RED_BETA, 0.0, w.sc);
		k_cg_dir<<<gv, CG_NT, 0, s>>>(n, w.sc, w.z, w.p);
	}
	return cudaGetLastError();
}

} // namespace pfg
