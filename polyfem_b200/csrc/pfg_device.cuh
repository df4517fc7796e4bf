// Element helpers shared by the assembly kernels (pfg_kernels.cu, pfg_materials.cu):
// gathers of geometry and nodal values, the per-point geometry, 32-byte staging
// slots and the deterministic two-level reduction.
#pragma once
#include "pfg_elem.cuh"
#include "pfg_internal.h"

namespace pfg
{

// ---------------------------------------------------------------------------
// shared element helpers
// ---------------------------------------------------------------------------
template <class EL, class T>
__device__ __forceinline__ void load_geom(const DevMesh &m, int e, T Xg[EL::NG][3])
{
#pragma unroll
	for (int j = 0; j < EL::NG; ++j)
	{
		const int g = __ldg(m.gconn + (size_t)j * m.E + e);
		const double *x = m.X + (size_t)g * 3;
		Xg[j][0] = T(__ldg(x + 0));
		Xg[j][1] = T(__ldg(x + 1));
		Xg[j][2] = T(__ldg(x + 2));
	}
}

template <class EL, class T>
__device__ __forceinline__ void load_nodal(const DevMesh &m, int e, const double *__restrict__ f, T U[EL::N][3], int nodes[EL::N])
{
#pragma unroll
	for (int a = 0; a < EL::N; ++a)
	{
		const int n = __ldg(m.conn + (size_t)a * m.E + e);
		nodes[a] = n;
		const double *p = f + (size_t)n * 3;
		U[a][0] = T(__ldg(p + 0));
		U[a][1] = T(__ldg(p + 1));
		U[a][2] = T(__ldg(p + 2));
	}
}

// Geometry at quadrature point q: J^-T and det J (ElementAssemblyValues.cpp:76-104).
// The determinant is always FP64; J^-T is kept in T.
template <class EL, class T>
__device__ __forceinline__ void geometry(int q, const T Xg[EL::NG][3], T Jit[3][3], double &detJ)
{
	T Jac[3][3];
	geom_jacobian<EL, T>(q, Xg, Jac);
	if constexpr (sizeof(T) == 8)
	{
		detJ = det3(Jac);
		inv_transpose3(Jac, T(detJ), Jit);
	}
	else
	{
		double Jd[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) Jd[r][c] = double(Jac[r][c]);
		detJ = det3(Jd);
		inv_transpose3(Jac, T(detJ), Jit);
	}
}

// physical gradients gphi[a][c] = sum_r gref(q,a,r) Jit[r][c]  (grad_t_m)
template <class EL, class T>
__device__ __forceinline__ void phys_grads(int q, const T Jit[3][3], T gphi[EL::N][3])
{
#pragma unroll
	for (int a = 0; a < EL::N; ++a)
#pragma unroll
		for (int c = 0; c < 3; ++c)
		{
			T s = T(0);
#pragma unroll
			for (int r = 0; r < 3; ++r)
			{
				const double gr = gref<EL>(q, a, r);
				if (gr != 0.0) s += T(gr) * Jit[r][c];
			}
			gphi[a][c] = s;
		}
}

// displacement gradient G[r][c] = sum_a U[a][r] gphi[a][c]
template <class EL, class T>
__device__ __forceinline__ void disp_grad(const T U[EL::N][3], const T gphi[EL::N][3], T G[3][3])
{
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c)
		{
			T s = T(0);
#pragma unroll
			for (int a = 0; a < EL::N; ++a) s += U[a][r] * gphi[a][c];
			G[r][c] = s;
		}
}

// one 32-byte staging slot (one DRAM sector): (x, y, z, 0) in two 16-byte stores
__device__ __forceinline__ void st_slot(double *p, double x, double y, double z)
{
	reinterpret_cast<double2 *>(p)[0] = make_double2(x, y);
	reinterpret_cast<double2 *>(p)[1] = make_double2(z, 0.0);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	return v;
}

// Deterministic two-level reduction: fixed tree inside each block, then the
// last block to finish sums the per-block partials in block order.
template <int NT>
__device__ void reduce_to_result(double v, double *partials, double *result, unsigned int *ticket)
{
	__shared__ double s_w[NT / 32];
	__shared__ bool s_last;
	v = warp_sum(v);
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	if (lane == 0) s_w[wid] = v;
	__syncthreads();
	if (threadIdx.x == 0)
	{
		double b = 0.0;
		for (int i = 0; i < NT / 32; ++i) b += s_w[i];
		partials[blockIdx.x] = b;
		__threadfence();
		const unsigned int t = atomicAdd(ticket, 1u);
		s_last = (t == gridDim.x - 1);
	}
	__syncthreads();
	if (!s_last) return;
	__threadfence();
	// the partials this thread sums, in index order; up to eight loads (from L2,
	// where the other blocks' writes are visible after their fences) are in flight
	// before the first add, so the tail is one round trip instead of one per partial
	double acc = 0.0;
	for (int i0 = threadIdx.x; i0 < (int)gridDim.x; i0 += 8 * NT)
	{
		double x[8];
#pragma unroll
		for (int j = 0; j < 8; ++j)
		{
			const int i = i0 + j * NT;
			x[j] = i < (int)gridDim.x ? __ldcg(partials + i) : 0.0;
		}
#pragma unroll
		for (int j = 0; j < 8; ++j)
			if (i0 + j * NT < (int)gridDim.x) acc += x[j];
	}
	acc = warp_sum(acc);
	if (lane == 0) s_w[wid] = acc;
	__syncthreads();
	if (threadIdx.x == 0)
	{
		double b = 0.0;
		for (int i = 0; i < NT / 32; ++i) b += s_w[i];
		*result = b;
		*ticket = 0u;
	}
}

// index pairs (a <= b) of an n x n symmetric table in tri_index order, for lane
// lookup tables in constant memory (n <= 10)
struct PairTable
{
	unsigned char a[55], b[55];
};
constexpr PairTable make_pairs(int n)
{
	PairTable t{};
	int p = 0;
	for (int a = 0; a < n; ++a)
		for (int b = a; b < n; ++b)
		{
			t.a[p] = (unsigned char)a;
			t.b[p] = (unsigned char)b;
			++p;
		}
	return t;
}

// F = I + (U^T gref_q) J^-T at quadrature point q
template <class EL>
__device__ __forceinline__ void gen_def_grad(int q, const double U[EL::N][3], const double Jit[3][3], double F[3][3])
{
	double A[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c)
		{
			double s_ = 0.0;
#pragma unroll
			for (int a = 0; a < EL::N; ++a) s_ += U[a][r] * gref<EL>(q, a, c);
			A[r][c] = s_;
		}
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) F[r][c] = A[r][0] * Jit[0][c] + A[r][1] * Jit[1][c] + A[r][2] * Jit[2][c] + (r == c);
}

} // namespace pfg
