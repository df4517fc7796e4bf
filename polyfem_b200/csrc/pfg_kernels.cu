// NeoHookean energy / gradient / Hessian / adjoint kernels for sm_100a.
//
// Mathematics (reference: assembler/NeoHookeanElasticity.cpp):
//   F   = I + sum_a u_a (x) grad(phi_a),   grad(phi_a) = gref_a * J^-T      (:337-388, :453-545)
//   psi = mu/2 (|F|^2 - 3 - 2 ln J) + lambda/2 ln^2 J                     (:384)
//   P   = mu F + (lambda ln J - mu)/J cof(F)                                (:532)
//   C   = mu I + (mu + lambda(1 - ln J))/J^2 g g^T + (lambda ln J - mu)/J d2J/dF2   (:636)
// The element Hessian is contracted analytically per node pair (a, b):
//   H_ab = sum_q da [ mu (ga.gb) I + alpha c_a c_b^T + beta eps(F (ga x gb)) ]
// with ga = grad(phi_a), c_a = cof(F) ga, alpha = (mu + lambda(1 - ln J))/J^2,
// beta = (lambda ln J - mu)/J and eps(w)[m][n] = sum_p eps_mnp w_p.  This is
// exactly B^T C B of the reference (d2J/dF_mk dF_nl = eps_mnp eps_klq F_pq),
// evaluated without the zeros of B.
#include "pfg_elem.cuh"
#include "pfg_internal.h"

#include <cstdio>

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
	double acc = 0.0;
	for (int i = threadIdx.x; i < (int)gridDim.x; i += NT) acc += *((volatile double *)partials + i);
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

// ---------------------------------------------------------------------------
// energy (NLAssembler::assemble_energy / assemble_energy_per_element)
// ---------------------------------------------------------------------------
template <class EL, class T>
__device__ __forceinline__ double element_energy(const DevMesh &m, const double *__restrict__ u, int e,
												 unsigned long long *inverted)
{
	T Xg[EL::NG][3];
	T U[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, T>(m, e, Xg);
	load_nodal<EL, T>(m, e, u, U, nodes);
	const double2 lm = __ldg(m.lame + e);
	const double lambda = lm.x, mu = lm.y;
	T Jit[3][3];
	double detJ = 0.0;
	if constexpr (EL::AFFINE) geometry<EL, T>(0, Xg, Jit, detJ);
	double en = 0.0;
	bool bad = false;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		if constexpr (!EL::AFFINE) geometry<EL, T>(q, Xg, Jit, detJ);
		// A = U^T * gref, G = A * Jit  (reference order: (local_disp^T grad) jac_it)
		T A[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				T s = T(0);
#pragma unroll
				for (int a = 0; a < EL::N; ++a)
				{
					const double g = gref<EL>(q, a, c);
					if (g != 0.0) s += U[a][r] * T(g);
				}
				A[r][c] = s;
			}
		double Fd[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				T s = T(0);
#pragma unroll
				for (int k = 0; k < 3; ++k) s += A[r][k] * Jit[k][c];
				Fd[r][c] = double(s);
			}
		double val;
		if constexpr (sizeof(T) == 8)
		{
#pragma unroll
			for (int r = 0; r < 3; ++r) Fd[r][r] += 1.0;
			const double J = det3(Fd);
			const double lj = log(J);
			bad |= !(J > 0.0);
			double sq = 0.0;
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) sq += Fd[r][c] * Fd[r][c];
			val = mu / 2 * (sq - 3 - 2 * lj) + lambda / 2 * lj * lj;
		}
		else
		{
			// FP32 displacement gradient G, invariants in FP64: |F|^2 - 3 = 2 tr G + |G|^2
			double tr = Fd[0][0] + Fd[1][1] + Fd[2][2];
			double g2 = 0.0;
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) g2 += Fd[r][c] * Fd[r][c];
#pragma unroll
			for (int r = 0; r < 3; ++r) Fd[r][r] += 1.0;
			const double J = det3(Fd);
			const double lj = log(J);
			bad |= !(J > 0.0);
			val = mu / 2 * (2 * tr + g2 - 2 * lj) + lambda / 2 * lj * lj;
		}
		en += val * (detJ * qweight<EL>(q));
	}
	if (bad) atomicAdd(inverted, 1ull);
	return en;
}

template <class EL, class T, int NT>
__global__ void __launch_bounds__(NT) k_energy(DevMesh m, const double *__restrict__ u, double *__restrict__ partials,
											   double *__restrict__ result, unsigned int *ticket,
											   unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	double en = 0.0;
	if (e < m.E) en = element_energy<EL, T>(m, u, e, inverted);
	reduce_to_result<NT>(en, partials, result, ticket);
}

template <class EL, class T, int NT>
__global__ void __launch_bounds__(NT) k_energy_per_element(DevMesh m, const double *__restrict__ u,
														   double *__restrict__ out, unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e < m.E) out[e] = element_energy<EL, T>(m, u, e, inverted);
}

// ---------------------------------------------------------------------------
// gradient (NLAssembler::assemble_gradient)
// ---------------------------------------------------------------------------
template <class EL, class T, int NT>
__global__ void __launch_bounds__(NT) k_gradient(DevMesh m, const double *__restrict__ u, double *__restrict__ g,
												 unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	T Xg[EL::NG][3];
	T U[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, T>(m, e, Xg);
	load_nodal<EL, T>(m, e, u, U, nodes);
	const double2 lm = __ldg(m.lame + e);
	const double lambda = lm.x, mu = lm.y;
	// element gradient, accumulated as G[a][d] = sum_q sum_r gref(q,a,r) (da P J^-1)[d][r]
	// so the physical basis gradients are never materialised
	T Gacc[EL::N][3];
#pragma unroll
	for (int a = 0; a < EL::N; ++a) Gacc[a][0] = Gacc[a][1] = Gacc[a][2] = T(0);
	T Jit[3][3];
	double detJ = 0.0;
	if constexpr (EL::AFFINE) geometry<EL, T>(0, Xg, Jit, detJ);
	bool bad = false;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		if constexpr (!EL::AFFINE) geometry<EL, T>(q, Xg, Jit, detJ);
		T A[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				T s = T(0);
#pragma unroll
				for (int a = 0; a < EL::N; ++a)
				{
					const double gr = gref<EL>(q, a, c);
					if (gr != 0.0) s += U[a][r] * T(gr);
				}
				A[r][c] = s;
			}
		T F[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
				F[r][c] = A[r][0] * Jit[0][c] + A[r][1] * Jit[1][c] + A[r][2] * Jit[2][c] + (r == c ? T(1) : T(0));
		double J;
		if constexpr (sizeof(T) == 8)
			J = det3(F);
		else
		{
			double Fd[3][3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) Fd[r][c] = F[r][c];
			J = det3(Fd);
		}
		const double lj = log(J);
		bad |= !(J > 0.0);
		T D[3][3];
		cofactor3(F, D);
		const T s2 = T((lambda * lj - mu) / J);
		const T tmu = T(mu);
		const T da = T(detJ * qweight<EL>(q));
		T P[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) P[r][c] = (tmu * F[r][c] + s2 * D[r][c]) * da;
		// Q = P J^-1 = P Jit^T
		T Q[3][3];
#pragma unroll
		for (int d = 0; d < 3; ++d)
#pragma unroll
			for (int r = 0; r < 3; ++r) Q[d][r] = P[d][0] * Jit[r][0] + P[d][1] * Jit[r][1] + P[d][2] * Jit[r][2];
#pragma unroll
		for (int a = 0; a < EL::N; ++a)
#pragma unroll
			for (int r = 0; r < 3; ++r)
			{
				const double gr = gref<EL>(q, a, r);
				if (gr != 0.0)
				{
#pragma unroll
					for (int d = 0; d < 3; ++d) Gacc[a][d] += T(gr) * Q[d][r];
				}
			}
	}
	if (bad) atomicAdd(inverted, 1ull);
#pragma unroll
	for (int a = 0; a < EL::N; ++a)
#pragma unroll
		for (int d = 0; d < 3; ++d) atomicAdd(g + (size_t)nodes[a] * 3 + d, double(Gacc[a][d]));
}

// ---------------------------------------------------------------------------
// Hessian (NLAssembler::assemble_hessian + SparseMatrixCache slot adds)
// ---------------------------------------------------------------------------
template <class EL>
struct HessTile
{
	static constexpr int TE = (EL::ET == 1) ? 32 : 8; // elements per tile
	static constexpr int NT = 256;
	static constexpr int N = EL::N, NQ = EL::NQ;
	static constexpr int NP = N * (N + 1) / 2; // symmetric node pairs
	static constexpr int NB = N * N;           // node blocks
};

template <class EL, class T>
struct HessSmem
{
	using TL = HessTile<EL>;
	T gphi[TL::TE][TL::NQ][TL::N][3]; // physical gradients
	T cvec[TL::TE][TL::NQ][TL::N][3]; // cof(F) * gphi_a
	T F[TL::TE][TL::NQ][9];
	T sc[TL::TE][TL::NQ][3];          // mu*da, alpha*da, beta*da
	T U[TL::TE][TL::N][3];
	T H[TL::TE][TL::NB * 9];          // element Hessian, [a*N+b][c*3+m] = H_e(3a+m, 3b+c)
	int slot[TL::TE][TL::NB];
	int stride[TL::TE][TL::N];
};

template <class EL, class T>
__global__ void __launch_bounds__(HessTile<EL>::NT) k_hessian(DevMesh m, DevPattern pat, const double *__restrict__ u)
{
	using TL = HessTile<EL>;
	constexpr int TE = TL::TE, NT = TL::NT, N = TL::N, NQ = TL::NQ, NP = TL::NP, NB = TL::NB;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	HessSmem<EL, T> &S = *reinterpret_cast<HessSmem<EL, T> *>(smem_raw);
	const int tid = threadIdx.x;
	const int e0 = blockIdx.x * TE;

	// phase 0: slots, column strides and nodal displacements of the tile
	for (int i = tid; i < TE * NB; i += NT)
	{
		const int el = i / NB, e = e0 + el;
		S.slot[el][i % NB] = (e < m.E) ? __ldg(pat.slot + (size_t)e0 * NB + i) : 0;
	}
	for (int i = tid; i < TE * N * 3; i += NT)
	{
		const int el = i / (N * 3), r = i % (N * 3), a = r / 3, d = r % 3, e = e0 + el;
		if (e < m.E)
		{
			const int node = __ldg(m.conn + (size_t)a * m.E + e);
			S.U[el][a][d] = T(__ldg(u + (size_t)node * 3 + d));
			if (d == 0) S.stride[el][a] = __ldg(pat.colstride + node);
		}
		else
		{
			S.U[el][a][d] = T(0);
			if (d == 0) S.stride[el][a] = 0;
		}
	}
	__syncthreads();

	// phase 1: per (element, quadrature point) kinematics
	for (int i = tid; i < TE * NQ; i += NT)
	{
		const int el = i / NQ, q = i % NQ, e = e0 + el;
		if (e >= m.E) continue;
		T Xg[EL::NG][3];
		load_geom<EL, T>(m, e, Xg);
		T Jit[3][3];
		double detJ;
		// the quadrature point index is a run-time value here; unrolled dispatch keeps tables constant
#pragma unroll
		for (int qq = 0; qq < NQ; ++qq)
		{
			if (qq != q) continue;
			geometry<EL, T>(qq, Xg, Jit, detJ);
			T gphi[N][3];
			phys_grads<EL, T>(qq, Jit, gphi);
			T F[3][3];
			{
				T U[N][3];
#pragma unroll
				for (int a = 0; a < N; ++a)
#pragma unroll
					for (int d = 0; d < 3; ++d) U[a][d] = S.U[el][a][d];
				disp_grad<EL, T>(U, gphi, F);
			}
#pragma unroll
			for (int r = 0; r < 3; ++r) F[r][r] += T(1);
			double J;
			if constexpr (sizeof(T) == 8)
				J = det3(F);
			else
			{
				double Fd[3][3];
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int c = 0; c < 3; ++c) Fd[r][c] = F[r][c];
				J = det3(Fd);
			}
			const double lj = log(J);
			const double2 lm = __ldg(m.lame + e);
			const double lambda = lm.x, mu = lm.y;
			const double da = detJ * qweight<EL>(qq);
			T D[3][3];
			cofactor3(F, D);
			S.sc[el][qq][0] = T(mu * da);
			S.sc[el][qq][1] = T((mu + lambda * (1 - lj)) / (J * J) * da);
			S.sc[el][qq][2] = T((lambda * lj - mu) / J * da);
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) S.F[el][qq][r * 3 + c] = F[r][c];
#pragma unroll
			for (int a = 0; a < N; ++a)
#pragma unroll
				for (int c = 0; c < 3; ++c)
				{
					S.gphi[el][qq][a][c] = gphi[a][c];
					S.cvec[el][qq][a][c] = D[c][0] * gphi[a][0] + D[c][1] * gphi[a][1] + D[c][2] * gphi[a][2];
				}
		}
	}
	__syncthreads();

	// phase 2: symmetric node pairs
	for (int i = tid; i < TE * NP; i += NT)
	{
		const int el = i / NP;
		int p = i % NP, a = 0;
		while (p >= N - a)
		{
			p -= N - a;
			++a;
		}
		const int b = a + p;
		T h[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r) h[r][0] = h[r][1] = h[r][2] = T(0);
		if (e0 + el < m.E)
		{
#pragma unroll
			for (int q = 0; q < NQ; ++q)
			{
				const T *ga = S.gphi[el][q][a], *gb = S.gphi[el][q][b];
				const T *ca = S.cvec[el][q][a], *cb = S.cvec[el][q][b];
				const T *F = S.F[el][q];
				const T smu = S.sc[el][q][0], sal = S.sc[el][q][1], sbe = S.sc[el][q][2];
				const T dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
				const T x0 = ga[1] * gb[2] - ga[2] * gb[1];
				const T x1 = ga[2] * gb[0] - ga[0] * gb[2];
				const T x2 = ga[0] * gb[1] - ga[1] * gb[0];
				const T w0 = (F[0] * x0 + F[1] * x1 + F[2] * x2) * sbe;
				const T w1 = (F[3] * x0 + F[4] * x1 + F[5] * x2) * sbe;
				const T w2 = (F[6] * x0 + F[7] * x1 + F[8] * x2) * sbe;
				const T md = smu * dot;
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int c = 0; c < 3; ++c) h[r][c] += sal * ca[r] * cb[c];
				h[0][0] += md;
				h[1][1] += md;
				h[2][2] += md;
				// + beta * eps_{mnp} w_p
				h[0][1] += w2;
				h[1][0] -= w2;
				h[1][2] += w0;
				h[2][1] -= w0;
				h[2][0] += w1;
				h[0][2] -= w1;
			}
		}
		T *Hab = S.H[el] + (a * N + b) * 9;
		T *Hba = S.H[el] + (b * N + a) * 9;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				Hab[c * 3 + r] = h[r][c];
				if (a != b) Hba[r * 3 + c] = h[r][c];
			}
	}
	__syncthreads();

	// phase 3: scatter through the slot map; consecutive threads hit consecutive rows
	for (int i = tid; i < TE * NB * 9; i += NT)
	{
		const int el = i / (NB * 9), r = i % (NB * 9);
		if (e0 + el >= m.E) continue;
		const int pair = r / 9, c = (r % 9) / 3, mrow = r % 3;
		const int b = pair % N;
		const long long idx = (long long)S.slot[el][pair] + (long long)c * S.stride[el][b] + mrow;
		atomicAdd(pat.values + idx, double(S.H[el][r]));
	}
}

// ---------------------------------------------------------------------------
// adjoint: material derivative (ElasticForceDerivative.cpp:91-132)
// ---------------------------------------------------------------------------
template <class EL, int NT>
__global__ void __launch_bounds__(NT) k_material_vjp(DevMesh m, const double *__restrict__ u,
													 const double *__restrict__ adj, double *__restrict__ out)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	double Xg[EL::NG][3];
	double U[EL::N][3], Pn[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, double>(m, e, Xg);
	load_nodal<EL, double>(m, e, u, U, nodes);
	load_nodal<EL, double>(m, e, adj, Pn, nodes);
	double Jit[3][3];
	double detJ = 0.0;
	if constexpr (EL::AFFINE) geometry<EL, double>(0, Xg, Jit, detJ);
	double tl = 0.0, tm = 0.0;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		if constexpr (!EL::AFFINE) geometry<EL, double>(q, Xg, Jit, detJ);
		double gphi[EL::N][3];
		phys_grads<EL, double>(q, Jit, gphi);
		double F[3][3], Gp[3][3];
		disp_grad<EL, double>(U, gphi, F);
		disp_grad<EL, double>(Pn, gphi, Gp);
#pragma unroll
		for (int r = 0; r < 3; ++r) F[r][r] += 1.0;
		const double J = det3(F);
		double FmT[3][3];
		inv_transpose3(F, J, FmT);
		const double lj = log(J);
		double imu = 0.0, ila = 0.0;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				imu += (F[r][c] - FmT[r][c]) * Gp[r][c];
				ila += FmT[r][c] * Gp[r][c];
			}
		const double da = detJ * qweight<EL>(q);
		tl -= lj * ila * da;
		tm -= imu * da;
	}
	out[e] = tl;
	out[(size_t)m.E + e] = tm;
}

// ---------------------------------------------------------------------------
// adjoint: shape derivative (ElasticForceDerivative.cpp:207-260), with the
// stress-gradient product of compute_stress_grad_multiply_mat
// (NeoHookeanElasticity.cpp:660-680) reduced to vector identities for the
// rank-one perturbation V = e_d (x) grad(phi^g_v):
//   R:grad p  = mu a.(Gp g) + (mu - lambda lnJ)(F^-T g).(Gp F^-1 a) + lambda (a.F^-T g)(F^-T:Gp)
//   (P V^T - tr(V) P):grad p = (P g).Gp[:,d] - g_d (P:Gp),     a = Gu[:,d]
// ---------------------------------------------------------------------------
template <class EL, class T, int NT>
__global__ void __launch_bounds__(NT) k_shape_vjp(DevMesh m, const double *__restrict__ u,
												  const double *__restrict__ adj, double *__restrict__ out)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	T Xg[EL::NG][3];
	T U[EL::N][3], Pn[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, T>(m, e, Xg);
	load_nodal<EL, T>(m, e, u, U, nodes);
	load_nodal<EL, T>(m, e, adj, Pn, nodes);
	int gnodes[EL::NG];
#pragma unroll
	for (int j = 0; j < EL::NG; ++j) gnodes[j] = __ldg(m.gconn + (size_t)j * m.E + e);
	const double2 lm = __ldg(m.lame + e);
	const T lambda = T(lm.x), mu = T(lm.y);
	T acc[EL::NG][3];
#pragma unroll
	for (int j = 0; j < EL::NG; ++j) acc[j][0] = acc[j][1] = acc[j][2] = T(0);
	T Jit[3][3];
	double detJ = 0.0;
	if constexpr (EL::AFFINE) geometry<EL, T>(0, Xg, Jit, detJ);
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		if constexpr (!EL::AFFINE) geometry<EL, T>(q, Xg, Jit, detJ);
		T gphi[EL::N][3];
		phys_grads<EL, T>(q, Jit, gphi);
		T Gu[3][3], Gp[3][3], F[3][3];
		disp_grad<EL, T>(U, gphi, Gu);
		disp_grad<EL, T>(Pn, gphi, Gp);
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) F[r][c] = Gu[r][c] + (r == c ? T(1) : T(0));
		double J;
		if constexpr (sizeof(T) == 8)
			J = det3(F);
		else
		{
			double Fd[3][3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) Fd[r][c] = F[r][c];
			J = det3(Fd);
		}
		const T lj = T(log(J));
		T FmT[3][3];
		inv_transpose3(F, T(J), FmT);
		T P[3][3];
		T PGp = T(0), FGp = T(0);
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				P[r][c] = mu * (F[r][c] - FmT[r][c]) + lambda * lj * FmT[r][c];
				PGp += P[r][c] * Gp[r][c];
				FGp += FmT[r][c] * Gp[r][c];
			}
		// F^-1 a for each column a = Gu[:,d]: (F^-1 a)_j = sum_i FmT[i][j] a_i
		T Fia[3][3]; // [d][j]
#pragma unroll
		for (int d = 0; d < 3; ++d)
#pragma unroll
			for (int j = 0; j < 3; ++j) Fia[d][j] = FmT[0][j] * Gu[0][d] + FmT[1][j] * Gu[1][d] + FmT[2][j] * Gu[2][d];
		const T da = T(detJ * qweight<EL>(q));
		const T cmix = mu - lambda * lj;
#pragma unroll
		for (int v = 0; v < EL::NG; ++v)
		{
			// physical gradient of the geometric basis function v
			T g[3];
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				T s = T(0);
#pragma unroll
				for (int r = 0; r < 3; ++r)
				{
					const double gr = ggref<EL>(q, v, r);
					if (gr != 0.0) s += T(gr) * Jit[r][c];
				}
				g[c] = s;
			}
			T Fg[3], Pg[3], Gpg[3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
			{
				Fg[r] = FmT[r][0] * g[0] + FmT[r][1] * g[1] + FmT[r][2] * g[2];
				Pg[r] = P[r][0] * g[0] + P[r][1] * g[1] + P[r][2] * g[2];
				Gpg[r] = Gp[r][0] * g[0] + Gp[r][1] * g[1] + Gp[r][2] * g[2];
			}
#pragma unroll
			for (int d = 0; d < 3; ++d)
			{
				const T a0 = Gu[0][d], a1 = Gu[1][d], a2 = Gu[2][d];
				// Gp * (F^-1 a)
				T t0 = Gp[0][0] * Fia[d][0] + Gp[0][1] * Fia[d][1] + Gp[0][2] * Fia[d][2];
				T t1 = Gp[1][0] * Fia[d][0] + Gp[1][1] * Fia[d][1] + Gp[1][2] * Fia[d][2];
				T t2 = Gp[2][0] * Fia[d][0] + Gp[2][1] * Fia[d][1] + Gp[2][2] * Fia[d][2];
				const T R = mu * (a0 * Gpg[0] + a1 * Gpg[1] + a2 * Gpg[2])
						  + cmix * (Fg[0] * t0 + Fg[1] * t1 + Fg[2] * t2)
						  + lambda * (a0 * Fg[0] + a1 * Fg[1] + a2 * Fg[2]) * FGp;
				const T tmp = Pg[0] * Gp[0][d] + Pg[1] * Gp[1][d] + Pg[2] * Gp[2][d] - g[d] * PGp;
				acc[v][d] -= (R + tmp) * da;
			}
		}
	}
#pragma unroll
	for (int v = 0; v < EL::NG; ++v)
#pragma unroll
		for (int d = 0; d < 3; ++d) atomicAdd(out + (size_t)gnodes[v] * 3 + d, double(acc[v][d]));
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline int blocks_for(int n, int nt) { return (n + nt - 1) / nt; }

template <class EL, class T>
static void energy_t(const DevMesh &m, const double *u, bool per_element, double *out, const Scratch &sc, cudaStream_t s)
{
	constexpr int NT = 256;
	const int nb = blocks_for(m.E, NT);
	if (per_element)
		k_energy_per_element<EL, T, NT><<<nb, NT, 0, s>>>(m, u, out, sc.inverted);
	else
		k_energy<EL, T, NT><<<nb, NT, 0, s>>>(m, u, sc.partials, out, sc.ticket, sc.inverted);
}

cudaError_t launch_energy(const DevMesh &m, const double *u, int prec, bool per_element, double *out,
						  const Scratch &sc, cudaStream_t s)
{
	if (m.E == 0)
		return per_element ? cudaSuccess : cudaMemsetAsync(out, 0, sizeof(double), s);
	const bool f32 = prec != PREC_FP64;
	switch (m.et)
	{
	case 1: f32 ? energy_t<P1Tet, float>(m, u, per_element, out, sc, s) : energy_t<P1Tet, double>(m, u, per_element, out, sc, s); break;
	case 2: f32 ? energy_t<P2Tet, float>(m, u, per_element, out, sc, s) : energy_t<P2Tet, double>(m, u, per_element, out, sc, s); break;
	case 3: f32 ? energy_t<Q1Hex, float>(m, u, per_element, out, sc, s) : energy_t<Q1Hex, double>(m, u, per_element, out, sc, s); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

template <class EL, class T>
static void gradient_t(const DevMesh &m, const double *u, double *g, const Scratch &sc, cudaStream_t s)
{
	constexpr int NT = 128;
	k_gradient<EL, T, NT><<<blocks_for(m.E, NT), NT, 0, s>>>(m, u, g, sc.inverted);
}

cudaError_t launch_gradient(const DevMesh &m, const double *u, int prec, double *g, const Scratch &sc, cudaStream_t s)
{
	cudaError_t err = cudaMemsetAsync(g, 0, sizeof(double) * 3 * (size_t)m.N, s);
	if (err != cudaSuccess || m.E == 0) return err;
	const bool f32 = prec != PREC_FP64;
	switch (m.et)
	{
	case 1: f32 ? gradient_t<P1Tet, float>(m, u, g, sc, s) : gradient_t<P1Tet, double>(m, u, g, sc, s); break;
	case 2: f32 ? gradient_t<P2Tet, float>(m, u, g, sc, s) : gradient_t<P2Tet, double>(m, u, g, sc, s); break;
	case 3: f32 ? gradient_t<Q1Hex, float>(m, u, g, sc, s) : gradient_t<Q1Hex, double>(m, u, g, sc, s); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

template <class EL, class T>
static cudaError_t hess_attr()
{
	return cudaFuncSetAttribute(k_hessian<EL, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(HessSmem<EL, T>));
}

cudaError_t hessian_kernel_setup(int)
{
	cudaError_t e;
	if ((e = hess_attr<P1Tet, double>()) != cudaSuccess) return e;
	if ((e = hess_attr<P1Tet, float>()) != cudaSuccess) return e;
	if ((e = hess_attr<P2Tet, double>()) != cudaSuccess) return e;
	if ((e = hess_attr<P2Tet, float>()) != cudaSuccess) return e;
	if ((e = hess_attr<Q1Hex, double>()) != cudaSuccess) return e;
	if ((e = hess_attr<Q1Hex, float>()) != cudaSuccess) return e;
	return cudaSuccess;
}

template <class EL, class T>
static void hessian_t(const DevMesh &m, const DevPattern &p, const double *u, cudaStream_t s)
{
	using TL = HessTile<EL>;
	const int nb = blocks_for(m.E, TL::TE);
	k_hessian<EL, T><<<nb, TL::NT, sizeof(HessSmem<EL, T>), s>>>(m, p, u);
}

cudaError_t launch_hessian(const DevMesh &m, const DevPattern &p, const double *u, int prec, cudaStream_t s)
{
	cudaError_t err = cudaMemsetAsync(p.values, 0, sizeof(double) * (size_t)p.nnz, s);
	if (err != cudaSuccess || m.E == 0) return err;
	const bool f32 = prec != PREC_FP64;
	switch (m.et)
	{
	case 1: f32 ? hessian_t<P1Tet, float>(m, p, u, s) : hessian_t<P1Tet, double>(m, p, u, s); break;
	case 2: f32 ? hessian_t<P2Tet, float>(m, p, u, s) : hessian_t<P2Tet, double>(m, p, u, s); break;
	case 3: f32 ? hessian_t<Q1Hex, float>(m, p, u, s) : hessian_t<Q1Hex, double>(m, p, u, s); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

cudaError_t launch_material_vjp(const DevMesh &m, const double *u, const double *adj, double *out, cudaStream_t s)
{
	if (m.E == 0) return cudaSuccess;
	constexpr int NT = 128;
	const int nb = blocks_for(m.E, NT);
	switch (m.et)
	{
	case 1: k_material_vjp<P1Tet, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	case 2: k_material_vjp<P2Tet, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	case 3: k_material_vjp<Q1Hex, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

cudaError_t launch_shape_vjp(const DevMesh &m, const double *u, const double *adj, int prec, double *out, cudaStream_t s)
{
	cudaError_t err = cudaMemsetAsync(out, 0, sizeof(double) * 3 * (size_t)m.Ng, s);
	if (err != cudaSuccess || m.E == 0) return err;
	constexpr int NT = 128;
	const int nb = blocks_for(m.E, NT);
	const bool f32 = prec != PREC_FP64;
	switch (m.et)
	{
	case 1: f32 ? k_shape_vjp<P1Tet, float, NT><<<nb, NT, 0, s>>>(m, u, adj, out) : k_shape_vjp<P1Tet, double, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	case 2: f32 ? k_shape_vjp<P2Tet, float, NT><<<nb, NT, 0, s>>>(m, u, adj, out) : k_shape_vjp<P2Tet, double, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	case 3: f32 ? k_shape_vjp<Q1Hex, float, NT><<<nb, NT, 0, s>>>(m, u, adj, out) : k_shape_vjp<Q1Hex, double, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

} // namespace pfg
