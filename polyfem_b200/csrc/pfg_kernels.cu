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
#include "pfg_device.cuh"

#include <cstdio>
#include <cstdlib>

namespace pfg
{

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

// P1 elements are small enough for four 256-thread CTAs per SM (64 registers)
template <class EL>
constexpr int elem_kernel_min_ctas()
{
	return EL::ET == 1 ? 4 : 1;
}

template <class EL, class T, int NT>
__global__ void __launch_bounds__(NT, elem_kernel_min_ctas<EL>()) k_energy(DevMesh m, const double *__restrict__ u, double *__restrict__ partials,
											   double *__restrict__ result, unsigned int *ticket,
											   unsigned long long *inverted)
{
	// grid-stride: a resident grid, each thread summing its elements in order, so the
	// block reduction and the partials' tail are paid once per resident block
	double en = 0.0;
	for (int e = blockIdx.x * NT + threadIdx.x; e < m.E; e += gridDim.x * NT) en += element_energy<EL, T>(m, u, e, inverted);
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
__global__ void __launch_bounds__(NT, EL::ET == 1 ? 8 : 1) k_gradient(DevMesh m, const double *__restrict__ u, double *__restrict__ stage,
												 unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	// The displacement gradient grad u = sum_a u_a (x) grad(phi_a) is formed in FP64
	// in every mode: it is a difference of nearby nodal values, and rounding u or
	// J^-T to FP32 first costs ~3x in the FP32 gradient's error on smooth fields.
	// The stress and its contraction then run in T.
	double Xg[EL::NG][3];
	double U[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, double>(m, e, Xg);
	load_nodal<EL, double>(m, e, u, U, nodes);
	const double2 lm = __ldg(m.lame + e);
	const double lambda = lm.x, mu = lm.y;
	// element gradient, accumulated as G[a][d] = sum_q sum_r gref(q,a,r) (da P J^-1)[d][r]
	// so the physical basis gradients are never materialised
	T Gacc[EL::N][3];
#pragma unroll
	for (int a = 0; a < EL::N; ++a) Gacc[a][0] = Gacc[a][1] = Gacc[a][2] = T(0);
	double Jitd[3][3];
	double detJ = 0.0;
	if constexpr (EL::AFFINE) geometry<EL, double>(0, Xg, Jitd, detJ);
	bool bad = false;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		if constexpr (!EL::AFFINE) geometry<EL, double>(q, Xg, Jitd, detJ);
		T Jit[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) Jit[r][c] = T(Jitd[r][c]);
		double A[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				double s = 0.0;
#pragma unroll
				for (int a = 0; a < EL::N; ++a)
				{
					const double gr = gref<EL>(q, a, c);
					if (gr != 0.0) s += U[a][r] * gr;
				}
				A[r][c] = s;
			}
		T F[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
				F[r][c] = T(A[r][0] * Jitd[0][c] + A[r][1] * Jitd[1][c] + A[r][2] * Jitd[2][c]) + (r == c ? T(1) : T(0));
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
	// the element's contributions, one 32-byte slot per incidence (e, a) at the
	// incidence's position in node order: (G0, G1, G2, 0)
#pragma unroll
	for (int a = 0; a < EL::N; ++a)
	{
		const int k = __ldg(m.eb_inc + (size_t)e * EL::N + a);
		st_slot(stage + (size_t)k * 4, double(Gacc[a][0]), double(Gacc[a][1]), double(Gacc[a][2]));
	}
}

// Per node: the sum of its incidences' contributions in incidence (element) order
// (NLAssembler::assemble_gradient's scatter, Assembler.cpp:613-629), one thread per
// node.  The slots are in node order, so a node's incidences are one contiguous
// run; loads are issued eight slots at a time.  Deterministic.
template <int NT>
__global__ void __launch_bounds__(NT) k_vec_gather(int n_nodes, const int *__restrict__ off,
												   const double *__restrict__ stage, double *__restrict__ out)
{
	constexpr int BATCH = 8;
	const int B = blockIdx.x * NT + threadIdx.x;
	if (B >= n_nodes) return;
	const int k0 = __ldg(off + B), k1 = __ldg(off + B + 1);
	const double2 *slots = reinterpret_cast<const double2 *>(stage);
	double t0 = 0.0, t1 = 0.0, t2 = 0.0;
	for (int kb = k0; kb < k1; kb += BATCH)
	{
		double2 x[BATCH], y[BATCH];
#pragma unroll
		for (int j = 0; j < BATCH; ++j)
			if (kb + j < k1)
			{
				x[j] = __ldg(slots + 2 * (size_t)(kb + j));
				y[j] = __ldg(slots + 2 * (size_t)(kb + j) + 1);
			}
#pragma unroll
		for (int j = 0; j < BATCH; ++j)
			if (kb + j < k1)
			{
				t0 += x[j].x;
				t1 += x[j].y;
				t2 += y[j].x;
			}
	}
	out[(size_t)B * 3 + 0] = t0;
	out[(size_t)B * 3 + 1] = t1;
	out[(size_t)B * 3 + 2] = t2;
}

// The same sums with G lanes per node: lane l loads slots l, l + G, ... of the
// node's contiguous run (consecutive lanes on consecutive 32-byte slots), sums
// them in that order, and the G partial sums meet in a fixed butterfly.  The
// order is fixed, so the result is deterministic.  Used when a node has many
// incidences on average (P1: ~19), where one thread per node queues too many
// loads per thread.
template <int G, int NT>
__global__ void __launch_bounds__(NT) k_vec_gather_group(int n_nodes, const int *__restrict__ off,
														 const double *__restrict__ stage, double *__restrict__ out)
{
	static_assert(G == 8 || G == 16 || G == 32, "node groups are aligned parts of a warp");
	const int t = blockIdx.x * NT + threadIdx.x;
	const int B = t / G, l = t % G;
	if (B >= n_nodes) return; // whole groups leave together: n_nodes is per group
	const unsigned mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
	const int k0 = __ldg(off + B), k1 = __ldg(off + B + 1);
	const double2 *slots = reinterpret_cast<const double2 *>(stage);
	double t0 = 0.0, t1 = 0.0, t2 = 0.0;
	for (int k = k0 + l; k < k1; k += G)
	{
		const double2 x = __ldg(slots + 2 * (size_t)k);
		const double2 y = __ldg(slots + 2 * (size_t)k + 1);
		t0 += x.x;
		t1 += x.y;
		t2 += y.x;
	}
#pragma unroll
	for (int o = G / 2; o > 0; o >>= 1)
	{
		t0 += __shfl_xor_sync(mask, t0, o);
		t1 += __shfl_xor_sync(mask, t1, o);
		t2 += __shfl_xor_sync(mask, t2, o);
	}
	if (l == 0)
	{
		out[(size_t)B * 3 + 0] = t0;
		out[(size_t)B * 3 + 1] = t1;
		out[(size_t)B * 3 + 2] = t2;
	}
}

__host__ __device__ constexpr int nodes_of(int et) { return et == 1 ? 4 : et == 2 ? 10 : 8; }
__host__ __device__ constexpr int geom_nodes_of(int et) { return et == 3 ? 8 : 4; }

// Per-node sums of one 32-byte slot per incidence: a G-lane group per node when
// nodes average more than 12 incidences, else one thread per node.
static void launch_vec_gather(int n_nodes, const int *off, long long n_inc, const double *stage, double *out,
							  cudaStream_t s)
{
	if (n_nodes <= 0) return;
	constexpr int NT = 128;
	if (n_inc > 12LL * n_nodes)
	{
		constexpr int G = 32;
		k_vec_gather_group<G, NT><<<(int)(((long long)n_nodes * G + NT - 1) / NT), NT, 0, s>>>(n_nodes, off, stage, out);
	}
	else
		k_vec_gather<NT><<<(n_nodes + NT - 1) / NT, NT, 0, s>>>(n_nodes, off, stage, out);
}

// ---------------------------------------------------------------------------
// Hessian (NLAssembler::assemble_hessian + SparseMatrixCache)
//
// Element block.  With g_a = grad(phi_a), d_a = F^-T g_a and the identity
// F (g_a x g_b) = (cof F g_a) x (cof F g_b) / J (cof cof F = J F), the
// reference's B^T C B (NeoHookeanElasticity.cpp:636-656) reduces exactly to
//   H_ab = sum_q da [ mu (g_a.g_b) I + lambda d_a d_b^T + (mu - lambda ln J) d_b d_a^T ].
//
// Assembly in two passes, both without atomics:
//  1. k_hessian_blocks: a tile of elements per CTA computes the symmetric node
//     blocks (a, b), a <= b, once each and writes every element's blocks as one
//     packed upper triangle (tri_index order, [c][r] = H_e(3a+r, 3b+c)), a
//     contiguous run of whole sectors per element.
//  2. k_hessian_reduce: one warp per column node B reads, through the reduction
//     plan built with the pattern (for each row rank, the staged blocks that land
//     on it; block (b, a) read transposed for a > b), the blocks of B's
//     incidences, sums every CSC entry in registers in incidence order and writes
//     B's three columns once.  Each CSC entry is summed in a fixed order: the
//     result is deterministic.  An off-diagonal block is read by the warps of both
//     its nodes, the second time mostly from L2.
// ---------------------------------------------------------------------------
// Per (element, point) kinematics in the contraction type T, in 16-byte groups:
// [mu da, lambda da, (mu - lambda lnJ) da, -], then for every local node a at
// 4 + NS*a the vectors g_a and d_a: FP32 [g0 g1 g2 - | d0 d1 d2 -] (NS = 8,
// two 16-byte loads), FP64 [g0 g1 | g2 d0 | d1 d2] (NS = 6, three).
template <class EL, class T>
struct BlockKin
{
	static constexpr int NS = sizeof(T) == 8 ? 6 : 8;
	static constexpr int PER_Q = 4 + NS * EL::N;
};

__device__ __forceinline__ void ld_w(const float *p, float w[3])
{
	const float4 x = *reinterpret_cast<const float4 *>(p);
	w[0] = x.x;
	w[1] = x.y;
	w[2] = x.z;
}
__device__ __forceinline__ void ld_w(const double *p, double w[3])
{
	const double2 x = *reinterpret_cast<const double2 *>(p);
	w[0] = x.x;
	w[1] = x.y;
	w[2] = p[2];
}
__device__ __forceinline__ void ld_gd(const float *p, float g[3], float d[3])
{
	const float4 x = *reinterpret_cast<const float4 *>(p);
	const float4 y = *reinterpret_cast<const float4 *>(p + 4);
	g[0] = x.x;
	g[1] = x.y;
	g[2] = x.z;
	d[0] = y.x;
	d[1] = y.y;
	d[2] = y.z;
}
__device__ __forceinline__ void ld_gd(const double *p, double g[3], double d[3])
{
	const double2 x = *reinterpret_cast<const double2 *>(p);
	const double2 y = *reinterpret_cast<const double2 *>(p + 2);
	const double2 z = *reinterpret_cast<const double2 *>(p + 4);
	g[0] = x.x;
	g[1] = x.y;
	g[2] = y.x;
	d[0] = y.y;
	d[1] = z.x;
	d[2] = z.y;
}
__device__ __forceinline__ void st_gd(float *p, const float g[3], const float d[3])
{
	*reinterpret_cast<float4 *>(p) = make_float4(g[0], g[1], g[2], 0.f);
	*reinterpret_cast<float4 *>(p + 4) = make_float4(d[0], d[1], d[2], 0.f);
}
__device__ __forceinline__ void st_gd(double *p, const double g[3], const double d[3])
{
	*reinterpret_cast<double2 *>(p) = make_double2(g[0], g[1]);
	*reinterpret_cast<double2 *>(p + 2) = make_double2(g[2], d[0]);
	*reinterpret_cast<double2 *>(p + 4) = make_double2(d[1], d[2]);
}


// elements per tile of k_hessian_blocks (four warps, each takes a quarter)
#ifndef PFG_TE_P1
#define PFG_TE_P1 64
#endif
#ifndef PFG_TE_P2
#define PFG_TE_P2 16
#endif
#ifndef PFG_TE_Q1
#define PFG_TE_Q1 8
#endif
template <class EL, class T>
struct EcTile
{
	static constexpr int TE = (EL::ET == 1) ? PFG_TE_P1 : (EL::ET == 2 ? PFG_TE_P2 : PFG_TE_Q1);
	static constexpr int NT = 128;
	static constexpr int N = EL::N, NG = EL::NG, NQ = EL::NQ;
	static constexpr int NP = N * (N + 1) / 2, NB = N * N, PQ = BlockKin<EL, T>::PER_Q, NS = BlockKin<EL, T>::NS;
	// A lane computes a group of NPB pairs (a, b), (a, b + 1), .. of one row node a:
	// two for Q1 (its 36 pairs in one round of 20 lanes, the row node's vectors loaded
	// once for both), one for P1 and P2 (measured: no gain for P2, a loss for P1).
	static constexpr int NPB = EL::ET == 3 ? 2 : 1;
	static constexpr int NPG = []() { int s = 0; for (int a = 0; a < N; ++a) s += (N - a + NPB - 1) / NPB; return s; }();
};

// g_a = grad(phi_a) J^-T and d_a = F^-T g_a in K, stored rounded to T at dst
template <class EL, class K, class T>
__device__ __forceinline__ void node_kin(const K gr[3], const K Jit[3][3], const K FmT[3][3], T *dst)
{
	K g[3];
#pragma unroll
	for (int c = 0; c < 3; ++c) g[c] = gr[0] * Jit[0][c] + gr[1] * Jit[1][c] + gr[2] * Jit[2][c];
	T gt[3], dt[3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
	{
		gt[r] = T(g[r]);
		dt[r] = T(FmT[r][0] * g[0] + FmT[r][1] * g[1] + FmT[r][2] * g[2]);
	}
	st_gd(dst, gt, dt);
}

// Block of node pair (a, b) of one element from its per-point kinematics:
//   h[r][c] = sum_q [ mu da (g_a.g_b) delta_rc + lambda da d_a[r] d_b[c] + (mu - lambda lnJ) da d_b[r] d_a[c] ]
// In FP32 the row pairs (0,1) of every column and the column pair (0,1) of row
// 2's partner are updated with packed FP32x2 FMAs; each entry sees the same
// operations in the same order as the scalar form.
// The blocks (a, b[j]), j < NPB, of one row node a: the weights, g_a, d_a and the
// products lambda da d_a, (mu - lambda lnJ) da d_a are loaded or formed once per
// point for all NPB partners.
template <class EL, class T, int NPB>
__device__ __forceinline__ void block_pairs(const T (*kin)[BlockKin<EL, T>::PER_Q], int a, const int (&b)[NPB],
											T (&h)[NPB][3][3])
{
	constexpr int NS = BlockKin<EL, T>::NS;
	if constexpr (sizeof(T) == 4)
	{
		float2 h0[NPB], h1[NPB], hc[NPB]; // (h00,h01) (h10,h11) (h02,h12)
		float h20[NPB], h21[NPB], h22[NPB];
#pragma unroll
		for (int j = 0; j < NPB; ++j)
		{
			h0[j] = h1[j] = hc[j] = make_float2(0.f, 0.f);
			h20[j] = h21[j] = h22[j] = 0.f;
		}
#pragma unroll
		for (int q = 0; q < EL::NQ; ++q)
		{
			const T *Kq = kin[q];
			T w[3], ga[3], da[3];
			ld_w(Kq, w);
			ld_gd(Kq + 4 + NS * a, ga, da);
			const float la0 = w[1] * da[0], la1 = w[1] * da[1], la2 = w[1] * da[2];
			const float gm0 = w[2] * da[0], gm1 = w[2] * da[1], gm2 = w[2] * da[2];
			const float2 gm01 = make_float2(gm0, gm1);
#pragma unroll
			for (int j = 0; j < NPB; ++j)
			{
				T gb[3], db[3];
				ld_gd(Kq + 4 + NS * b[j], gb, db);
				const float md = w[0] * (ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2]);
				const float2 db01 = make_float2(db[0], db[1]);
				// rows 0 and 1, columns 0 and 1
				h0[j] = __ffma2_rn(make_float2(db[0], db[0]), gm01, __ffma2_rn(make_float2(la0, la0), db01, h0[j]));
				h1[j] = __ffma2_rn(make_float2(db[1], db[1]), gm01, __ffma2_rn(make_float2(la1, la1), db01, h1[j]));
				// column 2 of rows 0 and 1
				hc[j] = __ffma2_rn(make_float2(db[0], db[1]), make_float2(gm2, gm2),
								   __ffma2_rn(make_float2(la0, la1), make_float2(db[2], db[2]), hc[j]));
				// row 2
				h20[j] = fmaf(db[2], gm0, fmaf(la2, db[0], h20[j]));
				h21[j] = fmaf(db[2], gm1, fmaf(la2, db[1], h21[j]));
				h22[j] = fmaf(db[2], gm2, fmaf(la2, db[2], h22[j]));
				h0[j].x += md;
				h1[j].y += md;
				h22[j] += md;
			}
		}
#pragma unroll
		for (int j = 0; j < NPB; ++j)
		{
			h[j][0][0] = h0[j].x;
			h[j][0][1] = h0[j].y;
			h[j][1][0] = h1[j].x;
			h[j][1][1] = h1[j].y;
			h[j][0][2] = hc[j].x;
			h[j][1][2] = hc[j].y;
			h[j][2][0] = h20[j];
			h[j][2][1] = h21[j];
			h[j][2][2] = h22[j];
		}
	}
	else
	{
#pragma unroll
		for (int j = 0; j < NPB; ++j)
#pragma unroll
			for (int r = 0; r < 3; ++r) h[j][r][0] = h[j][r][1] = h[j][r][2] = T(0);
#pragma unroll
		for (int q = 0; q < EL::NQ; ++q)
		{
			const T *Kq = kin[q];
			T w[3], ga[3], da[3];
			ld_w(Kq, w);
			ld_gd(Kq + 4 + NS * a, ga, da);
			const T la[3] = {w[1] * da[0], w[1] * da[1], w[1] * da[2]};
			const T gma[3] = {w[2] * da[0], w[2] * da[1], w[2] * da[2]};
#pragma unroll
			for (int j = 0; j < NPB; ++j)
			{
				T gb[3], db[3];
				ld_gd(Kq + 4 + NS * b[j], gb, db);
				const T md = w[0] * (ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2]);
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int c = 0; c < 3; ++c) h[j][r][c] = fma(db[r], gma[c], fma(la[r], db[c], h[j][r][c]));
				h[j][0][0] += md;
				h[j][1][1] += md;
				h[j][2][2] += md;
			}
		}
	}
}

// K: arithmetic of the kinematics (J^-T, F, F^-T, g, d); T: arithmetic of the
// contraction and the records (g, d and the weights are stored rounded to T)
template <class EL, class K, class T>
struct EcSmem
{
	using TL = EcTile<EL, T>;
	// one element's block triangle per warp (tri_pad values, copied out in 16-byte
	// vectors); before the blocks it holds the warp's J^-T and F^-T in K
	static constexpr int TP = tri_pad(TL::N), VW = 16 / (int)sizeof(T);
	static constexpr int JF_T = (int)(((TL::TE / (TL::NT / 32)) * TL::NQ * 18 * sizeof(K) + sizeof(T) - 1) / sizeof(T));
	static constexpr int TB = ((TP > JF_T ? TP : JF_T) + VW - 1) / VW * VW;
	__align__(16) T rec[TL::NT / 32][TB];
	__align__(16) T kin[TL::TE][TL::NQ][TL::PQ];
	K U[TL::TE][TL::N][3];
	K X[TL::TE][TL::NG][3];
	// reference gradients of the FE and geometric bases and the weights, indexed at
	// run time so that lanes at different quadrature points share one code path
	K gtab[TL::NQ][TL::N][3];
	K ggtab[EL::AFFINE ? 1 : TL::NQ][TL::NG][3];
	double wq[TL::NQ];
	int nodes[TL::TE][TL::N + TL::NG];
	unsigned char grp_a[TL::NPG], grp_b[TL::NPG]; // pair group: row node, first column node
};

// CTAs per SM the shared-memory footprint allows; the register budget follows it
#ifndef PFG_BLOCKS_CTAS_F32
#define PFG_BLOCKS_CTAS_F32 6
#endif
#ifndef PFG_BLOCKS_CTAS_F64
#define PFG_BLOCKS_CTAS_F64 5
#endif
template <class EL, class K, class T>
constexpr int blocks_min_ctas()
{
	constexpr int by_smem = (int)((227 * 1024) / (sizeof(EcSmem<EL, K, T>) + 1024));
	constexpr int cap = sizeof(T) == 8 ? PFG_BLOCKS_CTAS_F64 : PFG_BLOCKS_CTAS_F32;
	return by_smem < 1 ? 1 : (by_smem < cap ? by_smem : cap);
}

template <class EL, class K, class T>
__global__ void __launch_bounds__(128, blocks_min_ctas<EL, K, T>())
	k_hessian_blocks(DevMesh m, const double *__restrict__ u, T *__restrict__ stage, int e_begin, int e_end)
{
	using TL = EcTile<EL, T>;
	constexpr int TE = TL::TE, NT = TL::NT, N = TL::N, NG = TL::NG, NQ = TL::NQ;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	EcSmem<EL, K, T> &S = *reinterpret_cast<EcSmem<EL, K, T> *>(smem_raw);
	const int tid = threadIdx.x;
	const int e0 = e_begin + blockIdx.x * TE;
	const int ne = min(TE, e_end - e0);

	// basis tables and node-pair table, shared by the CTA's warps
	constexpr int GQ = EL::AFFINE ? 1 : NQ;
	if (tid < NQ)
	{
#pragma unroll
		for (int qq = 0; qq < NQ; ++qq)
		{
			if (qq != tid) continue;
#pragma unroll
			for (int a = 0; a < N; ++a)
#pragma unroll
				for (int r = 0; r < 3; ++r) S.gtab[qq][a][r] = K(gref<EL>(qq, a, r));
			if (qq < GQ)
			{
#pragma unroll
				for (int j = 0; j < NG; ++j)
#pragma unroll
					for (int r = 0; r < 3; ++r) S.ggtab[qq][j][r] = K(ggref<EL>(qq, j, r));
			}
			S.wq[qq] = qweight<EL>(qq);
		}
	}
	for (int g = tid; g < TL::NPG; g += NT)
	{
		int a = 0, r = g;
		while (r >= (N - a + TL::NPB - 1) / TL::NPB)
		{
			r -= (N - a + TL::NPB - 1) / TL::NPB;
			++a;
		}
		S.grp_a[g] = (unsigned char)a;
		S.grp_b[g] = (unsigned char)(a + TL::NPB * r);
	}
	__syncthreads();

	// From here each warp runs its own WE elements of the tile end to end (gathers,
	// kinematics, blocks, records) with warp-level synchronisation only, so the
	// warps of a CTA overlap one another's memory waits.
	constexpr int WPC = NT / 32, WE = TE / WPC;
	static_assert(TE % WPC == 0, "tile must split evenly over the warps");
	const int warp = tid >> 5, lane = tid & 31;
	const int w0 = warp * WE;
	const int wn = max(0, min(WE, ne - w0));
	for (int i = lane; i < WE * (N + NG); i += 32)
	{
		const int j = i / WE, el = w0 + i % WE, e = e0 + el;
		int v = 0;
		if (el - w0 < wn) v = (j < N) ? __ldg(m.conn + (size_t)j * m.E + e) : __ldg(m.gconn + (size_t)(j - N) * m.E + e);
		S.nodes[el][j] = v;
	}
	__syncwarp();
	for (int i = lane; i < WE * N * 3; i += 32)
	{
		const int el = w0 + i / (N * 3), a = (i / 3) % N, d = i % 3;
		S.U[el][a][d] = (el - w0 < wn) ? K(__ldg(u + (size_t)S.nodes[el][a] * 3 + d)) : K(0);
	}
	for (int i = lane; i < WE * NG * 3; i += 32)
	{
		const int el = w0 + i / (NG * 3), j = (i / 3) % NG, d = i % 3;
		S.X[el][j][d] = (el - w0 < wn) ? K(__ldg(m.X + (size_t)S.nodes[el][N + j] * 3 + d)) : K(0);
	}
	__syncwarp();

	// per (element, quadrature point): J^-T, F, det/log J and F^-T in K, then the
	// weights and, for every local node, g_a = grad(phi_a) J^-T and d_a = F^-T g_a,
	// stored rounded to T.  When J^-T and F^-T of the warp's points fit in its
	// (still unused) record buffer, the per-node vectors are a second step over
	// (element, point, node) so that every lane has work.
	constexpr bool SPLIT_KIN = true; // the warp's buffer is sized for J^-T and F^-T
	K *JF = reinterpret_cast<K *>(S.rec[warp]); // [WE * NQ][18]: J^-T, then F^-T
	for (int i = lane; i < wn * NQ; i += 32)
	{
		const int el = w0 + i / NQ, q = i % NQ;
		const double2 lm = __ldg(m.lame + e0 + el);
		T *Kq = S.kin[el][q];
		const K(*gq)[3] = S.gtab[q];
		const K(*gg)[3] = S.ggtab[EL::AFFINE ? 0 : q];
		// geometry: J = sum_j grad(psi_j) (x) X_j, rows d/dxi_r (ElementAssemblyValues.cpp:88-93)
		K Jac[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				K s_ = K(0);
#pragma unroll
				for (int j = 0; j < NG; ++j) s_ += gg[j][r] * S.X[el][j][c];
				Jac[r][c] = s_;
			}
		K Jit[3][3];
		double detJ;
		if constexpr (sizeof(K) == 8)
		{
			detJ = det3(Jac);
			inv_transpose3(Jac, K(detJ), Jit);
		}
		else
		{
			double Jd[3][3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) Jd[r][c] = double(Jac[r][c]);
			detJ = det3(Jd);
			inv_transpose3(Jac, K(detJ), Jit);
		}
		K Ar[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				K s_ = K(0);
#pragma unroll
				for (int a = 0; a < N; ++a) s_ += S.U[el][a][r] * gq[a][c];
				Ar[r][c] = s_;
			}
		K F[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
				F[r][c] = Ar[r][0] * Jit[0][c] + Ar[r][1] * Jit[1][c] + Ar[r][2] * Jit[2][c] + (r == c ? K(1) : K(0));
		double J;
		if constexpr (sizeof(K) == 8)
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
		const double da = detJ * S.wq[q];
		K FmT[3][3];
		inv_transpose3(F, K(J), FmT);
		Kq[0] = T(lm.y * da);
		Kq[1] = T(lm.x * da);
		Kq[2] = T((lm.y - lm.x * lj) * da);
		Kq[3] = T(0);
		if constexpr (SPLIT_KIN)
		{
			K *jf = JF + i * 18;
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c)
				{
					jf[r * 3 + c] = Jit[r][c];
					jf[9 + r * 3 + c] = FmT[r][c];
				}
		}
		else
		{
#pragma unroll
			for (int a = 0; a < N; ++a) node_kin<EL, K, T>(gq[a], Jit, FmT, Kq + 4 + TL::NS * a);
		}
	}
	__syncwarp();
	if constexpr (SPLIT_KIN)
	{
		// g_a and d_a of every (element, point, node) of the warp, all lanes busy
		for (int t = lane; t < wn * NQ * N; t += 32)
		{
			const int iq = t / N, a = t - iq * N;
			const int el = w0 + iq / NQ, q = iq % NQ;
			const K *jf = JF + iq * 18;
			K Jit[3][3], FmT[3][3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c)
				{
					Jit[r][c] = jf[r * 3 + c];
					FmT[r][c] = jf[9 + r * 3 + c];
				}
			node_kin<EL, K, T>(S.gtab[q][a], Jit, FmT, S.kin[el][q] + 4 + TL::NS * a);
		}
		__syncwarp();
	}

	// blocks: the warp takes its elements one at a time; every lane computes the
	// blocks of its pair group and writes them to the warp's triangle buffer, block
	// (a, b) at 9 * tri_index(a, b) as [c][r]; the triangle then goes to
	// stage[e * TP] in 16-byte vectors (padding included)
	constexpr int TP = EcSmem<EL, K, T>::TP, VW = EcSmem<EL, K, T>::VW, NPB = TL::NPB, NPG = TL::NPG;
	static_assert(TP % VW == 0, "triangles must be whole 16-byte vectors");
	T *R = S.rec[warp];
	for (int el = w0; el < w0 + wn; ++el)
	{
		for (int g = lane; g < NPG; g += 32)
		{
			const int a = S.grp_a[g], b0 = S.grp_b[g];
			int bb[NPB];
#pragma unroll
			for (int j = 0; j < NPB; ++j) bb[j] = b0 + j < N ? b0 + j : b0; // past a row's end: recomputed, not stored
			T h[NPB][3][3];
			block_pairs<EL, T, NPB>(S.kin[el], a, bb, h);
			T *Hab = R + 9 * tri_index(N, a, b0); // the group's blocks are tri_index neighbours
#pragma unroll
			for (int j = 0; j < NPB; ++j)
				if (b0 + j < N)
				{
#pragma unroll
					for (int r = 0; r < 3; ++r)
#pragma unroll
						for (int c = 0; c < 3; ++c) Hab[9 * j + c * 3 + r] = h[j][r][c];
				}
		}
		__syncwarp();
		uint4 *dst = reinterpret_cast<uint4 *>(stage + (size_t)(e0 + el) * TP);
		const uint4 *src = reinterpret_cast<const uint4 *>(R);
		for (int i = lane; i < TP / VW; i += 32) dst[i] = src[i];
		__syncwarp();
	}
}

// One warp per column node B; the warp's 3*deg(B) work items are the (row rank,
// column c) pairs of B's column block.  Each item sums, in FP64 and in incidence
// order, the three values (rows 3*rank .. 3*rank+2 of column 3B+c) of every
// staged block that lands on its rank, read through the reduction plan
// (consecutive values of block (a, b); for a flagged transposed block (b, a), the
// values c, c+3, c+6), and writes them once.  No shared memory, no atomics: the
// sum order of every entry is fixed.
template <class EL, class T, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 8)
	k_hessian_reduce(DevMesh m, DevPattern pat, const T *__restrict__ stage)
{
	constexpr int N = EL::N;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int B = blockIdx.x * WARPS + warp;
	if (B >= m.N) return;
	const int o0 = __ldg(pat.outer + 3 * B);
	const int stride = __ldg(pat.outer + 3 * B + 1) - o0; // 3 * deg(B)
	const int deg = stride / 3;
	const int s0 = __ldg(m.inc_off + B), s1 = __ldg(m.inc_off + B + 1);
	const int tot = (s1 - s0) * N;
	const unsigned *cl = pat.contrib + (size_t)s0 * N;
	const unsigned short *br = pat.blk_rel + o0 / 9;
	double *dst = pat.values + o0;
	for (int it = lane; it < stride; it += 32)
	{
		// (rank, column) items rank-major: the three items of the diagonal block,
		// which has the longest contribution list, share one pass of the warp
		const int r = it / 3, c = it - 3 * r;
		const int k0 = __ldg(br + r);
		const int k1 = (r + 1 < deg) ? (int)__ldg(br + r + 1) : tot;
		double a0 = 0.0, a1 = 0.0, a2 = 0.0;
		// two contributions per step, the next step's plan entries loaded ahead;
		// the sum order stays k ascending
		unsigned qa = k0 < k1 ? __ldg(cl + k0) : 0u;
		unsigned qb = k0 + 1 < k1 ? __ldg(cl + k0 + 1) : 0u;
		for (int k = k0; k < k1; k += 2)
		{
			const unsigned q0 = qa, q1 = qb;
			const bool two = k + 1 < k1;
			qa = k + 2 < k1 ? __ldg(cl + k + 2) : 0u;
			qb = k + 3 < k1 ? __ldg(cl + k + 3) : 0u;
			// (a, b): values 3c, 3c+1, 3c+2 of the block; transposed (b, a): c, c+3, c+6
			const bool t0 = q0 & TRI_TRANSPOSED, t1 = q1 & TRI_TRANSPOSED;
			const T *p0 = stage + (q0 & ~TRI_TRANSPOSED) + (t0 ? c : 3 * c);
			const T *p1 = stage + (q1 & ~TRI_TRANSPOSED) + (t1 ? c : 3 * c);
			const int s0_ = t0 ? 3 : 1, s1_ = t1 ? 3 : 1;
			const T x0 = __ldg(p0), x1 = __ldg(p0 + s0_), x2 = __ldg(p0 + 2 * s0_);
			T y0 = T(0), y1 = T(0), y2 = T(0);
			if (two)
			{
				y0 = __ldg(p1);
				y1 = __ldg(p1 + s1_);
				y2 = __ldg(p1 + 2 * s1_);
			}
			a0 += double(x0);
			a1 += double(x1);
			a2 += double(x2);
			if (two)
			{
				a0 += double(y0);
				a1 += double(y1);
				a2 += double(y2);
			}
		}
		if (pat.red_col_start == nullptr)
		{
			double *d = dst + c * stride + 3 * r;
			d[0] = a0;
			d[1] = a1;
			d[2] = a2;
		}
		else
		{
			// Dirichlet-reduced output: free rows of free columns only
			const int cs = __ldg(pat.red_col_start + 3 * B + c);
			if (cs >= 0)
			{
				const unsigned short *ro = pat.red_row_off + o0 / 3 + 3 * r;
				const unsigned short r0 = __ldg(ro), r1 = __ldg(ro + 1), r2 = __ldg(ro + 2);
				if (r0 != 0xFFFF) pat.values[cs + r0] = a0;
				if (r1 != 0xFFFF) pat.values[cs + r1] = a1;
				if (r2 != 0xFFFF) pat.values[cs + r2] = a2;
			}
		}
	}
}

// Pass 2 of every Hessian-pattern assembly.
template <class EL, class T>
static cudaError_t launch_reduce(const DevMesh &m, const DevPattern &p, const T *stage, cudaStream_t s)
{
	if (m.N <= 0) return cudaSuccess;
	constexpr int WARPS = 8;
	k_hessian_reduce<EL, T, WARPS><<<(m.N + WARPS - 1) / WARPS, WARPS * 32, 0, s>>>(m, p, stage);
	return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// ipc::project_to_psd (PSDProjectionMethod::CLAMP), applied to every element
// matrix before the scatter when NLAssembler::assemble_hessian is called with
// project_to_psd (Assembler.cpp:693-694): A = Z diag(l) Z^T is replaced by
// Z diag(max(l, 0)) Z^T when its smallest eigenvalue is <= 0.  Equivalently
// A+ = A + sum_{l_j < 0} |l_j| z_j z_j^T, which needs only the eigenpairs with
// l_j < 0; this kernel computes those and nothing else.  One warp per element,
// all in FP64, on the element matrix rebuilt from its staged block triangle:
//   1. Householder reduction to tridiagonal T = Q^T A Q (EISPACK tred2 without
//      the accumulation of Q), lane j holding row j of A in registers and
//      applying the symmetric rank-2 update to its own row; the reflectors
//      u_i (with 1/h_i) stay in shared memory.
//   2. T is scaled by its Gershgorin bound ||T|| (so |l| <= 1) and the number k
//      of eigenvalues below -tau is one Sturm count (LDL^T sign count).
//      k == 0: the matrix counts as PSD and the staged blocks stay as they are.
//   3. The k eigenvalues by multisection: 32 / k lanes per eigenvalue each
//      evaluate a Sturm count at an interior point of the eigenvalue's interval,
//      a ballot picks the sub-interval, until the width is <= 1e-15 ||T||.
//   4. Lane j (< k) computes eigenvector j of T by inverse iteration with that
//      shift (tridiagonal LU without pivoting, tiny pivots replaced by
//      +-eps ||T||), PSD_INV_ITERS steps, each followed by modified
//      Gram-Schmidt across the k lanes (clustered eigenvalues).
//   5. x_j = Q y_j through the stored reflectors, w_j = sqrt(|l_j|) x_j, and
//      every staged value becomes A + sum_j w_j w_j^T (rounded to the staging
//      type).
// Eigenvalues in (-tau ||T||, 0] are left in place where the reference clamps
// them to zero; tau sits above the rounding noise of the staging type: 1e-12 for
// FP64 blocks (the rigid-motion null space of an element matrix is computed at
// +-1e-15 ||A||), 1e-6 for FP32 blocks (rounding A to FP32 moves those null
// eigenvalues by up to ~3e-7 ||A||).  The difference is below tau ||A|| per
// element.
// A matrix holding NaN, or whose inverse iteration overflows, is left as it is.
// The reciprocals of the inverse iteration's LU pivots use the hardware
// approximation (rcp.approx.ftz.f64) refined by two Newton-Raphson steps.
// ---------------------------------------------------------------------------
template <class T>
__host__ __device__ constexpr double psd_tau() { return sizeof(T) == 8 ? 1e-12 : 1e-6; } // relative to ||T||
constexpr double PSD_PIVMIN = 1e-280;  // pivot given to a zero Sturm minor (scaled T)
constexpr double PSD_WIDTH = 1e-15;    // bisection stops at this interval width
constexpr int PSD_MAX_BISECT = 80;     // 53 halvings reach PSD_WIDTH from width 1
constexpr int PSD_INV_ITERS = 2;

template <class EL>
struct PsdWarp
{
	static constexpr int M = 3 * EL::N;
	static_assert(M % 2 == 0, "rows are read as double2");
	double V[M * M]; // reflector i in row i (zero beyond column i-1); later w_j in row j
	double2 de2[M];  // scaled diagonal of T and squared off-diagonal (T[i-1][i]^2)
	double en[M];    // off-diagonal T[i-1][i] (raw, then scaled); en[0] = 0
	double hinv[M];  // 1/h_i of reflector i, 0 where step i has none
	double row[M];   // row i of A during tridiagonalisation step i
	double buf[M];   // q of a tridiagonalisation step; a Gram-Schmidt vector
};

__device__ __forceinline__ double warp_allsum(double v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}
__device__ __forceinline__ double warp_allmax(double v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}

// 1/q: hardware approximation refined by two Newton-Raphson steps r += r (1 - q r)
__device__ __forceinline__ double rcp_nr(double q)
{
	double r;
	asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(q));
	double e = fma(-q, r, 1.0);
	r = fma(r, e, r);
	e = fma(-q, r, 1.0);
	return fma(r, e, r);
}

// Number of eigenvalues of the scaled T below x: the sign changes of the leading
// principal minors p_i = det(T_i - x I) = (d_i - x) p_{i-1} - e_i^2 p_{i-2}
// (Sturm sequence), i.e. the negative pivots q_i = p_i / p_{i-1} of the LDL^T
// factorisation of T - x I, without a division.  A zero minor becomes
// -PSD_PIVMIN p_{i-1} (a pivot of -PSD_PIVMIN, as the LDL^T count does); the pair
// (p_i, p_{i-1}) is rescaled by 2^500 every fourth step once |p_i| < 2^-500, so
// no minor underflows (|d_i - x| <= 2.001 and e_i^2 <= 1 bound the growth by
// (1 + sqrt 2)^30 < 2^40 between rescalings).
template <int M>
__device__ __forceinline__ int sturm_count(const double2 *__restrict__ de2, double x)
{
	double pm = 1.0, p = de2[0].x - x;
	if (p == 0.0) p = -PSD_PIVMIN;
	int c = p < 0.0;
#pragma unroll
	for (int i = 1; i < M; ++i)
	{
		const double2 v = de2[i];
		double pn = fma(v.x - x, p, -(v.y * pm));
		if (pn == 0.0) pn = -PSD_PIVMIN * p;
		c += (pn < 0.0) != (p < 0.0);
		if ((i & 3) == 0)
		{
			const double sc = fabs(pn) < 0x1p-500 ? 0x1p500 : 1.0;
			pn *= sc;
			p *= sc;
		}
		pm = p;
		p = pn;
	}
	return c;
}

// Householder step i (l = i - 1) of the tridiagonalisation (EISPACK tred2 without
// the accumulation of Q), on the lanes' register rows a (lane j < M owns row j):
// row i is broadcast through S.row by lane i; the reflector u = x - g e_l with
// x = A[i][0..l], g = -sign(x_l) |x|, h = |x|^2 - x_l g, goes to V[i][*] (zero
// beyond l); rows j <= l apply A -= u q^T + q u^T with p = A u / h,
// q = p - (u.p / 2h) u, the other lanes hold u_j = q_j = 0.  Columns >= W are
// untouched (W > l).  |x|^2 is formed unscaled when it lies in [1e-250, 1e250],
// else from x / sum|x_k| as tred2 does.
template <int M, int W, class PW>
__device__ __forceinline__ void psd_tred2_step(PW &S, double (&a)[M], int i, int lane)
{
	constexpr unsigned FULL = 0xffffffffu;
	const int l = i - 1;
	const bool mine = lane <= l;
	if (lane == i)
	{
		double2 *w2 = reinterpret_cast<double2 *>(S.row);
#pragma unroll
		for (int t = 0; t < W; t += 2) w2[t / 2] = make_double2(a[t], a[t + 1]);
	}
	__syncwarp();
	double x = mine ? S.row[lane] : 0.0; // A[i][lane]
	double sig = warp_allsum(x * x), scale = 1.0;
	if (!(sig >= 1e-250 && sig <= 1e250))
	{
		scale = warp_allsum(fabs(x));
		if (scale != 0.0)
		{
			x *= 1.0 / scale;
			sig = warp_allsum(x * x);
		}
	}
	double u = 0.0, g = 0.0, ih = 0.0;
	if (sig != 0.0)
	{
		const double f = __shfl_sync(FULL, x, l);
		g = f >= 0.0 ? -sqrt(sig) : sqrt(sig);
		ih = rcp_nr(sig - f * g);
		u = lane == l ? f - g : x;
	}
	double *V = S.V;
	if (lane < M) V[i * M + lane] = u;
	if (lane == 0)
	{
		S.en[i] = scale * g;
		S.hinv[i] = ih;
	}
	__syncwarp();
	if (ih != 0.0)
	{
		const double2 *u2 = reinterpret_cast<const double2 *>(V + i * M);
		const double2 *q2 = reinterpret_cast<const double2 *>(S.buf);
		double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
#pragma unroll
		for (int t = 0; t < W; t += 4)
		{
			const double2 u01 = u2[t / 2];
			p0 = fma(a[t], u01.x, p0);
			p1 = fma(a[t + 1], u01.y, p1);
			if (t + 2 < W)
			{
				const double2 u23 = u2[t / 2 + 1];
				p2 = fma(a[t + 2], u23.x, p2);
				p3 = fma(a[t + 3], u23.y, p3);
			}
		}
		const double p = ((p0 + p1) + (p2 + p3)) * ih;
		const double kk = warp_allsum(mine ? p * u : 0.0) * (0.5 * ih);
		const double q = mine ? p - kk * u : 0.0;
		if (lane < M) S.buf[lane] = q;
		__syncwarp();
#pragma unroll
		for (int t = 0; t < W; t += 2)
		{
			const double2 uu = u2[t / 2], qq = q2[t / 2];
			a[t] = fma(-u, qq.x, fma(-q, uu.x, a[t]));
			a[t + 1] = fma(-u, qq.y, fma(-q, uu.y, a[t + 1]));
		}
	}
	__syncwarp();
}

// y -= (u_i . y / h_i) u_i for the reflector u_i in V[i][*] (zero from column i on,
// so columns >= W > i - 1 are untouched)
template <int M, int W, class PW>
__device__ __forceinline__ void psd_reflect(const PW &S, double (&y)[M], int i)
{
	const double2 *u2 = reinterpret_cast<const double2 *>(S.V + i * M);
	double s0 = 0.0, s1 = 0.0;
#pragma unroll
	for (int t = 0; t < W; t += 2)
	{
		const double2 uu = u2[t / 2];
		s0 = fma(uu.x, y[t], s0);
		s1 = fma(uu.y, y[t + 1], s1);
	}
	const double s = (s0 + s1) * S.hinv[i];
#pragma unroll
	for (int t = 0; t < W; t += 2)
	{
		const double2 uu = u2[t / 2];
		y[t] = fma(-s, uu.x, y[t]);
		y[t + 1] = fma(-s, uu.y, y[t + 1]);
	}
}

// The projection of element e by one warp (all 32 lanes, converged on entry and
// on every return; S is the warp's shared workspace)
template <class EL, class T>
__device__ __forceinline__ void psd_element(PsdWarp<EL> &S, T *__restrict__ stage, int e, int lane)
{
	using W = PsdWarp<EL>;
	constexpr int N = EL::N, M = W::M;
	constexpr unsigned FULL = 0xffffffffu;
	static_assert(M <= 32, "one lane per row");
	// lane i = 3a + r < M owns row i of the element matrix: A[3a+r][3b+c] is value
	// 3c + r of staged block (a, b) for a <= b, value 3r + c of block (b, a) for a > b
	T *tri = stage + (size_t)e * tri_pad(N);
	const int ra = lane / 3, rr = lane % 3;
	const auto at = [&](int b, int c) {
		return ra <= b ? 9 * tri_index(N, ra, b) + 3 * c + rr : 9 * tri_index(N, b, ra) + 3 * rr + c;
	};

	double a[M];
#pragma unroll
	for (int b = 0; b < N; ++b)
#pragma unroll
		for (int c = 0; c < 3; ++c)
		{
			a[3 * b + c] = 0.0;
			if (lane < M) a[3 * b + c] = double(tri[at(b, c)]);
		}
	bool nan_in = false;
#pragma unroll
	for (int t = 0; t < M; ++t) nan_in |= isnan(a[t]);
	if (__any_sync(FULL, nan_in)) return; // NaN propagates unchanged

	// --- 1. tridiagonalisation ------------------------------------------------
	// steps M-1 .. H+1 touch all columns, steps H .. 2 only columns < H
	constexpr int H = ((M / 2) + 1) & ~1;
#pragma unroll 1
	for (int i = M - 1; i > H; --i) psd_tred2_step<M, M>(S, a, i, lane);
#pragma unroll 1
	for (int i = H; i >= 2; --i) psd_tred2_step<M, H>(S, a, i, lane);
	double *V = S.V;
	double dj = 0.0;
#pragma unroll
	for (int t = 0; t < M; ++t)
		if (t == lane) dj = a[t];
	if (lane == 1) S.en[1] = a[0]; // A[1][0]
	if (lane == 0)
	{
		S.en[0] = 0.0;
		S.hinv[0] = 0.0;
		S.hinv[1] = 0.0;
	}
	__syncwarp();

	// --- 2./3. scale; count below -tau, then multisection ------------------------
	const double ej = lane < M ? S.en[lane] : 0.0;
	const double ej1 = lane + 1 < M ? S.en[lane + 1] : 0.0;
	const double nrm = warp_allmax(lane < M ? fabs(dj) + fabs(ej) + fabs(ej1) : 0.0);
	if (!(nrm > 0.0 && nrm <= 1.7976931348623157e308)) return; // zero, Inf or NaN
	const double inv = 1.0 / nrm;
	__syncwarp();
	if (lane < M)
	{
		const double en = ej * inv;
		S.de2[lane] = make_double2(dj * inv, en * en);
		S.en[lane] = en;
	}
	__syncwarp();
	// iteration -1 counts the eigenvalues below -tau on every lane; later
	// iterations: 32 / k lanes per eigenvalue j < k, each at an interior point of
	// the eigenvalue's interval [lo, hi) (count(lo) <= j < count(hi))
	int k = 0, G = 1, jg = 0;
	bool act = false;
	unsigned gmask = 0u;
	double frac = 0.0, lo = -1.0 - 1e-3, hi = -psd_tau<T>(), x = hi;
#pragma unroll 1
	for (int it = -1; it < PSD_MAX_BISECT; ++it)
	{
		bool done = true;
		if (it >= 0)
		{
			done = !act || hi - lo <= PSD_WIDTH;
			if (__all_sync(FULL, done)) break;
			x = fma(hi - lo, frac, lo);
		}
		const int c = sturm_count<M>(S.de2, x);
		if (it < 0)
		{
			k = c;
			if (k == 0) return; // PSD: the staged blocks stay as they are
			G = 32 / k;
			jg = lane / G;
			act = jg < k;
			gmask = G == 32 ? FULL : ((1u << G) - 1u);
			frac = double(lane - jg * G + 1) / double(G + 1);
			continue;
		}
		const unsigned bal = __ballot_sync(FULL, c <= jg);
		const unsigned mg = act ? (bal >> (jg * G)) & gmask : 0u;
		// first point of the group with more than jg eigenvalues below it
		const int tf = mg == gmask ? G : __ffs(~mg) - 1;
		const double xlo = __shfl_sync(FULL, x, (jg * G + tf - 1) & 31);
		const double xhi = __shfl_sync(FULL, x, (jg * G + tf) & 31);
		if (!done)
		{
			if (tf > 0) lo = xlo;
			if (tf < G) hi = xhi;
		}
	}
	const bool vec = lane < k;
	const double sig = __shfl_sync(FULL, 0.5 * (lo + hi), (lane * G) & 31);

	// --- 4. inverse iteration, lane j -> eigenvector j ---------------------------
	double y[M];
#pragma unroll
	for (int i = 0; i < M; ++i)
	{
		const unsigned hsh = (unsigned)(i * 7919 + lane * 104729 + 12345) * 2654435761u;
		y[i] = 1.0 + 0.5 * (double)(hsh >> 8) * (1.0 / 16777216.0);
	}
	bool bad = false;
	constexpr double PMIN = 2.220446049250313e-16;
	double2 *b2 = reinterpret_cast<double2 *>(S.buf);
#pragma unroll 1
	for (int it = 0; it < PSD_INV_ITERS; ++it)
	{
		// T is re-read from shared memory in every pass (an opaque pointer keeps the
		// compiler from holding all of it in registers across the passes)
		const double2 *de2 = S.de2;
		const double *enp = S.en;
		asm volatile("" : "+l"(de2), "+l"(enp));
		double rp[M];
		{
			double pv = de2[0].x - sig;
			if (fabs(pv) < PMIN) pv = pv >= 0.0 ? PMIN : -PMIN;
			rp[0] = rcp_nr(pv);
		}
#pragma unroll
		for (int i = 1; i < M; ++i)
		{
			const double eni = enp[i];
			const double mi = eni * rp[i - 1];
			double pv = (de2[i].x - sig) - mi * eni;
			if (fabs(pv) < PMIN) pv = pv >= 0.0 ? PMIN : -PMIN;
			rp[i] = rcp_nr(pv);
			y[i] = fma(-mi, y[i - 1], y[i]);
		}
		y[M - 1] *= rp[M - 1];
#pragma unroll
		for (int i = M - 2; i >= 0; --i) y[i] = fma(-enp[i + 1], y[i + 1], y[i]) * rp[i];
		double ym = 0.0;
#pragma unroll
		for (int i = 0; i < M; ++i) ym = fmax(ym, fabs(y[i]));
		bad |= vec && !(ym > 0.0 && ym <= 1.7976931348623157e308);
		const double iy = 1.0 / ym;
#pragma unroll
		for (int i = 0; i < M; ++i) y[i] *= iy;
		// modified Gram-Schmidt over lanes 0..k-1
#pragma unroll 1
		for (int j = 0; j < k; ++j)
		{
			if (lane == j)
			{
				double s0 = 0.0, s1 = 0.0;
#pragma unroll
				for (int i = 0; i < M; i += 2)
				{
					s0 = fma(y[i], y[i], s0);
					s1 = fma(y[i + 1], y[i + 1], s1);
				}
				const double s = s0 + s1;
				bad |= !(s > 0.0 && s <= 1.7976931348623157e308); // NaN, overflow or a lost vector
				const double r = rsqrt(s);
#pragma unroll
				for (int i = 0; i < M; i += 2)
				{
					y[i] *= r;
					y[i + 1] *= r;
					b2[i / 2] = make_double2(y[i], y[i + 1]);
				}
			}
			__syncwarp();
			if (lane > j && vec)
			{
				double d0 = 0.0, d1 = 0.0;
#pragma unroll
				for (int i = 0; i < M; i += 2)
				{
					const double2 bb = b2[i / 2];
					d0 = fma(y[i], bb.x, d0);
					d1 = fma(y[i + 1], bb.y, d1);
				}
				const double dot = d0 + d1;
#pragma unroll
				for (int i = 0; i < M; i += 2)
				{
					const double2 bb = b2[i / 2];
					y[i] = fma(-dot, bb.x, y[i]);
					y[i + 1] = fma(-dot, bb.y, y[i + 1]);
				}
			}
			__syncwarp();
		}
	}
	if (__any_sync(FULL, bad)) return;

	// --- 5. back-transform x = P_2 ... P_{M-1} y (reflector 2 first), w = sqrt|l| x
#pragma unroll 1
	for (int i = 2; i <= H; ++i) psd_reflect<M, H>(S, y, i);
#pragma unroll 1
	for (int i = H + 1; i < M; ++i) psd_reflect<M, M>(S, y, i);
	__syncwarp();
	if (vec)
	{
		const double sw = sqrt(-sig * nrm);
		double2 *w2 = reinterpret_cast<double2 *>(V + lane * M);
#pragma unroll
		for (int t = 0; t < M; t += 2) w2[t / 2] = make_double2(sw * y[t], sw * y[t + 1]);
	}
	__syncwarp();

	// --- 6. row i of A + sum_j w_j w_j^T, blocks (a, b >= a), back into the triangle
	if (lane < M)
	{
		double r[M];
#pragma unroll
		for (int b = 0; b < N; ++b)
#pragma unroll
			for (int c = 0; c < 3; ++c) r[3 * b + c] = double(tri[at(b, c)]);
#pragma unroll 1
		for (int j = 0; j < k; ++j)
		{
			const double wi = V[j * M + lane];
			const double2 *w2 = reinterpret_cast<const double2 *>(V + j * M);
#pragma unroll
			for (int t = 0; t < M; t += 2)
			{
				const double2 ww = w2[t / 2];
				r[t] = fma(wi, ww.x, r[t]);
				r[t + 1] = fma(wi, ww.y, r[t + 1]);
			}
		}
#pragma unroll
		for (int b = 0; b < N; ++b)
#pragma unroll
			for (int c = 0; c < 3; ++c)
				if (b >= ra) tri[at(b, c)] = T(r[3 * b + c]); // each stored value once
	}
}

// One warp per element, 3 CTAs of 4 warps per SM for P2 and Q1 and 5 for P1 (at most
// 168 registers a thread, a few spill for P2).  For P1 the warps are persistent:
// each takes the next element from the counter m.work (zero at launch) until none
// is left, so a warp whose element is already PSD, or has few negative eigenvalues,
// goes on to the next one instead of idling until the other warps of its CTA
// finish (P1 48^3: 5.51 -> 4.97 ms).  The larger P2 and Q1 kernels run one element
// per warp: persistent warps drift apart in phase and were slower there (P2 40^3
// 16.3 -> 17.6 ms).  Each element's arithmetic does not depend on which warp
// projects it.
template <class EL>
__host__ __device__ constexpr bool psd_persistent() { return EL::ET == 1; }

template <class EL, class T, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, EL::ET == 1 ? 5 : 3) k_project_psd(DevMesh m, T *__restrict__ stage)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	PsdWarp<EL> &S = reinterpret_cast<PsdWarp<EL> *>(smem_raw)[threadIdx.x >> 5];
	const int lane = threadIdx.x & 31;
	if constexpr (!psd_persistent<EL>())
	{
		const int e = blockIdx.x * WARPS + (threadIdx.x >> 5);
		if (e < m.E) psd_element<EL, T>(S, stage, e, lane);
	}
	else
	{
		for (;;)
		{
			int e = 0;
			if (lane == 0) e = atomicAdd(m.work, 1);
			e = __shfl_sync(0xffffffffu, e, 0);
			if (e >= m.E) return;
			// an opaque copy of the lane keeps the lane-dependent offsets inside the
			// element (hoisted out of the loop they would stay live and spill)
			int ln = lane;
			asm volatile("" : "+r"(ln));
			psd_element<EL, T>(S, stage, e, ln);
			__syncwarp();
		}
	}
}

// ---------------------------------------------------------------------------
// Other materials of the GenericElastic family, FP64: energy, gradient and the
// element blocks of the Hessian (the scatter, the PSD projection and the Dirichlet
// reduction are the NeoHookean path's).  The reference differentiates psi(F) with
// dual numbers (GenericElastic.cpp, AutodiffType::STRESS); here the first Piola
// stress P = dpsi/dF and the blocks H_ab = sum_q da sum_jl g_a[j] dP_ij/dF_kl g_b[l]
// are written out analytically with the per-node vectors g_a (physical basis
// gradient), f_a = F g_a and d_a = F^-T g_a:
//  IsochoricNeoHookean (IsochoricNeoHookean.hpp:19-33), psi = mu/2 (|F|^2 J^-2/3 - 3):
//    P = mu J^-2/3 (F - |F|^2/3 F^-T)
//    H_ab = mu J^-2/3 da [ (g_a.g_b) I - 2/3 (f_a d_b^T + d_a f_b^T)
//                          + 2/9 |F|^2 d_a d_b^T + |F|^2/3 d_b d_a^T ]
//  SaintVenant, isotropic (SaintVenantElasticity.cpp:209-267 with the tensor of
//  ElasticityTensor::set_from_lambda_mu, MatParams.cpp:211-260),
//  psi = lambda/2 tr(E)^2 + mu |E|^2, E = (F^T F - I)/2, S = lambda tr(E) I + 2 mu E:
//    P = F S
//    H_ab = da [ (g_a^T S g_b) I + lambda f_a f_b^T + mu (g_a.g_b) F F^T + mu f_b f_a^T ]
// ---------------------------------------------------------------------------
constexpr int MAT_ISO_NEOHOOKEAN = 1, MAT_SAINT_VENANT = 2;

// node pairs (a <= b) in tri_index order for n = 4, 10, 8 nodes (P1, P2, Q1), in
// constant memory: lanes at different pairs read them without a decoding loop
__constant__ PairTable c_pairs[3] = {make_pairs(4), make_pairs(10), make_pairs(8)};

// Green strain from the displacement gradient G = F - I: E = (G^T G + G + G^T) / 2
__device__ __forceinline__ void green_strain(const double F[3][3], double E[3][3])
{
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c)
		{
			double gtg = 0.0;
#pragma unroll
			for (int k = 0; k < 3; ++k) gtg += (F[k][r] - (k == r)) * (F[k][c] - (k == c));
			E[r][c] = 0.5 * (gtg + (F[r][c] - (r == c)) + (F[c][r] - (r == c)));
		}
}

template <int MAT>
__device__ __forceinline__ double mat_psi(const double F[3][3], double lambda, double mu)
{
	if constexpr (MAT == MAT_ISO_NEOHOOKEAN)
	{
		double I1 = 0.0;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) I1 += F[r][c] * F[r][c];
		return mu / 2 * (I1 * pow(det3(F), -2.0 / 3.0) - 3.0);
	}
	else
	{
		double E[3][3];
		green_strain(F, E);
		const double tr = E[0][0] + E[1][1] + E[2][2];
		double e2 = 0.0;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) e2 += E[r][c] * E[r][c];
		return lambda / 2 * tr * tr + mu * e2;
	}
}

template <int MAT>
__device__ __forceinline__ void mat_piola(const double F[3][3], double lambda, double mu, double P[3][3])
{
	if constexpr (MAT == MAT_ISO_NEOHOOKEAN)
	{
		double I1 = 0.0;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) I1 += F[r][c] * F[r][c];
		const double J = det3(F);
		double G[3][3];
		inv_transpose3(F, J, G);
		const double cj = mu * pow(J, -2.0 / 3.0);
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) P[r][c] = cj * (F[r][c] - I1 / 3 * G[r][c]);
	}
	else
	{
		double E[3][3];
		green_strain(F, E);
		const double tr = E[0][0] + E[1][1] + E[2][2];
		double S[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) S[r][c] = 2 * mu * E[r][c] + (r == c ? lambda * tr : 0.0);
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) P[r][c] = F[r][0] * S[0][c] + F[r][1] * S[1][c] + F[r][2] * S[2][c];
	}
}


template <class EL, int MAT>
__device__ __forceinline__ double gen_element_energy(const DevMesh &m, const double *__restrict__ u, int e,
													 unsigned long long *inverted)
{
	double Xg[EL::NG][3], U[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, double>(m, e, Xg);
	load_nodal<EL, double>(m, e, u, U, nodes);
	const double2 lm = __ldg(m.lame + e);
	double en = 0.0;
	bool bad = false;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		double Jit[3][3], detJ, F[3][3];
		geometry<EL, double>(q, Xg, Jit, detJ);
		gen_def_grad<EL>(q, U, Jit, F);
		bad |= !(det3(F) > 0.0);
		en += mat_psi<MAT>(F, lm.x, lm.y) * (detJ * qweight<EL>(q));
	}
	if (bad) atomicAdd(inverted, 1ull);
	return en;
}

template <class EL, int MAT, int NT>
__global__ void __launch_bounds__(NT) k_gen_energy(DevMesh m, const double *__restrict__ u, double *__restrict__ partials,
												   double *__restrict__ result, unsigned int *ticket,
												   unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	double en = 0.0;
	if (e < m.E) en = gen_element_energy<EL, MAT>(m, u, e, inverted);
	reduce_to_result<NT>(en, partials, result, ticket);
}

template <class EL, int MAT, int NT>
__global__ void __launch_bounds__(NT) k_gen_energy_per_element(DevMesh m, const double *__restrict__ u,
															   double *__restrict__ out, unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e < m.E) out[e] = gen_element_energy<EL, MAT>(m, u, e, inverted);
}

// element gradient G[a][d] = sum_q da (P J^-1)[d][r] gref(q, a, r), staged per
// incidence like the NeoHookean gradient
template <class EL, int MAT, int NT>
__global__ void __launch_bounds__(NT) k_gen_gradient(DevMesh m, const double *__restrict__ u, double *__restrict__ stage,
													 unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	double Xg[EL::NG][3], U[EL::N][3], Gacc[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, double>(m, e, Xg);
	load_nodal<EL, double>(m, e, u, U, nodes);
	const double2 lm = __ldg(m.lame + e);
#pragma unroll
	for (int a = 0; a < EL::N; ++a) Gacc[a][0] = Gacc[a][1] = Gacc[a][2] = 0.0;
	bool bad = false;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		double Jit[3][3], detJ, F[3][3], P[3][3];
		geometry<EL, double>(q, Xg, Jit, detJ);
		gen_def_grad<EL>(q, U, Jit, F);
		bad |= !(det3(F) > 0.0);
		mat_piola<MAT>(F, lm.x, lm.y, P);
		const double da = detJ * qweight<EL>(q);
		double Q[3][3]; // da P J^-1 = da P Jit^T
#pragma unroll
		for (int d = 0; d < 3; ++d)
#pragma unroll
			for (int r = 0; r < 3; ++r) Q[d][r] = da * (P[d][0] * Jit[r][0] + P[d][1] * Jit[r][1] + P[d][2] * Jit[r][2]);
#pragma unroll
		for (int a = 0; a < EL::N; ++a)
#pragma unroll
			for (int r = 0; r < 3; ++r)
			{
				const double gr = gref<EL>(q, a, r);
				if (gr != 0.0)
				{
#pragma unroll
					for (int d = 0; d < 3; ++d) Gacc[a][d] += gr * Q[d][r];
				}
			}
	}
	if (bad) atomicAdd(inverted, 1ull);
#pragma unroll
	for (int a = 0; a < EL::N; ++a)
	{
		const int k = __ldg(m.eb_inc + (size_t)e * EL::N + a);
		st_slot(stage + (size_t)k * 4, Gacc[a][0], Gacc[a][1], Gacc[a][2]);
	}
}

// Element blocks for the other materials, one warp per element: per point (lanes
// q < NQ) J^-T, F, F^-T and the material's coefficients; per (point, node) the
// vectors g, f = F g, d = F^-T g; per node pair (a <= b, tri_index order) the block,
// written as the packed block triangle of the element (as k_hessian_blocks does).
template <class EL>
struct GenWarp
{
	static constexpr int N = EL::N, NG = EL::NG, NQ = EL::NQ, TP = tri_pad(EL::N);
	double U[N][3], X[NG][3];
	double F[NQ][9], G[NQ][9], Jit[NQ][9];
	double c[NQ][16]; // IsochoricNeoHookean: mu J^-2/3 da, |F|^2; SaintVenant: da, lambda, mu, S (row-major 9)
	alignas(16) double nv[NQ][N][10]; // g, f, d, pad: five 16-byte loads
	alignas(16) double tri[TP]; // copied out as double2 (the members above can end on an odd double)
};

// 128-thread CTAs per SM the register budget allows: P2 five (at most 102 registers),
// Q1 three (IsochoricNeoHookean) or four, P1 five or seven
template <class EL, int MAT>
constexpr int gen_blocks_min_ctas()
{
	return EL::ET == 2 ? 5 : EL::ET == 3 ? (MAT == MAT_ISO_NEOHOOKEAN ? 3 : 4) : (MAT == MAT_ISO_NEOHOOKEAN ? 5 : 7);
}

template <class EL, int MAT, int WPB>
__global__ void __launch_bounds__(WPB * 32, gen_blocks_min_ctas<EL, MAT>())
	k_gen_blocks(DevMesh m, const double *__restrict__ u, double *__restrict__ stage)
{
	using W = GenWarp<EL>;
	constexpr int N = EL::N, NG = EL::NG, NQ = EL::NQ, NP = N * (N + 1) / 2, TP = W::TP;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	W &S = reinterpret_cast<W *>(smem_raw)[threadIdx.x >> 5];
	const int lane = threadIdx.x & 31;
	// the node pairs in shared memory: lanes at different pairs read them without the
	// serialisation of divergent constant-memory reads
	__shared__ unsigned char s_pa[NP], s_pb[NP];
	for (int t = threadIdx.x; t < NP; t += WPB * 32)
	{
		s_pa[t] = c_pairs[EL::ET - 1].a[t];
		s_pb[t] = c_pairs[EL::ET - 1].b[t];
	}
	__syncthreads();
	for (int e = blockIdx.x * WPB + (threadIdx.x >> 5); e < m.E; e += gridDim.x * WPB)
	{
		for (int i = lane; i < N * 3; i += 32)
			S.U[i / 3][i % 3] = __ldg(u + (size_t)__ldg(m.conn + (size_t)(i / 3) * m.E + e) * 3 + i % 3);
		for (int i = lane; i < NG * 3; i += 32)
			S.X[i / 3][i % 3] = __ldg(m.X + (size_t)__ldg(m.gconn + (size_t)(i / 3) * m.E + e) * 3 + i % 3);
		__syncwarp();
		if (lane < NQ)
		{
			const int q = lane;
			const double2 lm = __ldg(m.lame + e);
			double Jit[3][3], detJ, F[3][3];
			geometry<EL, double>(q, S.X, Jit, detJ);
			gen_def_grad<EL>(q, S.U, Jit, F);
			const double da = detJ * qweight<EL>(q);
			const double J = det3(F);
			double G[3][3];
			inv_transpose3(F, J, G);
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c)
				{
					S.F[q][3 * r + c] = F[r][c];
					S.G[q][3 * r + c] = G[r][c];
					S.Jit[q][3 * r + c] = Jit[r][c];
				}
			if constexpr (MAT == MAT_ISO_NEOHOOKEAN)
			{
				double I1 = 0.0;
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int c = 0; c < 3; ++c) I1 += F[r][c] * F[r][c];
				S.c[q][0] = lm.y * pow(J, -2.0 / 3.0) * da;
				S.c[q][1] = I1;
			}
			else
			{
				// c = [da, lambda, mu, S (row-major 9), -] and F F^T in S.G (F^-T unused)
				double E[3][3];
				green_strain(F, E);
				const double tr = E[0][0] + E[1][1] + E[2][2];
				S.c[q][0] = da;
				S.c[q][1] = lm.x;
				S.c[q][2] = lm.y;
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int c = 0; c < 3; ++c)
					{
						S.c[q][3 + 3 * r + c] = 2 * lm.y * E[r][c] + (r == c ? lm.x * tr : 0.0);
						S.G[q][3 * r + c] = F[r][0] * F[c][0] + F[r][1] * F[c][1] + F[r][2] * F[c][2];
					}
			}
		}
		__syncwarp();
		for (int i = lane; i < NQ * N; i += 32)
		{
			const int q = i / N, a = i - q * N;
			double g[3];
#pragma unroll
			for (int c = 0; c < 3; ++c)
				g[c] = gref<EL>(q, a, 0) * S.Jit[q][c] + gref<EL>(q, a, 1) * S.Jit[q][3 + c] + gref<EL>(q, a, 2) * S.Jit[q][6 + c];
			double *v = S.nv[q][a];
#pragma unroll
			for (int r = 0; r < 3; ++r)
			{
				v[r] = g[r];
				v[3 + r] = S.F[q][3 * r] * g[0] + S.F[q][3 * r + 1] * g[1] + S.F[q][3 * r + 2] * g[2];
				v[6 + r] = MAT == MAT_ISO_NEOHOOKEAN ? S.G[q][3 * r] * g[0] + S.G[q][3 * r + 1] * g[1] + S.G[q][3 * r + 2] * g[2] : 0.0;
			}
			v[9] = 0.0;
		}
		__syncwarp();
		for (int p = lane; p < NP; p += 32)
		{
			const int a = s_pa[p], b = s_pb[p];
			double h[3][3] = {};
			for (int q = 0; q < NQ; ++q)
			{
				double va[10], vb[10];
				const double2 *pa = reinterpret_cast<const double2 *>(S.nv[q][a]), *pb = reinterpret_cast<const double2 *>(S.nv[q][b]);
#pragma unroll
				for (int t = 0; t < 5; ++t)
				{
					const double2 x = pa[t], y = pb[t];
					va[2 * t] = x.x;
					va[2 * t + 1] = x.y;
					vb[2 * t] = y.x;
					vb[2 * t + 1] = y.y;
				}
				const double gab = va[0] * vb[0] + va[1] * vb[1] + va[2] * vb[2];
				if constexpr (MAT == MAT_ISO_NEOHOOKEAN)
				{
					const double c0 = S.c[q][0], I1 = S.c[q][1];
#pragma unroll
					for (int r = 0; r < 3; ++r)
#pragma unroll
						for (int k = 0; k < 3; ++k)
							h[r][k] += c0 * ((r == k ? gab : 0.0) - 2.0 / 3.0 * (va[3 + r] * vb[6 + k] + va[6 + r] * vb[3 + k]) +
											 2.0 / 9.0 * I1 * va[6 + r] * vb[6 + k] + I1 / 3.0 * vb[6 + r] * va[6 + k]);
				}
				else
				{
					const double da = S.c[q][0], lam = S.c[q][1], mu = S.c[q][2];
					const double *Sm = S.c[q] + 3, *B = S.G[q];
					double sab = 0.0;
#pragma unroll
					for (int r = 0; r < 3; ++r)
#pragma unroll
						for (int k = 0; k < 3; ++k) sab += va[r] * Sm[3 * r + k] * vb[k];
#pragma unroll
					for (int r = 0; r < 3; ++r)
#pragma unroll
						for (int k = 0; k < 3; ++k)
							h[r][k] += da * ((r == k ? sab : 0.0) + lam * va[3 + r] * vb[3 + k] + mu * gab * B[3 * r + k] +
											 mu * vb[3 + r] * va[3 + k]);
				}
			}
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int k = 0; k < 3; ++k) S.tri[9 * p + 3 * k + r] = h[r][k];
		}
		__syncwarp();
		double2 *dst = reinterpret_cast<double2 *>(stage + (size_t)e * TP);
		const double2 *src = reinterpret_cast<const double2 *>(S.tri);
		for (int i = lane; i < TP / 2; i += 32) dst[i] = src[i];
		__syncwarp();
	}
}

// P1: one resident grid of persistent warps over all elements, m.work cleared on
// the stream first; P2 and Q1: one warp per element
template <class EL, class T>
static cudaError_t launch_project_psd(const DevMesh &m, T *stage, cudaStream_t s)
{
	constexpr int PW = 4;
	if (m.E <= 0) return cudaSuccess;
	const size_t bytes_p = PW * sizeof(PsdWarp<EL>);
	cudaError_t e = cudaFuncSetAttribute(k_project_psd<EL, T, PW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes_p);
	if (e != cudaSuccess) return e;
	const long long need = (m.E + PW - 1) / PW;
	int grid = (int)need;
	if constexpr (psd_persistent<EL>())
	{
		if (!m.work) return cudaErrorInvalidValue;
		static int per_sm = 0; // resident CTAs per SM of this instance (the same on every B200)
		if (per_sm == 0)
		{
			int nb = 0;
			e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_project_psd<EL, T, PW>, PW * 32, bytes_p);
			if (e != cudaSuccess) return e;
			per_sm = nb > 0 ? nb : 1;
		}
		int dev = 0, sms = 0;
		if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
		if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
		grid = (int)std::min<long long>(need, (long long)per_sm * sms);
		if ((e = cudaMemsetAsync(m.work, 0, sizeof(int), s)) != cudaSuccess) return e;
	}
	k_project_psd<EL, T, PW><<<grid, PW * 32, bytes_p, s>>>(m, stage);
	return cudaGetLastError();
}

// FP64 staged element triangles -> (PSD projection) -> CSC values: the tail of the
// Hessian for every material other than NeoHookean
template <class EL>
static cudaError_t finish_fp64_hessian(const DevMesh &m, const DevPattern &p, double *stage, bool project_psd,
									   cudaStream_t s)
{
	constexpr int WARPS = 8;
	if (project_psd)
	{
		const cudaError_t e = launch_project_psd<EL, double>(m, stage, s);
		if (e != cudaSuccess) return e;
	}
	const int ng = (m.N + WARPS - 1) / WARPS;
	if (ng > 0) return launch_reduce<EL, double>(m, p, stage, s);
	return cudaGetLastError();
}

template <class EL, int MAT>
static cudaError_t gen_hessian(const DevMesh &m, const DevPattern &p, const double *u, double *stage, bool project_psd,
							   cudaStream_t s)
{
	constexpr int WPB = 4;
	const size_t bytes = WPB * sizeof(GenWarp<EL>);
	cudaError_t e = cudaFuncSetAttribute(k_gen_blocks<EL, MAT, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
	if (e != cudaSuccess) return e;
	if (m.E > 0)
	{
		const int nb = std::min((m.E + WPB - 1) / WPB, 148 * 32);
		k_gen_blocks<EL, MAT, WPB><<<nb, WPB * 32, bytes, s>>>(m, u, stage);
	}
	return finish_fp64_hessian<EL>(m, p, stage, project_psd, s);
}

template <class EL>
static cudaError_t gen_hessian_mat(const DevMesh &m, const DevPattern &p, const double *u, double *stage,
								   bool project_psd, cudaStream_t s)
{
	return m.mat == MAT_ISO_NEOHOOKEAN ? gen_hessian<EL, MAT_ISO_NEOHOOKEAN>(m, p, u, stage, project_psd, s)
									   : gen_hessian<EL, MAT_SAINT_VENANT>(m, p, u, stage, project_psd, s);
}

// ---------------------------------------------------------------------------
// Mass matrix (MassMatrixAssembler: LinearAssembler::assemble with the Mass term,
// assembler/Assembler.cpp:157-260, assembler/Mass.cpp:5-24): node block (a, b) =
// rho_e int phi_a phi_b dV * I.  The mass quadrature has order 2p
// (AssemblerUtils::quadrature_order("Mass"), AssemblerUtils.cpp:201-211), exact for
// phi_a phi_b on the affine tets, where the integral is taken in closed form from
// int lambda^alpha = |T| 3! alpha! / (|alpha| + 3)!:
//   P1: |T| (1 + delta_ab) / 20;   P2: |T| c_mass_p2[a][b] / 420
// (P2 nodes: vertices lambda_i (2 lambda_i - 1), edges 4 lambda_i lambda_j in the order
// 01, 12, 20, 03, 13, 23); Q1 uses its 2x2x2 Gauss points, as the reference does.
// ---------------------------------------------------------------------------
__constant__ int c_mass_p2[10][10] = {{6, 1, 1, 1, -4, -6, -4, -4, -6, -6},   {1, 6, 1, 1, -4, -4, -6, -6, -4, -6},
									   {1, 1, 6, 1, -6, -4, -4, -6, -6, -4},   {1, 1, 1, 6, -6, -6, -6, -4, -4, -4},
									   {-4, -4, -6, -6, 32, 16, 16, 16, 16, 8}, {-6, -4, -4, -6, 16, 32, 16, 8, 16, 16},
									   {-4, -6, -4, -6, 16, 16, 32, 16, 8, 16}, {-4, -6, -6, -4, 16, 8, 16, 32, 16, 16},
									   {-6, -4, -6, -4, 16, 16, 8, 16, 32, 16}, {-6, -6, -4, -4, 8, 16, 16, 16, 16, 32}};

// trilinear Q1 basis value of node i at (x, y, z): corners 000 100 110 010 001 101 111 011
__host__ __device__ constexpr double q1_value(int i, double x, double y, double z)
{
	const int cx = (i == 1 || i == 2 || i == 5 || i == 6), cy = (i == 2 || i == 3 || i == 6 || i == 7), cz = i >= 4;
	return (cx ? x : 1 - x) * (cy ? y : 1 - y) * (cz ? z : 1 - z);
}

template <class EL, int WPB>
__global__ void __launch_bounds__(WPB * 32) k_mass_blocks(DevMesh m, const double *__restrict__ rho, double *__restrict__ stage)
{
	constexpr int N = EL::N, NQ = EL::NQ, NP = N * (N + 1) / 2, TP = tri_pad(EL::N);
	__shared__ double wdet[WPB][NQ];
	__shared__ double vpair[WPB][NP];
	// per pair (tri_index order): its nodes, and on the affine tets the closed-form
	// factor of |T| (P1 (1 + delta_ab) / 20, P2 c_mass_p2[a][b] / 420)
	__shared__ unsigned char s_pa[NP], s_pb[NP];
	__shared__ double s_coef[NP];
	for (int p = threadIdx.x; p < NP; p += WPB * 32)
	{
		int a = 0, b = p;
		while (b >= N - a)
		{
			b -= N - a;
			++a;
		}
		b += a;
		s_pa[p] = (unsigned char)a;
		s_pb[p] = (unsigned char)b;
		s_coef[p] = EL::ET == 1 ? (a == b ? 2.0 : 1.0) / 20.0 : EL::ET == 2 ? c_mass_p2[a][b] / 420.0 : 0.0;
	}
	__syncthreads();
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	for (int e = blockIdx.x * WPB + w; e < m.E; e += gridDim.x * WPB)
	{
		const double r_e = rho ? __ldg(rho + e) : 1.0;
		if (lane < NQ)
		{
			double Xg[EL::NG][3], Jit[3][3], detJ;
			load_geom<EL, double>(m, e, Xg);
			geometry<EL, double>(lane, Xg, Jit, detJ);
			wdet[w][lane] = detJ * qweight<EL>(lane);
		}
		__syncwarp();
		// the pairs' values, then the whole triangle in consecutive stores
		for (int p = lane; p < NP; p += 32)
		{
			const int a = s_pa[p], b = s_pb[p];
			double v;
			if constexpr (EL::ET == 3)
			{
				v = 0.0;
				for (int q = 0; q < NQ; ++q)
					v += q1_value(a, qpoint<EL>(q, 0), qpoint<EL>(q, 1), qpoint<EL>(q, 2)) *
						 q1_value(b, qpoint<EL>(q, 0), qpoint<EL>(q, 1), qpoint<EL>(q, 2)) * wdet[w][q];
			}
			else
			{
				// |T| = sum_q detJ w_q (the stiffness rule's weights sum to 1/6)
				double vol = 0.0;
				for (int q = 0; q < NQ; ++q) vol += wdet[w][q];
				v = vol * s_coef[p];
			}
			vpair[w][p] = v * r_e;
		}
		__syncwarp();
		double *tri = stage + (size_t)e * TP;
		for (int i = lane; i < TP; i += 32)
		{
			const int p = i / 9, k = i - 9 * p;
			tri[i] = (p < NP && (k == 0 || k == 4 || k == 8)) ? vpair[w][p] : 0.0;
		}
		__syncwarp();
	}
}

cudaError_t launch_mass(const DevMesh &m, const DevPattern &p, const double *rho, void *stage_v, cudaStream_t s)
{
	if (p.nnz == 0) return cudaSuccess;
	double *stage = static_cast<double *>(stage_v);
	constexpr int WPB = 4, WARPS = 8;
	const int nb = m.E > 0 ? std::min((m.E + WPB - 1) / WPB, 148 * 32) : 0;
	const int ng = (m.N + WARPS - 1) / WARPS;
	switch (m.et)
	{
	case 1:
		if (nb) k_mass_blocks<P1Tet, WPB><<<nb, WPB * 32, 0, s>>>(m, rho, stage);
		if (ng) return launch_reduce<P1Tet, double>(m, p, stage, s);
		break;
	case 2:
		if (nb) k_mass_blocks<P2Tet, WPB><<<nb, WPB * 32, 0, s>>>(m, rho, stage);
		if (ng) return launch_reduce<P2Tet, double>(m, p, stage, s);
		break;
	case 3:
		if (nb) k_mass_blocks<Q1Hex, WPB><<<nb, WPB * 32, 0, s>>>(m, rho, stage);
		if (ng) return launch_reduce<Q1Hex, double>(m, p, stage, s);
		break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

template <class EL, class K, class T>
static cudaError_t hessian_two_pass(const DevMesh &m, const DevPattern &p, const double *u, void *stage_v,
									bool project_psd, cudaStream_t s)
{
	using TL = EcTile<EL, T>;
	constexpr int WARPS = 8;
	T *stage = static_cast<T *>(stage_v);
	const size_t bytes1 = sizeof(EcSmem<EL, K, T>);
	cudaError_t e = cudaFuncSetAttribute(k_hessian_blocks<EL, K, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes1);
	if (e != cudaSuccess) return e;
	const int nb = (m.E + TL::TE - 1) / TL::TE;
	if (nb > 0) k_hessian_blocks<EL, K, T><<<nb, TL::NT, bytes1, s>>>(m, u, stage, 0, m.E);
	if (project_psd)
	{
		e = launch_project_psd<EL, T>(m, stage, s);
		if (e != cudaSuccess) return e;
	}
	const int ng = (m.N + WARPS - 1) / WARPS;
	if (ng > 0) return launch_reduce<EL, T>(m, p, stage, s);
	return cudaGetLastError();
}

cudaError_t hessian_kernel_setup(int device) { return tc_tables_setup(device); }

// split mode on the tensor cores: element blocks by tcgen05 (FP32 triangles), then
// the optional projection and the same reduction as the other modes
template <class EL>
static cudaError_t hessian_tc(const DevMesh &m, const DevPattern &p, const double *u, void *stage_v, bool project_psd,
							  cudaStream_t s)
{
	constexpr int WARPS = 8;
	float *stage = static_cast<float *>(stage_v);
	cudaError_t e = launch_hessian_blocks_tc(m, u, stage, s);
	if (e != cudaSuccess) return e;
	if (project_psd)
	{
		e = launch_project_psd<EL, float>(m, stage, s);
		if (e != cudaSuccess) return e;
	}
	const int ng = (m.N + WARPS - 1) / WARPS;
	if (ng > 0) return launch_reduce<EL, float>(m, p, stage, s);
	return cudaGetLastError();
}

cudaError_t launch_hessian(const DevMesh &m, const DevPattern &p, const double *u, int prec, int project_psd,
						   void *stage, cudaStream_t s)
{
	const bool psd = project_psd != 0;
	if (p.nnz == 0) return cudaSuccess;
	if (m.mat >= MAT_FIRST_AD) // automatically differentiated materials: FP64 blocks
	{
		double *st = static_cast<double *>(stage);
		cudaError_t e = launch_ad_blocks(m, u, st, s);
		if (e != cudaSuccess) return e;
		switch (m.et)
		{
		case 1: return finish_fp64_hessian<P1Tet>(m, p, st, psd, s);
		case 2: return finish_fp64_hessian<P2Tet>(m, p, st, psd, s);
		case 3: return finish_fp64_hessian<Q1Hex>(m, p, st, psd, s);
		}
		return cudaErrorInvalidValue;
	}
	if (m.mat != 0) // other materials: FP64 blocks (the caller admits PREC_FP64 only)
	{
		double *st = static_cast<double *>(stage);
		switch (m.et)
		{
		case 1: return gen_hessian_mat<P1Tet>(m, p, u, st, psd, s);
		case 2: return gen_hessian_mat<P2Tet>(m, p, u, st, psd, s);
		case 3: return gen_hessian_mat<Q1Hex>(m, p, u, st, psd, s);
		}
		return cudaErrorInvalidValue;
	}
	// FP64: everything in FP64.  FP32: everything in FP32 except det/log J.
	// SPLIT32_SIMT: kinematics (J^-T, F^-T, det/log J, g, d) in FP64, contraction and
	// records in FP32 on CUDA cores, per-entry sums in FP64.  SPLIT32: the same
	// kinematics, the contraction on the tensor cores (3xTF32) for P2 and Q1.
	switch (m.et)
	{
	case 1:
		return prec == PREC_FP64 ? hessian_two_pass<P1Tet, double, double>(m, p, u, stage, psd, s)
			 : prec == PREC_FP32 ? hessian_two_pass<P1Tet, float, float>(m, p, u, stage, psd, s)
								 : hessian_two_pass<P1Tet, double, float>(m, p, u, stage, psd, s);
	case 2:
		return prec == PREC_FP64	? hessian_two_pass<P2Tet, double, double>(m, p, u, stage, psd, s)
			 : prec == PREC_FP32	? hessian_two_pass<P2Tet, float, float>(m, p, u, stage, psd, s)
			 : prec == PREC_SPLIT32 ? hessian_tc<P2Tet>(m, p, u, stage, psd, s)
									: hessian_two_pass<P2Tet, double, float>(m, p, u, stage, psd, s);
	case 3:
		return prec == PREC_FP64	? hessian_two_pass<Q1Hex, double, double>(m, p, u, stage, psd, s)
			 : prec == PREC_FP32	? hessian_two_pass<Q1Hex, float, float>(m, p, u, stage, psd, s)
			 : prec == PREC_SPLIT32 ? hessian_tc<Q1Hex>(m, p, u, stage, psd, s)
									: hessian_two_pass<Q1Hex, double, float>(m, p, u, stage, psd, s);
	}
	return cudaErrorInvalidValue;
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
												  const double *__restrict__ adj, double *__restrict__ stage)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	T Xg[EL::NG][3];
	T U[EL::N][3], Pn[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, T>(m, e, Xg);
	load_nodal<EL, T>(m, e, u, U, nodes);
	load_nodal<EL, T>(m, e, adj, Pn, nodes);
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
	{
		const int k = __ldg(m.g_eb_inc + (size_t)e * EL::NG + v);
		st_slot(stage + (size_t)k * 4, double(acc[v][0]), double(acc[v][1]), double(acc[v][2]));
	}
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
	{
		// as many blocks as stay resident (never more than one per 256 elements, the
		// partials' capacity)
		static int resident = 0;
		if (!resident)
		{
			int dev = 0, sms = 0, per_sm = 0;
			cudaGetDevice(&dev);
			cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
			cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_energy<EL, T, NT>, NT, 0);
			resident = std::max(1, sms) * std::max(1, per_sm);
		}
		k_energy<EL, T, NT><<<std::min(nb, resident), NT, 0, s>>>(m, u, sc.partials, out, sc.ticket, sc.inverted);
	}
}

template <class EL, int MAT>
static void gen_energy_t(const DevMesh &m, const double *u, bool per_element, double *out, const Scratch &sc, cudaStream_t s)
{
	constexpr int NT = 256;
	const int nb = blocks_for(m.E, NT);
	if (per_element)
		k_gen_energy_per_element<EL, MAT, NT><<<nb, NT, 0, s>>>(m, u, out, sc.inverted);
	else
		k_gen_energy<EL, MAT, NT><<<nb, NT, 0, s>>>(m, u, sc.partials, out, sc.ticket, sc.inverted);
}

template <class EL>
static void gen_energy_mat(const DevMesh &m, const double *u, bool per_element, double *out, const Scratch &sc,
						   cudaStream_t s)
{
	if (m.mat == MAT_ISO_NEOHOOKEAN)
		gen_energy_t<EL, MAT_ISO_NEOHOOKEAN>(m, u, per_element, out, sc, s);
	else
		gen_energy_t<EL, MAT_SAINT_VENANT>(m, u, per_element, out, sc, s);
}

template <class EL>
static void gen_gradient_mat(const DevMesh &m, const double *u, const Scratch &sc, cudaStream_t s)
{
	constexpr int NT = 128;
	if (m.mat == MAT_ISO_NEOHOOKEAN)
		k_gen_gradient<EL, MAT_ISO_NEOHOOKEAN, NT><<<blocks_for(m.E, NT), NT, 0, s>>>(m, u, sc.vec_stage, sc.inverted);
	else
		k_gen_gradient<EL, MAT_SAINT_VENANT, NT><<<blocks_for(m.E, NT), NT, 0, s>>>(m, u, sc.vec_stage, sc.inverted);
}

int energy_elems_per_block(int) { return 256; }

cudaError_t launch_energy(const DevMesh &m, const double *u, int prec, bool per_element, double *out,
						  const Scratch &sc, cudaStream_t s)
{
	if (m.E == 0)
		return per_element ? cudaSuccess : cudaMemsetAsync(out, 0, sizeof(double), s);
	if (m.mat >= MAT_FIRST_AD) return launch_ad_energy(m, u, per_element, out, sc, s);
	if (m.mat != 0) // other materials: FP64 (the caller admits PREC_FP64 only)
	{
		switch (m.et)
		{
		case 1: gen_energy_mat<P1Tet>(m, u, per_element, out, sc, s); break;
		case 2: gen_energy_mat<P2Tet>(m, u, per_element, out, sc, s); break;
		case 3: gen_energy_mat<Q1Hex>(m, u, per_element, out, sc, s); break;
		default: return cudaErrorInvalidValue;
		}
		return cudaGetLastError();
	}
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
static void gradient_t(const DevMesh &m, const double *u, const Scratch &sc, cudaStream_t s)
{
	constexpr int NT = 128;
	k_gradient<EL, T, NT><<<blocks_for(m.E, NT), NT, 0, s>>>(m, u, sc.vec_stage, sc.inverted);
}

cudaError_t launch_gradient(const DevMesh &m, const double *u, int prec, double *g, const Scratch &sc, cudaStream_t s)
{
	if (m.E == 0) return cudaMemsetAsync(g, 0, sizeof(double) * 3 * (size_t)m.N, s);
	const bool f32 = prec != PREC_FP64;
	if (m.mat >= MAT_FIRST_AD)
	{
		cudaError_t e = launch_ad_gradient_stage(m, u, sc, s);
		if (e != cudaSuccess) return e;
	}
	else if (m.mat != 0) // other materials: FP64 (the caller admits PREC_FP64 only)
		switch (m.et)
		{
		case 1: gen_gradient_mat<P1Tet>(m, u, sc, s); break;
		case 2: gen_gradient_mat<P2Tet>(m, u, sc, s); break;
		case 3: gen_gradient_mat<Q1Hex>(m, u, sc, s); break;
		default: return cudaErrorInvalidValue;
		}
	else
		switch (m.et)
		{
		case 1: f32 ? gradient_t<P1Tet, float>(m, u, sc, s) : gradient_t<P1Tet, double>(m, u, sc, s); break;
		case 2: f32 ? gradient_t<P2Tet, float>(m, u, sc, s) : gradient_t<P2Tet, double>(m, u, sc, s); break;
		case 3: f32 ? gradient_t<Q1Hex, float>(m, u, sc, s) : gradient_t<Q1Hex, double>(m, u, sc, s); break;
		default: return cudaErrorInvalidValue;
		}
	launch_vec_gather(m.N, m.inc_off, (long long)m.E * nodes_of(m.et), sc.vec_stage, g, s);
	return cudaGetLastError();
}

cudaError_t launch_material_vjp(const DevMesh &m, const double *u, const double *adj, double *out, cudaStream_t s)
{
	if (m.E == 0) return cudaSuccess;
	if (m.mat != 0) return launch_ad_material_vjp(m, u, adj, out, s);
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

cudaError_t launch_shape_vjp(const DevMesh &m, const double *u, const double *adj, int prec, double *out,
							 const Scratch &sc, cudaStream_t s)
{
	if (m.E == 0) return cudaMemsetAsync(out, 0, sizeof(double) * 3 * (size_t)m.Ng, s);
	constexpr int NT = 128;
	const int nb = blocks_for(m.E, NT);
	const bool f32 = prec != PREC_FP64;
	double *st = sc.vec_stage;
	if (m.mat != 0)
	{
		cudaError_t e = launch_ad_shape_vjp_stage(m, u, adj, sc, s);
		if (e != cudaSuccess) return e;
	}
	else
		switch (m.et)
		{
		case 1: f32 ? k_shape_vjp<P1Tet, float, NT><<<nb, NT, 0, s>>>(m, u, adj, st) : k_shape_vjp<P1Tet, double, NT><<<nb, NT, 0, s>>>(m, u, adj, st); break;
		case 2: f32 ? k_shape_vjp<P2Tet, float, NT><<<nb, NT, 0, s>>>(m, u, adj, st) : k_shape_vjp<P2Tet, double, NT><<<nb, NT, 0, s>>>(m, u, adj, st); break;
		case 3: f32 ? k_shape_vjp<Q1Hex, float, NT><<<nb, NT, 0, s>>>(m, u, adj, st) : k_shape_vjp<Q1Hex, double, NT><<<nb, NT, 0, s>>>(m, u, adj, st); break;
		default: return cudaErrorInvalidValue;
		}
	launch_vec_gather(m.Ng, m.ginc_off, (long long)m.E * geom_nodes_of(m.et), st, out, s);
	return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Dirichlet reduction of vectors (BCLagrangianForm::project_gradient,
// BCLagrangianForm.cpp:149-155; NLProblem::reduced_to_full, NLProblem.cpp:713-735)
// ---------------------------------------------------------------------------
__global__ void k_gather_free(const double *__restrict__ full, const int *__restrict__ free, int n_free,
							  double *__restrict__ out)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n_free) out[i] = __ldg(full + __ldg(free + i));
}

__global__ void k_reduced_to_full(const double *__restrict__ y, const double *__restrict__ x_bc,
								  const int *__restrict__ old_to_new, int ndof, double *__restrict__ x)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= ndof) return;
	const int k = __ldg(old_to_new + i);
	x[i] = k >= 0 ? __ldg(y + k) : (x_bc ? __ldg(x_bc + i) : 0.0);
}

// ---------------------------------------------------------------------------
// utils::lump_matrix (utils/MatrixUtils.cpp:84-101): diag[r] = sum_k M(r, k).  The
// reference walks the CSC column by column and hands every (row, value) to
// setFromTriplets as a diagonal triplet, which sums the duplicates of row r in
// insertion order starting from the first value: ascending column k.  One thread
// per row r = 3A + m reads row r across the columns 3B + c of every neighbour node
// B of A, ascending, through the node-block pattern: in column 3B + c, row r sits
// at outer[3B + c] + 3 rank_B(A) + m, rank_B(A) found by binary search in B's
// neighbour list (rows 3 * rank of column 3B).  The pattern is structurally
// symmetric, so A is always in B's list.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_lump_rows(int n_nodes, const int *__restrict__ outer,
												   const int *__restrict__ inner, const double *__restrict__ vals,
												   double *__restrict__ diag)
{
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= 3 * n_nodes) return;
	const int A = r / 3, m = r - 3 * A;
	const int oA = __ldg(outer + 3 * A), degA = (__ldg(outer + 3 * A + 1) - oA) / 3;
	double s = 0.0;
	bool first = true;
	for (int i = 0; i < degA; ++i)
	{
		const int B = __ldg(inner + oA + 3 * i) / 3;
		const int oB = __ldg(outer + 3 * B), degB = (__ldg(outer + 3 * B + 1) - oB) / 3;
		int lo = 0, hi = degB - 1;
		while (lo < hi)
		{
			const int mid = (lo + hi) >> 1;
			if (__ldg(inner + oB + 3 * mid) / 3 < A)
				lo = mid + 1;
			else
				hi = mid;
		}
#pragma unroll
		for (int c = 0; c < 3; ++c)
		{
			const double v = __ldg(vals + __ldg(outer + 3 * B + c) + 3 * lo + m);
			s = first ? v : s + v;
			first = false;
		}
	}
	diag[r] = s;
}

cudaError_t launch_lump_rows(int n_nodes, const int *outer, const int *inner, const double *vals, double *diag,
							 cudaStream_t s)
{
	const int n = 3 * n_nodes;
	if (n > 0) k_lump_rows<<<(n + 255) / 256, 256, 0, s>>>(n_nodes, outer, inner, vals, diag);
	return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Compositions of formulations: MaterialSum (SumModel.cpp:43-78, the element
// energies, gradients and Hessians of several formulations added) and MultiModels
// (MultiModel.cpp:35-58, the formulation chosen per element).  Each component runs
// its own FP64 element kernels into its own per-element buffers; the combination
// below adds them per element (components ascending), keeping of a MultiModels
// element only its own component's values; the usual tail (energy reduction,
// incidence gather, PSD projection, scatter) then runs on the combined buffers.
// ---------------------------------------------------------------------------
// acc[e * per + i] (=|+=) src[e * per + i] for elements e whose component is comp
// (every element when sel is NULL); first: acc starts from zero
__global__ void k_combine_elements(double *__restrict__ acc, const double *__restrict__ src, long long per, int E,
								   const int *__restrict__ sel, int comp, int first)
{
	const long long total = per * (long long)E;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
	{
		const int e = (int)(i / per);
		const bool on = sel == nullptr || __ldg(sel + e) == comp;
		const double v = on ? __ldg(src + i) : 0.0;
		acc[i] = first ? v : acc[i] + v;
	}
}

// the same over the 32-byte incidence slots of the gradient stage (slot k belongs to
// element inc_eb[k] / n)
__global__ void k_combine_slots(double *__restrict__ acc, const double *__restrict__ src, long long n_inc, int n,
								const int *__restrict__ inc_eb, const int *__restrict__ sel, int comp, int first)
{
	for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n_inc; k += (long long)gridDim.x * blockDim.x)
	{
		const bool on = sel == nullptr || __ldg(sel + __ldg(inc_eb + k) / n) == comp;
#pragma unroll
		for (int c = 0; c < 4; ++c)
		{
			const double v = on ? __ldg(src + 4 * k + c) : 0.0;
			acc[4 * k + c] = first ? v : acc[4 * k + c] + v;
		}
	}
}

// the sum of x[0..n), fixed order (grid-stride per thread, block tree, block
// partials in index order by the last block): deterministic
template <int NT>
__global__ void __launch_bounds__(NT) k_sum_array(const double *__restrict__ x, int n, double *__restrict__ partials,
												  double *__restrict__ result, unsigned int *ticket)
{
	double v = 0.0;
	for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) v += __ldg(x + i);
	reduce_to_result<NT>(v, partials, result, ticket);
}

static inline int combine_blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 16); }

cudaError_t launch_combine_elements(double *acc, const double *src, long long per, int E, const int *sel, int comp,
									bool first, cudaStream_t s)
{
	if (per * (long long)E > 0)
		k_combine_elements<<<combine_blocks(per * (long long)E), 256, 0, s>>>(acc, src, per, E, sel, comp, first ? 1 : 0);
	return cudaGetLastError();
}

cudaError_t launch_combine_slots(double *acc, const double *src, long long n_inc, int n, const int *inc_eb, const int *sel,
								 int comp, bool first, cudaStream_t s)
{
	if (n_inc > 0) k_combine_slots<<<combine_blocks(n_inc), 256, 0, s>>>(acc, src, n_inc, n, inc_eb, sel, comp, first ? 1 : 0);
	return cudaGetLastError();
}

cudaError_t launch_sum_array(const double *x, int n, double *out, const Scratch &sc, cudaStream_t s)
{
	constexpr int NT = 256;
	if (n <= 0) return cudaMemsetAsync(out, 0, sizeof(double), s);
	const int nb = std::min(blocks_for(n, NT), sc.max_blocks);
	k_sum_array<NT><<<nb, NT, 0, s>>>(x, n, sc.partials, out, sc.ticket);
	return cudaGetLastError();
}

// pass 1 alone in FP64: the element block triangles of the context's material
cudaError_t launch_fp64_blocks(const DevMesh &m, const double *u, double *stage, cudaStream_t s)
{
	if (m.E <= 0) return cudaSuccess;
	if (m.mat >= MAT_FIRST_AD) return launch_ad_blocks(m, u, stage, s);
	auto gen = [&](auto el) -> cudaError_t {
		using EL = decltype(el);
		constexpr int WPB = 4;
		const size_t bytes = WPB * sizeof(GenWarp<EL>);
		const int nb = std::min((m.E + WPB - 1) / WPB, 148 * 32);
		cudaError_t e;
		if (m.mat == MAT_ISO_NEOHOOKEAN)
		{
			e = cudaFuncSetAttribute(k_gen_blocks<EL, MAT_ISO_NEOHOOKEAN, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
			if (e == cudaSuccess) k_gen_blocks<EL, MAT_ISO_NEOHOOKEAN, WPB><<<nb, WPB * 32, bytes, s>>>(m, u, stage);
		}
		else
		{
			e = cudaFuncSetAttribute(k_gen_blocks<EL, MAT_SAINT_VENANT, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
			if (e == cudaSuccess) k_gen_blocks<EL, MAT_SAINT_VENANT, WPB><<<nb, WPB * 32, bytes, s>>>(m, u, stage);
		}
		return e != cudaSuccess ? e : cudaGetLastError();
	};
	auto nh = [&](auto el) -> cudaError_t {
		using EL = decltype(el);
		using TL = EcTile<EL, double>;
		const size_t bytes1 = sizeof(EcSmem<EL, double, double>);
		cudaError_t e = cudaFuncSetAttribute(k_hessian_blocks<EL, double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes1);
		if (e != cudaSuccess) return e;
		k_hessian_blocks<EL, double, double><<<(m.E + TL::TE - 1) / TL::TE, TL::NT, bytes1, s>>>(m, u, stage, 0, m.E);
		return cudaGetLastError();
	};
	switch (m.et)
	{
	case 1: return m.mat ? gen(P1Tet{}) : nh(P1Tet{});
	case 2: return m.mat ? gen(P2Tet{}) : nh(P2Tet{});
	case 3: return m.mat ? gen(Q1Hex{}) : nh(Q1Hex{});
	}
	return cudaErrorInvalidValue;
}

// projection (optional) and scatter of FP64 block triangles
cudaError_t launch_fp64_finish(const DevMesh &m, const DevPattern &p, double *stage, bool project_psd, cudaStream_t s)
{
	if (p.nnz == 0) return cudaSuccess;
	switch (m.et)
	{
	case 1: return finish_fp64_hessian<P1Tet>(m, p, stage, project_psd, s);
	case 2: return finish_fp64_hessian<P2Tet>(m, p, stage, project_psd, s);
	case 3: return finish_fp64_hessian<Q1Hex>(m, p, stage, project_psd, s);
	}
	return cudaErrorInvalidValue;
}

// the gradient's incidence slots alone (FP64), and their gather
cudaError_t launch_gradient_stage(const DevMesh &m, const double *u, const Scratch &sc, cudaStream_t s)
{
	if (m.E == 0) return cudaSuccess;
	if (m.mat >= MAT_FIRST_AD) return launch_ad_gradient_stage(m, u, sc, s);
	if (m.mat != 0)
		switch (m.et)
		{
		case 1: gen_gradient_mat<P1Tet>(m, u, sc, s); break;
		case 2: gen_gradient_mat<P2Tet>(m, u, sc, s); break;
		case 3: gen_gradient_mat<Q1Hex>(m, u, sc, s); break;
		default: return cudaErrorInvalidValue;
		}
	else
		switch (m.et)
		{
		case 1: gradient_t<P1Tet, double>(m, u, sc, s); break;
		case 2: gradient_t<P2Tet, double>(m, u, sc, s); break;
		case 3: gradient_t<Q1Hex, double>(m, u, sc, s); break;
		default: return cudaErrorInvalidValue;
		}
	return cudaGetLastError();
}

cudaError_t launch_gradient_gather(const DevMesh &m, const double *stage, double *g, cudaStream_t s)
{
	if (m.E == 0) return cudaMemsetAsync(g, 0, sizeof(double) * 3 * (size_t)m.N, s);
	launch_vec_gather(m.N, m.inc_off, (long long)m.E * nodes_of(m.et), stage, g, s);
	return cudaGetLastError();
}

// DenseMatrixCache (utils/MatrixCache.hpp:136-177): the matrix in the Hessian pattern
// as a dense column-major ndof x ndof array.  One warp per column; every entry of
// the pattern is written once, the rest of the column is zero (cleared before).
__global__ void k_csc_to_dense(int ndof, const int *__restrict__ outer, const int *__restrict__ inner,
							   const double *__restrict__ vals, double *__restrict__ dense)
{
	const int col = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
	if (col >= ndof) return;
	double *d = dense + (size_t)col * ndof;
	for (int k = __ldg(outer + col) + lane; k < __ldg(outer + col + 1); k += 32) d[__ldg(inner + k)] = __ldg(vals + k);
}

cudaError_t launch_csc_to_dense(int ndof, const int *outer, const int *inner, const double *vals, double *dense,
								cudaStream_t s)
{
	if (ndof <= 0) return cudaSuccess;
	cudaError_t e = cudaMemsetAsync(dense, 0, sizeof(double) * (size_t)ndof * (size_t)ndof, s);
	if (e != cudaSuccess) return e;
	k_csc_to_dense<<<(int)(((size_t)ndof * 32 + 255) / 256), 256, 0, s>>>(ndof, outer, inner, vals, dense);
	return cudaGetLastError();
}

cudaError_t launch_gather_free(const double *full, const int *free, int n_free, double *out, cudaStream_t s)
{
	if (n_free > 0) k_gather_free<<<(n_free + 255) / 256, 256, 0, s>>>(full, free, n_free, out);
	return cudaGetLastError();
}

cudaError_t launch_reduced_to_full(const double *y, const double *x_bc, const int *old_to_new, int ndof, double *x,
								   cudaStream_t s)
{
	if (ndof > 0) k_reduced_to_full<<<(ndof + 255) / 256, 256, 0, s>>>(y, x_bc, old_to_new, ndof, x);
	return cudaGetLastError();
}

} // namespace pfg
