// Element traits, reference-element tables and small dense math for the
// NeoHookean assembly kernels (sm_100a).
//
// The quadrature rules and reference basis gradients are the reference's
// tables, evaluated at compile time so that every ∇φ̂ entry becomes an
// immediate operand and the zero entries fold away:
//   P1 tet : 1 point (1/4,1/4,1/4), w = 1/6          (quadrature/TetQuadrature.cpp:43-55,
//                                                     autogen/auto_tetrahedron.ipp:1-6)
//   P2 tet : Hammer-Marlowe-Stroud 4 points, w = 1/24 (autogen/auto_tetrahedron.ipp:7-12)
//            basis gradients of autogen/auto_p_bases.cpp:1248-1306
//   Q1 hex : 2x2x2 Gauss on [0,1], w = 1/8, point index (i*2+j)*2+k -> (x_k, x_j, x_i)
//            (quadrature/HexQuadrature.cpp:17-44, LineQuadrature.cpp:4708-4740)
//            basis gradients of autogen/auto_q_bases_3d_grad_1.cpp:7-53
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace pfg
{

struct P1Tet
{
	static constexpr int ET = 1, N = 4, NG = 4, NQ = 1;
	static constexpr bool AFFINE = true;
};
struct P2Tet
{
	static constexpr int ET = 2, N = 10, NG = 4, NQ = 4;
	static constexpr bool AFFINE = true;
};
struct Q1Hex
{
	static constexpr int ET = 3, N = 8, NG = 8, NQ = 8;
	static constexpr bool AFFINE = false;
};

// ---- quadrature -----------------------------------------------------------
__host__ __device__ constexpr double hms_a() { return 0.13819660112501053195188660538406111299991607666015625; }
__host__ __device__ constexpr double hms_b() { return 0.58541019662496840414434018384781666100025177001953125; }
// 2-point Gauss-Legendre mapped to [0,1] the way LineQuadrature does it: x/2 + 0.5
__host__ __device__ constexpr double gl2(int k)
{
	return k == 0 ? (-0.57735026918962576450914878050195745564760175127012687601860232648397767 / 2) + 0.5
				  : (0.57735026918962576450914878050195745564760175127012687601860232648397767 / 2) + 0.5;
}

template <class EL>
__host__ __device__ constexpr double qweight(int)
{
	if constexpr (EL::ET == 1)
		return 1.0 / 6.0;
	else if constexpr (EL::ET == 2)
		return 0.25 / 6.0;
	else
		return 0.125;
}

template <class EL>
__host__ __device__ constexpr double qpoint(int q, int d)
{
	if constexpr (EL::ET == 1)
		return 0.25;
	else if constexpr (EL::ET == 2)
	{
		// rows (a,a,b), (a,b,a), (b,a,a), (a,a,a)
		return (q == 3) ? hms_a() : ((d == 2 - q) ? hms_b() : hms_a());
	}
	else
	{
		// index (i*2+j)*2+k -> (x_k, x_j, x_i)
		const int i = (q >> 2) & 1, j = (q >> 1) & 1, k = q & 1;
		return d == 0 ? gl2(k) : (d == 1 ? gl2(j) : gl2(i));
	}
}

// ---- reference basis gradients ---------------------------------------------
__host__ __device__ constexpr double p1_grad(int a, int r)
{
	return a == 0 ? -1.0 : (a - 1 == r ? 1.0 : 0.0);
}

__host__ __device__ constexpr double p2_grad(int i, int r, double x, double y, double z)
{
	switch (i)
	{
	case 0: return 4 * x + 4 * y + 4 * z - 3;
	case 1: return r == 0 ? 4 * x - 1 : 0.0;
	case 2: return r == 1 ? 4 * y - 1 : 0.0;
	case 3: return r == 2 ? 4 * z - 1 : 0.0;
	case 4: return r == 0 ? 4 * (-2 * x - y - z + 1) : -4 * x;
	case 5: return r == 0 ? 4 * y : (r == 1 ? 4 * x : 0.0);
	case 6: return r == 1 ? 4 * (-x - 2 * y - z + 1) : -4 * y;
	case 7: return r == 2 ? 4 * (-x - y - 2 * z + 1) : -4 * z;
	case 8: return r == 0 ? 4 * z : (r == 2 ? 4 * x : 0.0);
	default: return r == 1 ? 4 * z : (r == 2 ? 4 * y : 0.0);
	}
}

__host__ __device__ constexpr double q1_grad(int i, int r, double x, double y, double z)
{
	switch (i)
	{
	case 0: return r == 0 ? -1.0 * (y - 1) * (z - 1) : (r == 1 ? -1.0 * (x - 1) * (z - 1) : -1.0 * (x - 1) * (y - 1));
	case 1: return r == 0 ? 1.0 * (y - 1) * (z - 1) : (r == 1 ? 1.0 * x * (z - 1) : 1.0 * x * (y - 1));
	case 2: return r == 0 ? -1.0 * y * (z - 1) : (r == 1 ? -1.0 * x * (z - 1) : -1.0 * x * y);
	case 3: return r == 0 ? 1.0 * y * (z - 1) : (r == 1 ? 1.0 * (x - 1) * (z - 1) : 1.0 * y * (x - 1));
	case 4: return r == 0 ? 1.0 * z * (y - 1) : (r == 1 ? 1.0 * z * (x - 1) : 1.0 * (x - 1) * (y - 1));
	case 5: return r == 0 ? -1.0 * z * (y - 1) : (r == 1 ? -1.0 * x * z : -1.0 * x * (y - 1));
	case 6: return r == 0 ? 1.0 * y * z : (r == 1 ? 1.0 * x * z : 1.0 * x * y);
	default: return r == 0 ? -1.0 * y * z : (r == 1 ? -1.0 * z * (x - 1) : -1.0 * y * (x - 1));
	}
}

// FE basis gradient in reference coordinates at quadrature point q
template <class EL>
__host__ __device__ constexpr double gref(int q, int a, int r)
{
	if constexpr (EL::ET == 1)
		return p1_grad(a, r);
	else if constexpr (EL::ET == 2)
		return p2_grad(a, r, qpoint<EL>(q, 0), qpoint<EL>(q, 1), qpoint<EL>(q, 2));
	else
		return q1_grad(a, r, qpoint<EL>(q, 0), qpoint<EL>(q, 1), qpoint<EL>(q, 2));
}

// Geometric basis gradient in reference coordinates (P1 for both tets)
template <class EL>
__host__ __device__ constexpr double ggref(int q, int a, int r)
{
	if constexpr (EL::ET == 3)
		return q1_grad(a, r, qpoint<EL>(q, 0), qpoint<EL>(q, 1), qpoint<EL>(q, 2));
	else
		return p1_grad(a, r);
}

// ---- 3x3 math -----------------------------------------------------------------
template <class T>
__device__ __forceinline__ T det3(const T m[3][3])
{
	return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1])
		 - m[1][0] * (m[0][1] * m[2][2] - m[0][2] * m[2][1])
		 + m[2][0] * (m[0][1] * m[1][2] - m[0][2] * m[1][1]);
}

// inverse transpose via cofactors: it[r][c] = cof(m)[r][c] / det
template <class T>
__device__ __forceinline__ void inv_transpose3(const T m[3][3], T det, T it[3][3])
{
	const T id = T(1) / det;
	it[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * id;
	it[0][1] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * id;
	it[0][2] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * id;
	it[1][0] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
	it[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
	it[1][2] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
	it[2][0] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
	it[2][1] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
	it[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
}

// cofactor matrix of F = dJ/dF: columns (v x w, w x u, u x v) with u,v,w the columns of F
template <class T>
__device__ __forceinline__ void cofactor3(const T F[3][3], T D[3][3])
{
	D[0][0] = F[1][1] * F[2][2] - F[2][1] * F[1][2];
	D[1][0] = F[2][1] * F[0][2] - F[0][1] * F[2][2];
	D[2][0] = F[0][1] * F[1][2] - F[1][1] * F[0][2];
	D[0][1] = F[1][2] * F[2][0] - F[2][2] * F[1][0];
	D[1][1] = F[2][2] * F[0][0] - F[0][2] * F[2][0];
	D[2][1] = F[0][2] * F[1][0] - F[1][2] * F[0][0];
	D[0][2] = F[1][0] * F[2][1] - F[2][0] * F[1][1];
	D[1][2] = F[2][0] * F[0][1] - F[0][0] * F[2][1];
	D[2][2] = F[0][0] * F[1][1] - F[1][0] * F[0][1];
}

// Jacobian of the geometric map at quadrature point q (rows = d/dxi_r),
// as ElementAssemblyValues::finalize3d builds it (ElementAssemblyValues.cpp:76-94).
template <class EL, class T>
__device__ __forceinline__ void geom_jacobian(int q, const T Xg[EL::NG][3], T Jac[3][3])
{
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c)
		{
			T s = T(0);
#pragma unroll
			for (int j = 0; j < EL::NG; ++j)
			{
				const double gg = ggref<EL>(q, j, r);
				if (gg != 0.0) s += T(gg) * Xg[j][c];
			}
			Jac[r][c] = s;
		}
}

} // namespace pfg
