// Tensor-core element Hessians for the split-precision mode (sm_100a: tcgen05,
// TMEM, bulk-async copies).
//
// The NeoHookean element block of NeoHookeanElasticity.cpp:547-658 is
//   H_e(3a+r, 3b+c) = sum_q da [ mu (g_a.g_b) d_rc + lambda d_a[r] d_b[c]
//                                + (mu - lambda ln J) d_b[r] d_a[c] ],
// with g_a = J^-T-mapped reference gradient and d_a = F^-T g_a (the reduced
// form of B^T C B).  Writing g_a = Jit^T gh_a(q) and d_a = Kt gh_a(q), with
// gh_a(q) the reference-element gradient (a constant of the element type),
// Kt = F^-T Jit^T and G = Jit Jit^T, every entry becomes
//   H_e(3a+r, 3b+c) = sum_{q,k,l} gh_a[k](q) gh_b[l](q) W_e[(r,c), (k,l,q)],
//   W_e[(r,c),(k,l,q)] = da [ mu G[k][l] d_rc + lambda Kt[r][k] Kt[c][l]
//                             + (mu - lambda ln J) Kt[c][k] Kt[r][l] ],
// i.e. one GEMM per tile of elements:
//   D[(e, r, c), (a <= b)] = sum_j W[(e, r, c), j] * Phi[(a, b), j]
// with M = 9 rows per element (14 elements per 128-row tile), K = 9 NQ
// (P2 36 -> 40, Q1 72) and N = the n(n+1)/2 node pairs (P2 55 -> 64, Q1 36 -> 48).
// Phi (the products of reference gradients) is the same for every element: it
// is built once per device, and each CTA stages it into shared memory once with
// one bulk (TMA) copy.
//
// Precision (split32): J^-T, F, det/log J, F^-T, Kt and G in FP64; W in FP32;
// both operands split into TF32 pairs (x = hi + lo, each rounded to nearest)
// and multiplied as hi*hi + hi*lo + lo*hi (the lo*lo term is below 2^-22
// relative), accumulated in FP32 in TMEM by tcgen05.mma kind::tf32.  The
// element blocks leave as the packed FP32 block triangles the reduction kernel
// reads (tri_index order, [c][r]), written by one bulk copy per tile.
//
// CTA roles (256 threads): warps 4-7 gather the tile's nodes, u, X and the Lame
// pair and compute the per-(element, point) kinematics into one of two
// buffers; warps 0-3 turn a buffer into the A operand, thread 0 issues the
// MMAs, and each of warps 0-3 reads its 32 TMEM lanes (rows) back.  Named
// barriers hand the two kinematics buffers back and forth, so the gathers of
// the next tile overlap the MMA and the write-out of this one.  Every wait on an
// mbarrier is bounded; when one gives up, the kernel records it in the
// context's error flag, skips the remaining tensor-core work and still frees
// its TMEM.
#include "pfg_internal.h"
#include "pfg_elem.cuh"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace pfg
{
namespace
{

// ---------------------------------------------------------------------------
// tile shape per element type
// ---------------------------------------------------------------------------
template <class EL>
struct TcCfg
{
	static constexpr int N = EL::N, NG = EL::NG, NQ = EL::NQ;
	static constexpr int NP = N * (N + 1) / 2;         // node pairs a <= b
	static constexpr int NPAD = (NP + 15) / 16 * 16;   // MMA N (multiple of 16 for M = 128)
	// The K dimension runs in parts of four points (Q1: two parts) through one A
	// buffer, so that the A operand of an 8-point element fits two CTAs per SM.
	static constexpr int NQH = NQ < 4 ? NQ : 4;        // points per part
	static constexpr int KH = NQ / NQH;                // parts
	static constexpr int KD = 9 * NQH;                 // (k, l, q) of one part
	static constexpr int KP = (KD + 7) / 8 * 8;        // MMA K of a part, padded to the TF32 K step of 8
	static constexpr int KC = KP / 4;                  // 16-byte K chunks (4 TF32 values)
	static constexpr int TE = 14;                      // elements per 128-row tile (9 rows each)
	static constexpr int ROWS = 9 * TE;                // 126 valid rows of 128
	static constexpr int TP = tri_pad(N);              // floats per staged block triangle
	static constexpr int KIN = 24;                     // floats per (element, point) record
	static constexpr uint32_t TMEM_COLS = 64;          // power of two >= NPAD
	static constexpr uint32_t A_CHUNK = 128 * 16;      // bytes of one K chunk of A (128 rows)
	static constexpr uint32_t B_CHUNK = NPAD * 16;     // bytes of one K chunk of B
	static constexpr uint32_t B_PART = 2u * KC * B_CHUNK;   // hi and lo halves of one part of Phi
	static constexpr uint32_t B_BYTES = KH * B_PART;
	static_assert(NPAD <= (int)TMEM_COLS, "accumulator must fit the TMEM allocation");
	static_assert(KD <= KP && KP % 8 == 0, "K padding");
	static_assert(NQH == 4 && NQ % NQH == 0, "K order groups four points of one (k, l) in a 16-byte chunk");
	static_assert(TE * TP <= 2 * KC * 128 * 4, "the block triangles must fit the A operand's bytes");
};

// Shared memory of one CTA.  A and B use the canonical K-major layout without
// swizzle: a K chunk is 16 bytes (4 TF32) of every row, rows 16 bytes apart,
// consecutive chunks A_CHUNK / B_CHUNK bytes apart (LBO), 8-row groups 128
// bytes apart (SBO).  K index within part h: j = (3k + l) * 4 + (q - 4h).
template <class EL>
struct TcSmem
{
	using C = TcCfg<EL>;
	// A operand (hi, lo); once the tile's MMAs have completed the same bytes hold
	// the tile's block triangles for the bulk store ([TE][TP] floats)
	union
	{
		struct
		{
			alignas(1024) float Ah[C::KC][128][4];
			alignas(1024) float Al[C::KC][128][4];
		};
		alignas(1024) float out[C::TE * C::TP];
	};
	alignas(1024) float B[C::KH][2][C::KC][C::NPAD][4]; // Phi per part: hi then lo, all parts contiguous (one bulk copy)
	alignas(16) float kin[2][C::TE][C::NQ][C::KIN];
	// gathered inputs, two tiles: the next tile's copies are in flight while this
	// tile's kinematics run
	double U[2][C::TE][C::N][3];
	double X[2][C::TE][C::NG][3];
	double2 lame[2][C::TE];
	int nodes[2][C::TE][C::N + C::NG];
	double geo[EL::AFFINE ? 2 : 1][C::TE][20]; // affine elements: J (9), G = J^-T J^-1 (9), det J
	double gtab[C::NQ][C::N][3];
	double ggtab[EL::AFFINE ? 1 : C::NQ][C::NG][3];
	double wq[C::NQ];
	alignas(8) unsigned long long bar_b;   // Phi bulk copy
	unsigned long long bar_mma;            // MMA completion (tcgen05.commit)
	uint32_t tmem_base;
	int abort;                             // a bounded wait gave up: skip the tensor-core work
};

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile("{\n\t.reg .pred p;\n\t"
				 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
				 "selp.u32 %0, 1, 0, p;\n\t}"
				 : "=r"(ok)
				 : "r"(smem_u32(bar)), "r"(parity)
				 : "memory");
	return ok != 0;
}
// Bounded wait on a phase of an mbarrier: false when it gave up (each try_wait
// itself suspends for a while before returning false, so this is seconds).
constexpr int MBAR_TRIES = 1 << 22;
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity)
{
	for (int i = 0; i < MBAR_TRIES; ++i)
		if (mbar_try_wait(bar, parity)) return true;
	return false;
}
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src_gmem, uint32_t bytes, unsigned long long *bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
					 smem_u32(dst_smem)),
				 "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
				 : "memory");
}
__device__ __forceinline__ void bulk_store(void *dst_gmem, const void *src_smem, uint32_t bytes)
{
	asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem), "r"(smem_u32(src_smem)),
				 "r"(bytes)
				 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)), "r"(ncols)
				 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, kind::tf32, one CTA, FP32 accumulate
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
	asm volatile("{\n\t.reg .pred p;\n\t"
				 "setp.ne.b32 p, %4, 0;\n\t"
				 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
				 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
				 : "memory");
}
__device__ __forceinline__ void mma_commit(unsigned long long *bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
				 : "memory");
}

// 32 (or 16) consecutive accumulator columns of the warp's 32 lanes, waited on in
// the same statement so that no use of the registers can be scheduled before the wait
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
	uint32_t r[32];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
				 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
				 "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
				 "tcgen05.wait::ld.sync.aligned;"
				 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
				   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
				   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
				   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
				 : "r"(taddr)
				 : "memory");
#pragma unroll
	for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
	uint32_t r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
				 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
				 "tcgen05.wait::ld.sync.aligned;"
				 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
				   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
				 : "r"(taddr)
				 : "memory");
#pragma unroll
	for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void named_arrive(int id, int n) { asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// Shared-memory matrix descriptor, canonical K-major layout without swizzle
// (start address, leading (K-chunk) byte offset, stride (8-row group) byte offset;
// bits 46-47 = 1 for this descriptor version, swizzle mode 0)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
	return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
		   ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::tf32: F32 accumulator, A and B TF32, both K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N)
{
	return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// round to the nearest TF32 (10 explicit mantissa bits), ties away from zero
__host__ __device__ __forceinline__ float tf32_round(float x)
{
#ifdef __CUDA_ARCH__
	return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
#else
	uint32_t b;
	std::memcpy(&b, &x, 4);
	b = (b + 0x1000u) & 0xFFFFE000u;
	float y;
	std::memcpy(&y, &b, 4);
	return y;
#endif
}

// ---------------------------------------------------------------------------
// Phi tables (device globals, filled per device at context creation): hi half
// then lo half, each [KC][NPAD][4] in the smem layout above.
// ---------------------------------------------------------------------------
__device__ __align__(128) float g_phi_p2[TcCfg<P2Tet>::B_BYTES / 4];
__device__ __align__(128) float g_phi_q1[TcCfg<Q1Hex>::B_BYTES / 4];

template <class EL>
std::vector<float> build_phi()
{
	using C = TcCfg<EL>;
	std::vector<float> t(C::B_BYTES / 4, 0.f);
	int p = 0;
	for (int a = 0; a < C::N; ++a)
		for (int b = a; b < C::N; ++b, ++p)
			for (int k = 0; k < 3; ++k)
				for (int l = 0; l < 3; ++l)
					for (int q = 0; q < C::NQ; ++q)
					{
						const double x = gref<EL>(q, a, k) * gref<EL>(q, b, l);
						const float h = tf32_round((float)x);
						const float r = tf32_round((float)(x - (double)h));
						const int part = q / C::NQH, j = (3 * k + l) * C::NQH + (q - part * C::NQH);
						float *hi = t.data() + (size_t)part * (C::B_PART / 4);
						float *lo = hi + C::KC * C::NPAD * 4;
						const size_t off = ((size_t)(j / 4) * C::NPAD + p) * 4 + (j % 4);
						hi[off] = h;
						lo[off] = r;
					}
	return t;
}

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------
constexpr int TC_THREADS = 256;
constexpr int BAR_FULL0 = 1, BAR_EMPTY0 = 3, BAR_LOAD = 5, BAR_MATH = 6;

// CTAs per SM that the shared memory allows (the register budget follows it)
template <class EL>
constexpr int tc_min_ctas()
{
	return (int)((227 * 1024) / (sizeof(TcSmem<EL>) + 1024)) >= 2 ? 2 : 1;
}

template <class EL>
__global__ void __launch_bounds__(TC_THREADS, tc_min_ctas<EL>())
	k_hessian_blocks_tc(DevMesh m, const double *__restrict__ u, const float *__restrict__ phi,
						float *__restrict__ stage, int ntiles)
{
	using C = TcCfg<EL>;
	constexpr int TE = C::TE, N = C::N, NG = C::NG, NQ = C::NQ, TP = C::TP;
	extern __shared__ __align__(1024) unsigned char smem_raw[];
	TcSmem<EL> &S = *reinterpret_cast<TcSmem<EL> *>(smem_raw);
	const int tid = threadIdx.x, warp = tid >> 5;

	// ---- set-up: TMEM, barriers, constant tables, zero padding of A ----
	if (warp == 0)
	{
		tmem_alloc(&S.tmem_base, C::TMEM_COLS);
		tmem_relinquish();
	}
	if (tid == 0)
	{
		mbar_init(&S.bar_b, 1);
		mbar_init(&S.bar_mma, 1);
		fence_mbar_init();
		S.abort = 0;
	}
	for (int i = tid; i < NQ * N * 3; i += TC_THREADS)
	{
		const int q = i / (N * 3), a = (i / 3) % N, r = i % 3;
		S.gtab[q][a][r] = gref<EL>(q, a, r);
	}
	constexpr int GQ = EL::AFFINE ? 1 : NQ;
	for (int i = tid; i < GQ * NG * 3; i += TC_THREADS)
	{
		const int q = i / (NG * 3), j = (i / 3) % NG, r = i % 3;
		S.ggtab[q][j][r] = ggref<EL>(q, j, r);
	}
	if (tid < NQ) S.wq[tid] = qweight<EL>(tid);
	// K padding columns (never written by the tiles) and rows 126-127: zero
	for (int i = tid; i < C::KC * 128; i += TC_THREADS)
	{
		const int kc = i / 128, row = i % 128;
		if (kc * 4 >= C::KD || row >= C::ROWS)
		{
			*reinterpret_cast<float4 *>(S.Ah[kc][row]) = make_float4(0.f, 0.f, 0.f, 0.f);
			*reinterpret_cast<float4 *>(S.Al[kc][row]) = make_float4(0.f, 0.f, 0.f, 0.f);
		}
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (tid == 0)
	{
		mbar_expect_tx(&S.bar_b, C::B_BYTES);
		bulk_load(&S.B[0][0][0][0][0], phi, C::B_BYTES, &S.bar_b);
	}
	const uint32_t tmem = S.tmem_base;

	if (warp >= 4)
	{
		// ================= load group: nodes, gathers, kinematics =================
		// Pipeline over this CTA's tiles (buffers by tile parity, loads in flight in
		// registers): while tile t's kinematics run, the u / X / Lame values of the next
		// tile and the node ids of the tile after it are in flight, and (affine
		// elements) the otherwise idle warps compute the next tile's geometry.
		const int lt = tid - 128;
		constexpr int NJ = N + NG, NR = (TE * NJ + 127) / 128;
		constexpr int NU = TE * N * 3, NX = TE * NG * 3, NV = (NU + NX + 127) / 128;
		constexpr int GEO0 = ((TE * NQ + 31) / 32) * 32; // first thread of the geometry group
		static_assert(!EL::AFFINE || GEO0 + TE <= 128, "the geometry group needs idle producer threads");
		int nr[NR];
		double gv[NV];
		double2 glm = make_double2(0.0, 0.0);
		auto load_nodes = [&](int tt) {
			const int e0 = tt * TE, ne = min(TE, m.E - e0);
#pragma unroll
			for (int k = 0; k < NR; ++k)
			{
				const int i = lt + 128 * k, j = i / TE, el = i % TE, e = e0 + el;
				int v = 0;
				if (i < TE * NJ && el < ne)
					v = (j < N) ? __ldg(m.conn + (size_t)j * m.E + e) : __ldg(m.gconn + (size_t)(j - N) * m.E + e);
				nr[k] = v;
			}
		};
		auto store_nodes = [&](int b) {
#pragma unroll
			for (int k = 0; k < NR; ++k)
			{
				const int i = lt + 128 * k;
				if (i < TE * NJ) S.nodes[b][i % TE][i / TE] = nr[k];
			}
		};
		auto load_values = [&](int b, int tt) { // node ids of tile tt in nodes[b]
			const int e0 = tt * TE, ne = min(TE, m.E - e0);
#pragma unroll
			for (int k = 0; k < NV; ++k)
			{
				const int i = lt + 128 * k;
				double v = 0.0;
				if (i < NU)
				{
					const int el = i / (N * 3), a = (i / 3) % N, d = i % 3;
					if (el < ne) v = __ldg(u + (size_t)S.nodes[b][el][a] * 3 + d);
				}
				else if (i < NU + NX)
				{
					const int i2 = i - NU, el = i2 / (NG * 3), j = (i2 / 3) % NG, d = i2 % 3;
					if (el < ne) v = __ldg(m.X + (size_t)S.nodes[b][el][N + j] * 3 + d);
				}
				gv[k] = v;
			}
			if (lt < TE) glm = lt < ne ? __ldg(m.lame + e0 + lt) : make_double2(0.0, 0.0);
		};
		auto store_values = [&](int b) {
#pragma unroll
			for (int k = 0; k < NV; ++k)
			{
				const int i = lt + 128 * k;
				if (i < NU)
					S.U[b][i / (N * 3)][(i / 3) % N][i % 3] = gv[k];
				else if (i < NU + NX)
				{
					const int i2 = i - NU;
					S.X[b][i2 / (NG * 3)][(i2 / 3) % NG][i2 % 3] = gv[k];
				}
			}
			if (lt < TE) S.lame[b][lt] = glm;
		};
		// affine elements: J, det J and G = J^-T J^-1 of element el of the tile whose
		// node ids are in nodes[b], read straight from X
		auto geometry = [&](int b, int el, bool valid) {
			double *geo = S.geo[b][el];
			if (!valid)
			{
				for (int k = 0; k < 19; ++k) geo[k] = k == 18 ? 1.0 : 0.0;
				return;
			}
			double Xe[NG][3];
#pragma unroll
			for (int j = 0; j < NG; ++j)
#pragma unroll
				for (int d = 0; d < 3; ++d) Xe[j][d] = __ldg(m.X + (size_t)S.nodes[b][el][N + j] * 3 + d);
			double Jac[3][3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c)
				{
					double s_ = 0.0;
#pragma unroll
					for (int j = 0; j < NG; ++j) s_ += S.ggtab[0][j][r] * Xe[j][c];
					Jac[r][c] = s_;
				}
			const double detJ = det3(Jac);
			double Jit[3][3];
			inv_transpose3(Jac, detJ, Jit);
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c)
				{
					geo[3 * r + c] = Jac[r][c];
					geo[9 + 3 * r + c] = Jit[r][0] * Jit[c][0] + Jit[r][1] * Jit[c][1] + Jit[r][2] * Jit[c][2];
				}
			geo[18] = detJ;
		};
		int t = blockIdx.x;
		if (t < ntiles)
		{
			load_nodes(t);
			store_nodes(0);
		}
		named_sync(BAR_LOAD, 128);
		if (t < ntiles)
		{
			load_values(0, t);
			if constexpr (EL::AFFINE)
				if (lt >= GEO0 && lt < GEO0 + TE) geometry(0, lt - GEO0, lt - GEO0 < min(TE, m.E - t * TE));
		}
		if (t + (int)gridDim.x < ntiles) load_nodes(t + gridDim.x);
		int it = 0;
		for (; t < ntiles; t += gridDim.x, ++it)
		{
			const int buf = it & 1, g = it & 1;
			const int tn = t + gridDim.x, tnn = tn + gridDim.x;
			store_values(g);
			if (tn < ntiles) store_nodes(g ^ 1);
			named_sync(BAR_LOAD, 128); // this tile's inputs and geometry are in place; the other buffers are free
			if (tn < ntiles) load_values(g ^ 1, tn);
			if (tnn < ntiles) load_nodes(tnn);
			const int e0 = t * TE, ne = min(TE, m.E - e0);
			if constexpr (EL::AFFINE)
				if (lt >= GEO0 && lt < GEO0 + TE && tn < ntiles)
					geometry(g ^ 1, lt - GEO0, lt - GEO0 < min(TE, m.E - tn * TE));
			if (it >= 2) named_sync(BAR_EMPTY0 + buf, TC_THREADS);
			for (int i = lt; i < TE * NQ; i += 128)
			{
				const int el = i / NQ, q = i % NQ;
				float *rec = S.kin[buf][el][q];
				if (el >= ne)
				{
#pragma unroll
					for (int k = 0; k < C::KIN; ++k) rec[k] = 0.f;
					continue;
				}
				// With M = J^T + sum_a u_a (x) grad_ref(phi_a) (the deformed map's gradient,
				// rows spatial, columns reference): F = M J^-T, so det F = det M / det J and
				// Kt = F^-T J^-1 = M^-T; and G = J^-T J^-1 depends on the geometry only.
				const double(*gq)[3] = S.gtab[q];
				double Jac[3][3], G[3][3], detJ;
				if constexpr (EL::AFFINE)
				{
					const double *geo = S.geo[g][el];
#pragma unroll
					for (int r = 0; r < 3; ++r)
#pragma unroll
						for (int c = 0; c < 3; ++c)
						{
							Jac[r][c] = geo[3 * r + c];
							G[r][c] = geo[9 + 3 * r + c];
						}
					detJ = geo[18];
				}
				else
				{
					const double(*gg)[3] = S.ggtab[q];
#pragma unroll
					for (int r = 0; r < 3; ++r)
#pragma unroll
						for (int c = 0; c < 3; ++c)
						{
							double s_ = 0.0;
#pragma unroll
							for (int j = 0; j < NG; ++j) s_ += gg[j][r] * S.X[g][el][j][c];
							Jac[r][c] = s_;
						}
					detJ = det3(Jac);
					double Jit[3][3];
					inv_transpose3(Jac, detJ, Jit);
#pragma unroll
					for (int r = 0; r < 3; ++r)
#pragma unroll
						for (int c = 0; c < 3; ++c) G[r][c] = Jit[r][0] * Jit[c][0] + Jit[r][1] * Jit[c][1] + Jit[r][2] * Jit[c][2];
				}
				double M[3][3];
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int c = 0; c < 3; ++c)
					{
						double s_ = Jac[c][r];
#pragma unroll
						for (int a = 0; a < N; ++a) s_ += S.U[g][el][a][r] * gq[a][c];
						M[r][c] = s_;
					}
				const double detM = det3(M);
				const double J = detM / detJ;
				const double lj = log(J);
				double Kt[3][3];
				inv_transpose3(M, detM, Kt);
				const double da = detJ * S.wq[q];
				const double2 lm = S.lame[g][el]; // (lambda, mu)
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int k = 0; k < 3; ++k)
					{
						rec[3 * r + k] = (float)Kt[r][k];
						rec[9 + 3 * r + k] = (float)G[r][k];
					}
				rec[18] = (float)(lm.y * da);
				rec[19] = (float)(lm.x * da);
				rec[20] = (float)((lm.y - lm.x * lj) * da);
				// J <= 0 (log J is NaN or -inf, as in the reference): the whole element
				// matrix must come out NaN.  The tensor cores do not carry a NaN operand
				// through a zero factor of Phi, so the epilogue writes the NaNs itself.
				rec[21] = (J > 0.0 && isfinite(lj)) ? 0.f : 1.f;
				rec[22] = rec[23] = 0.f;
			}
			named_arrive(BAR_FULL0 + buf, TC_THREADS);
		}
		// balance the consumers' arrivals on the buffers of the last two tiles
		for (int k = (it >= 2 ? it - 2 : 0); k < it; ++k) named_sync(BAR_EMPTY0 + (k & 1), TC_THREADS);
	}
	else
	{
		// ================= math group: A operand, MMA, write-out =================
		const int row = tid; // A row and TMEM lane
		// Only thread 0 waits on the mbarriers; it publishes the outcome in shared
		// memory before the next barrier of the group, so that all four warps take the
		// same branch around the warp-wide tcgen05.ld.
		if (tid == 0 && !mbar_wait(&S.bar_b, 0))
		{
			S.abort = 1;
			if (m.err) atomicExch(m.err, 1);
		}
		int it = 0;
		unsigned mma_phase = 0; // completed phases of bar_mma waited on so far (one per part of every tile)
		for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it)
		{
			const int buf = it & 1;
			const int e0 = t * TE, ne = min(TE, m.E - e0);
			named_sync(BAR_FULL0 + buf, TC_THREADS);
			bool bad = false; // the row's element has a point with J <= 0
#pragma unroll 1
			for (int h = 0; h < C::KH; ++h)
			{
				if (h == 0)
				{
					if (tid == 0) bulk_wait_read_all(); // the previous tile's store has left the A bytes
				}
				else if (tid == 0 && !S.abort)
				{
					// the previous part's MMAs must be done with A before it is rewritten
					if (!mbar_wait(&S.bar_mma, mma_phase & 1))
					{
						S.abort = 1;
						if (m.err) atomicExch(m.err, 1);
					}
				}
				if (h > 0) ++mma_phase;
				named_sync(BAR_MATH, 128);
				if (row < C::ROWS)
				{
					const int el = row / 9, rc = row % 9, r = rc / 3, c = rc % 3;
					float w[9][C::NQH];
#pragma unroll
					for (int qh = 0; qh < C::NQH; ++qh)
					{
						// the (element, point) record as six 16-byte loads; rows r and c of Kt
						// picked by selects (no indexed register access)
						float R[24];
						const float4 *R4 = reinterpret_cast<const float4 *>(S.kin[buf][el][h * C::NQH + qh]);
#pragma unroll
						for (int k = 0; k < 6; ++k)
						{
							const float4 x = R4[k];
							R[4 * k] = x.x;
							R[4 * k + 1] = x.y;
							R[4 * k + 2] = x.z;
							R[4 * k + 3] = x.w;
						}
						float kr[3], kc[3], g[9];
#pragma unroll
						for (int k = 0; k < 3; ++k)
						{
							kr[k] = r == 0 ? R[k] : (r == 1 ? R[3 + k] : R[6 + k]);
							kc[k] = c == 0 ? R[k] : (c == 1 ? R[3 + k] : R[6 + k]);
						}
#pragma unroll
						for (int k = 0; k < 9; ++k) g[k] = R[9 + k];
						const float dmu = (r == c) ? R[18] : 0.f, dl = R[19], dw = R[20];
						bad |= R[21] != 0.f;
#pragma unroll
						for (int k = 0; k < 3; ++k)
						{
							const float a1 = dl * kr[k], a2 = dw * kc[k];
#pragma unroll
							for (int l = 0; l < 3; ++l) w[3 * k + l][qh] = fmaf(a1, kc[l], fmaf(a2, kr[l], dmu * g[3 * k + l]));
						}
					}
#pragma unroll
					for (int kl = 0; kl < 9; ++kl)
					{
						float hh[4], ll[4];
#pragma unroll
						for (int i = 0; i < 4; ++i)
						{
							hh[i] = tf32_round(w[kl][i]);
							ll[i] = tf32_round(w[kl][i] - hh[i]);
						}
						*reinterpret_cast<float4 *>(S.Ah[kl][row]) = make_float4(hh[0], hh[1], hh[2], hh[3]);
						*reinterpret_cast<float4 *>(S.Al[kl][row]) = make_float4(ll[0], ll[1], ll[2], ll[3]);
					}
				}
				if (h == C::KH - 1) named_arrive(BAR_EMPTY0 + buf, TC_THREADS); // kin[buf] consumed
				fence_proxy_async_smem();
				named_sync(BAR_MATH, 128);
				if (tid == 0 && !S.abort)
				{
					tc_fence_after();
					const uint32_t idesc = idesc_tf32(128, C::NPAD);
					const uint32_t a_h = smem_u32(&S.Ah[0][0][0]), a_l = smem_u32(&S.Al[0][0][0]);
					const uint32_t b_h = smem_u32(&S.B[h][0][0][0][0]), b_l = smem_u32(&S.B[h][1][0][0][0]);
#pragma unroll 1
					for (int ks = 0; ks < C::KP / 8; ++ks)
					{
						const uint32_t ao = ks * 2 * C::A_CHUNK, bo = ks * 2 * C::B_CHUNK;
						const uint64_t dah = smem_desc(a_h + ao, C::A_CHUNK, 128), dal = smem_desc(a_l + ao, C::A_CHUNK, 128);
						const uint64_t dbh = smem_desc(b_h + bo, C::B_CHUNK, 128), dbl = smem_desc(b_l + bo, C::B_CHUNK, 128);
						mma_tf32(tmem, dal, dbh, idesc, (h > 0 || ks > 0) ? 1u : 0u);
						mma_tf32(tmem, dah, dbl, idesc, 1u);
						mma_tf32(tmem, dah, dbh, idesc, 1u);
					}
					mma_commit(&S.bar_mma);
				}
			}
			if (tid == 0 && !S.abort && !mbar_wait(&S.bar_mma, mma_phase & 1))
			{
				S.abort = 1;
				if (m.err) atomicExch(m.err, 1);
			}
			++mma_phase;
			tc_fence_before();
			named_sync(BAR_MATH, 128);
			tc_fence_after();
			const bool got = !S.abort;
			float v[C::NPAD];
			if (got)
			{
#pragma unroll
				for (int c0 = 0; c0 < C::NPAD; c0 += 32)
				{
					if (c0 + 32 <= C::NPAD)
					{
						float x[32];
						tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + c0, x);
#pragma unroll
						for (int i = 0; i < 32; ++i) v[c0 + i] = x[i];
					}
					else
					{
						float x[16];
						tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, x);
#pragma unroll
						for (int i = 0; i < 16; ++i) v[c0 + i] = x[i];
					}
				}
			}
			else
			{
#pragma unroll
				for (int i = 0; i < C::NPAD; ++i) v[i] = __int_as_float(0x7fc00000); // NaN: the result is invalid
			}
			if (bad)
			{
#pragma unroll
				for (int i = 0; i < C::NPAD; ++i) v[i] = __int_as_float(0x7fc00000);
			}
			if (row < 9 * ne)
			{
				const int el = row / 9, rc = row % 9, r = rc / 3, c = rc % 3;
				float *o = S.out + el * TP;
#pragma unroll
				for (int p = 0; p < C::NP; ++p) o[9 * p + 3 * c + r] = v[p];
				if (rc == 0)
					for (int k = 9 * C::NP; k < TP; ++k) o[k] = 0.f;
			}
			fence_proxy_async_smem();
			tc_fence_before();
			named_sync(BAR_MATH, 128);
			if (tid == 0 && ne > 0)
			{
				bulk_store(stage + (size_t)e0 * TP, S.out, (uint32_t)(ne * TP * sizeof(float)));
				bulk_commit();
			}
		}
		if (tid == 0) bulk_wait_all();
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (warp == 0) tmem_dealloc(tmem, C::TMEM_COLS);
}

template <class EL>
struct TcLaunch
{
	static int grid_limit(int device)
	{
		static int cached[64] = {};
		if (device < 0 || device >= 64) return 148;
		if (!cached[device])
		{
			// CTAs per SM from the kernel's own footprint: shared memory (plus the 1 KB
			// the runtime reserves per CTA) and registers
			int sms = 0, smem_sm = 0, regs_sm = 0;
			cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
			cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
			cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device);
			cudaFuncAttributes fa{};
			cudaFuncGetAttributes(&fa, k_hessian_blocks_tc<EL>);
			const int by_smem = smem_sm / (int)(sizeof(TcSmem<EL>) + 1024);
			const int by_regs = fa.numRegs > 0 ? regs_sm / (fa.numRegs * TC_THREADS) : 1;
			cached[device] = std::max(1, sms) * std::max(1, std::min(std::min(by_smem, by_regs), 4));
		}
		return cached[device];
	}
};

template <class EL>
cudaError_t tc_setup_one(float *symbol_dummy_unused)
{
	(void)symbol_dummy_unused;
	return cudaFuncSetAttribute(k_hessian_blocks_tc<EL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
								(int)sizeof(TcSmem<EL>));
}

} // namespace

cudaError_t tc_tables_setup(int)
{
	static const std::vector<float> p2 = build_phi<P2Tet>();
	static const std::vector<float> q1 = build_phi<Q1Hex>();
	cudaError_t e = cudaMemcpyToSymbol(g_phi_p2, p2.data(), p2.size() * sizeof(float));
	if (e != cudaSuccess) return e;
	e = cudaMemcpyToSymbol(g_phi_q1, q1.data(), q1.size() * sizeof(float));
	if (e != cudaSuccess) return e;
	e = tc_setup_one<P2Tet>(nullptr);
	if (e != cudaSuccess) return e;
	return tc_setup_one<Q1Hex>(nullptr);
}

cudaError_t launch_hessian_blocks_tc(const DevMesh &m, const double *u, float *stage, cudaStream_t s)
{
	if (m.E <= 0) return cudaSuccess;
	int dev = 0;
	cudaGetDevice(&dev);
	void *phi = nullptr;
	if (m.et == 2)
	{
		cudaError_t e = cudaGetSymbolAddress(&phi, g_phi_p2);
		if (e != cudaSuccess) return e;
		const int ntiles = (m.E + TcCfg<P2Tet>::TE - 1) / TcCfg<P2Tet>::TE;
		const int grid = std::min(ntiles, TcLaunch<P2Tet>::grid_limit(dev));
		k_hessian_blocks_tc<P2Tet><<<grid, TC_THREADS, sizeof(TcSmem<P2Tet>), s>>>(m, u, static_cast<const float *>(phi),
																					 stage, ntiles);
	}
	else if (m.et == 3)
	{
		cudaError_t e = cudaGetSymbolAddress(&phi, g_phi_q1);
		if (e != cudaSuccess) return e;
		const int ntiles = (m.E + TcCfg<Q1Hex>::TE - 1) / TcCfg<Q1Hex>::TE;
		const int grid = std::min(ntiles, TcLaunch<Q1Hex>::grid_limit(dev));
		k_hessian_blocks_tc<Q1Hex><<<grid, TC_THREADS, sizeof(TcSmem<Q1Hex>), s>>>(m, u, static_cast<const float *>(phi),
																					 stage, ntiles);
	}
	else
		return cudaErrorInvalidValue;
	return cudaGetLastError();
}

size_t tc_smem_bytes(int et)
{
	return et == 2 ? sizeof(TcSmem<P2Tet>) : et == 3 ? sizeof(TcSmem<Q1Hex>) : 0;
}

} // namespace pfg
