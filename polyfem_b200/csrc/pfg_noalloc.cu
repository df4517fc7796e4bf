// pfg_energy_noalloc: the NeoHookean total energy for callers that cannot
// allocate device memory.
//
// Some hosts embed the assembly inside code that must not call cudaMalloc:
// a solver running inside a memory pool it does not own, a plugin whose
// allocations are forbidden after start-up, or a caller that pre-plans every
// byte of device memory.  This entry point takes every array from the caller
// (already on the device) and keeps the energy kernel's reduction scratch in a
// fixed-size array that lives in the library's own device image, so the call
// allocates nothing: no cudaMalloc, no cudaFree, no allocating library routine.
//
// Limits and rules (also in include/pfgpu.h):
//  * at most PFG_NOALLOC_MAX_BLOCKS thread blocks of the energy kernel
//    (energy_elems_per_block: 256 elements), i.e. n_elements <= 256 *
//    PFG_NOALLOC_MAX_BLOCKS; larger meshes are rejected;
//  * the scratch array (512 KiB of partial sums plus two counters) is held by
//    every GPU that loads the library until the process exits;
//  * all calls share that one array: calls that overlap on the GPU (different
//    streams, or several host threads) race and give wrong results;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current); make that first call
//    before any stream capture.
#include "../../include/pfgpu.h"
#include "pfg_internal.h"

#include <cstdint>
#include <mutex>
#include <string>

namespace
{

// file-scope device scratch: per-block partial sums, the last-block ticket and
// the inverted-element counter
struct NoallocScratch
{
	double partials[PFG_NOALLOC_MAX_BLOCKS];
	unsigned int ticket;
	unsigned int pad;
	unsigned long long inverted;
};
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
NoallocScratch *g_noalloc_ptr[kMaxDevices] = {};

// the message is readable through pfg_last_error(NULL)
int noalloc_fail(int status, const std::string &msg)
{
	pfg::set_global_error(msg);
	return status;
}

// Device address of the scratch array for `device`, looked up once per device
// with that device current.  cudaGetSymbolAddress allocates nothing.
int noalloc_scratch(int device, NoallocScratch **out)
{
	std::lock_guard<std::mutex> lock(g_noalloc_mutex);
	if (!g_noalloc_ptr[device])
	{
		int prev = -1;
		cudaGetDevice(&prev);
		if (prev != device && cudaSetDevice(device) != cudaSuccess)
			return noalloc_fail(PFG_ERR_CUDA, "cudaSetDevice failed");
		void *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (prev >= 0 && prev != device) cudaSetDevice(prev);
		if (e != cudaSuccess || !p)
			return noalloc_fail(PFG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
		g_noalloc_ptr[device] = static_cast<NoallocScratch *>(p);
	}
	*out = g_noalloc_ptr[device];
	return PFG_OK;
}
} // namespace

extern "C" int pfg_energy_noalloc(int elem_type, int n_elements, int n_nodes, int n_geom_nodes, const int *conn_soa,
								  const int *gconn_soa, const double *X, const double *lame, const double *u, int prec,
								  double *out, void *stream)
{
	if (elem_type != PFG_P1_TET && elem_type != PFG_P2_TET && elem_type != PFG_Q1_HEX)
		return noalloc_fail(PFG_ERR_INVALID, "unknown elem_type");
	if (prec != PFG_FP64 && prec != PFG_FP32 && prec != PFG_SPLIT32) return noalloc_fail(PFG_ERR_INVALID, "bad precision");
	if (n_elements < 0 || n_nodes < 0 || n_geom_nodes < 0) return noalloc_fail(PFG_ERR_INVALID, "negative size");
	if (!out) return noalloc_fail(PFG_ERR_INVALID, "out is NULL");
	if (n_elements > 0 && (!conn_soa || !X || !lame || !u)) return noalloc_fail(PFG_ERR_INVALID, "NULL input array");
	if (elem_type == PFG_P2_TET && n_elements > 0 && !gconn_soa)
		return noalloc_fail(PFG_ERR_INVALID, "gconn_soa is required for P2 elements");
	// the size limits pfg_create applies to the same inputs
	if ((long long)n_nodes * 3 > 0x7fffffffLL) return noalloc_fail(PFG_ERR_UNSUPPORTED, "too many nodes (3 * n_nodes > 2^31-1)");
	if ((long long)n_geom_nodes * 3 > 0x7fffffffLL)
		return noalloc_fail(PFG_ERR_UNSUPPORTED, "too many geometric nodes (3 * n_geom_nodes > 2^31-1)");
	const int n_per = elem_type == PFG_P1_TET ? 4 : (elem_type == PFG_P2_TET ? 10 : 8);
	if ((long long)n_elements * n_per > 0x7fffffffLL) return noalloc_fail(PFG_ERR_UNSUPPORTED, "E * n exceeds 2^31-1");
	// The caller owns these pointers, so nothing guarantees the alignment the kernel's
	// loads assume: (lambda, mu) is read as one 16-byte pair per element, the other
	// arrays element by element.  A misaligned pointer would fault on the device and
	// lose the CUDA context, so it is refused here, before any CUDA call.
	auto misaligned = [](const void *p, unsigned a) { return p && (reinterpret_cast<uintptr_t>(p) & (a - 1)) != 0; };
	if (misaligned(lame, 16)) return noalloc_fail(PFG_ERR_INVALID, "lame must be 16-byte aligned ((lambda, mu) pairs are read as one 16-byte load)");
	if (misaligned(u, 8) || misaligned(X, 8) || misaligned(out, 8))
		return noalloc_fail(PFG_ERR_INVALID, "u, X and out must be 8-byte aligned");
	if (misaligned(conn_soa, 4) || misaligned(gconn_soa, 4))
		return noalloc_fail(PFG_ERR_INVALID, "conn_soa and gconn_soa must be 4-byte aligned");
	const long long per_block = pfg::energy_elems_per_block(elem_type);
	const long long blocks = ((long long)n_elements + per_block - 1) / per_block;
	if (blocks > PFG_NOALLOC_MAX_BLOCKS)
		return noalloc_fail(PFG_ERR_UNSUPPORTED, "n_elements = " + std::to_string(n_elements) + " exceeds the limit of " +
													 std::to_string((long long)PFG_NOALLOC_MAX_BLOCKS * per_block) +
													 " elements of pfg_energy_noalloc for this element type");
	int device = -1;
	cudaError_t ce = cudaGetDevice(&device);
	if (ce != cudaSuccess || device < 0 || device >= kMaxDevices)
		return noalloc_fail(PFG_ERR_CUDA, std::string("no current CUDA device: ") + cudaGetErrorString(ce));
	NoallocScratch *s = nullptr;
	int st = noalloc_scratch(device, &s);
	if (st != PFG_OK) return st;

	cudaStream_t cs = static_cast<cudaStream_t>(stream);
	// the ticket and the inverted counter must start at zero
	ce = cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned int) * 2 + sizeof(unsigned long long), cs);
	if (ce != cudaSuccess) return noalloc_fail(PFG_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(ce));

	pfg::DevMesh m;
	m.et = elem_type;
	m.E = n_elements;
	m.N = n_nodes;
	m.Ng = n_geom_nodes;
	m.conn = conn_soa;
	m.gconn = (elem_type == PFG_P2_TET) ? gconn_soa : (gconn_soa ? gconn_soa : conn_soa);
	m.X = X;
	m.lame = reinterpret_cast<const double2 *>(lame);
	pfg::Scratch sc;
	sc.partials = s->partials;
	sc.ticket = &s->ticket;
	sc.inverted = &s->inverted;
	sc.max_blocks = PFG_NOALLOC_MAX_BLOCKS;
	ce = pfg::launch_energy(m, u, prec, false, out, sc, cs);
	if (ce != cudaSuccess) return noalloc_fail(PFG_ERR_CUDA, std::string("energy kernel: ") + cudaGetErrorString(ce));
	return PFG_OK;
}
