// Internal declarations shared by the host API (pfg_api.cu) and the kernel
// launchers (pfg_kernels.cu, pfg_tc.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace pfg
{

// Device-resident mesh in the layout the kernels read.
//  conn  : [n][E] int32 (structure of arrays: local node a of all elements is contiguous)
//  gconn : [n_g][E] int32 (aliases conn for isoparametric elements)
//  X     : [N_g][3] float64 rest positions
//  lame  : [E] (lambda, mu) float64 pairs
struct DevMesh
{
	int et = 0, E = 0, N = 0, Ng = 0;
	const int *conn = nullptr;
	const int *gconn = nullptr;
	const double *X = nullptr;
	const double2 *lame = nullptr;
};

// Device-resident Hessian pattern.
//  outer/inner : CSC arrays (3N+1 / nnz)
//  slot        : [E][n*n] int32, CSC index of entry (3A, 3B) for the node pair
//                (A = conn[e][a], B = conn[e][b]); entry (3A+m, 3B+c) is at
//                slot + c*colstride[B] + m
//  colstride   : [N] int32, 3*deg(B) = length of each of node B's three columns
struct DevPattern
{
	long long nnz = 0;
	const int *outer = nullptr;
	const int *inner = nullptr;
	const int *slot = nullptr;
	const int *colstride = nullptr;
	double *values = nullptr;
};

struct Scratch
{
	double *partials = nullptr;       // per-block energy partial sums
	unsigned int *ticket = nullptr;   // last-block-done counter (returns to 0 after each launch)
	unsigned long long *inverted = nullptr;
	int max_blocks = 0;
};

constexpr int PREC_FP64 = 0;
constexpr int PREC_FP32 = 1;
constexpr int PREC_SPLIT32 = 2;

// All launchers return cudaGetLastError() after enqueueing on `s`.
cudaError_t launch_energy(const DevMesh &m, const double *u, int prec, bool per_element, double *out,
						  const Scratch &sc, cudaStream_t s);
cudaError_t launch_gradient(const DevMesh &m, const double *u, int prec, double *g, const Scratch &sc,
							cudaStream_t s);
cudaError_t launch_hessian(const DevMesh &m, const DevPattern &p, const double *u, int prec, cudaStream_t s);
cudaError_t launch_material_vjp(const DevMesh &m, const double *u, const double *adj, double *out, cudaStream_t s);
cudaError_t launch_shape_vjp(const DevMesh &m, const double *u, const double *adj, int prec, double *out,
							 cudaStream_t s);
cudaError_t hessian_kernel_setup(int device);

// Sets the message pfg_last_error(NULL) returns on this host thread.
void set_global_error(const std::string &msg);

} // namespace pfg
