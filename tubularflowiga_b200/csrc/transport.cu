// Two-species transport (N0 attached, N+ advected by a prescribed velocity):
// the kernels of the reference's `iga_cuda transport` command
// (solvers/cuda/src/iga_cuda.cu:621-732).
//
// Assembly (AssembleTransportKernel, IgaCudaKernels.cuh:155-237) runs once per
// transport run.  The reference gives every CTA a tile of basis pairs and
// re-evaluates the basis, the interpolated velocity and tau at every Gauss
// point in every tile.  Here one CTA owns an element: the basis tables built
// once per mesh (phi, qdata) are staged in shared memory eight Gauss points at
// a time, one warp per point forms u, tau and the SUPG test function
// T_a = N_a + tau u.grad N_a, and each thread then accumulates sixteen (a, b)
// pairs in registers over all 64 points.  The six reference sums reduce to
// four independent ones,
//   M = sum w N_a N_b,  S = sum w grad N_a.grad N_b,  P = sum w T_a N_b,
//   X = sum w T_a (dt u.grad N_b + dt v+ ad grad N_a.grad N_b),
// from which the 2x2 blocks follow in the epilogue:
//   L00 = (1 + dt (k+ + k-)) M + dt D S,  L0+ = -k'+ dt M,
//   L+0 = -k+ dt P,  L++ = (1 + dt k'+) P + X,  P00 = M,  P++ = P.
// The pair -> block map is the per-mesh element_blocks table (no search).
//
// SpMV (BlockSpmvKernel<2>, SparseKernels.cuh:25-40): one warp per block row,
// lane l multiplies blocks l, l + 32, ... (32 bytes of FP64 values each, two
// 16-byte loads; or 16 bytes of FP32 values, one load), so a warp streams up
// to 1 KB of the matrix per step.
#include "common.hpp"
#include "kernels.cuh"
#include "transport.hpp"

namespace tfiga {
namespace {

constexpr int kPointsPerPass = 8;   // Gauss points staged per shared-memory pass (one warp each)
constexpr int kPairsPerThread = 16; // (a, b) pairs per thread: a = t / 4, b = t % 4 + 4 j

__global__ void __launch_bounds__(256, 1) TransportAssemblyKernel(DeviceMeshView mesh,
	const double* __restrict__ phi, const double* __restrict__ qdata, const int32_t* __restrict__ element_blocks,
	const double* __restrict__ velocity, TransportCoefficients c, double* __restrict__ left,
	double* __restrict__ previous)
{
	__shared__ double sN[kPointsPerPass][kMaxBasis];
	__shared__ double sG[3][kPointsPerPass][kMaxBasis];
	__shared__ double sT[kPointsPerPass][kMaxBasis];
	__shared__ double sA[kPointsPerPass][kMaxBasis];
	__shared__ double sW[kPointsPerPass];
	__shared__ double sVel[kMaxBasis][3];

	const int e = blockIdx.x;
	const int tid = threadIdx.x;
	const int warp = tid >> 5, lane = tid & 31;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	for (int i = tid; i < kMaxBasis*3; i += blockDim.x) {
		const int a = i/3, d = i-3*a;
		sVel[a][d] = a < nen ? velocity[3*(size_t)mesh.connectivity[begin+a]+d] : 0.0;
	}

	const int a = tid >> 2, bset = tid & 3;
	double M[kPairsPerThread], S[kPairsPerThread], P[kPairsPerThread], X[kPairsPerThread];
	#pragma unroll
	for (int j = 0; j < kPairsPerThread; ++j) { M[j] = 0.0; S[j] = 0.0; P[j] = 0.0; X[j] = 0.0; }
	const double cad = c.dt*c.vplus*c.artificial_diffusion;

	for (int q0 = 0; q0 < kQuad; q0 += kPointsPerPass) {
		__syncthreads();   // previous pass done with the tiles (and sVel written on the first)
		// Stage N and grad N of the pass's points: phi[((e*5 + t)*64 + q)*64 + a].
		for (int i = tid; i < 4*kPointsPerPass*kMaxBasis; i += blockDim.x) {
			const int b = i % kMaxBasis, q = (i/kMaxBasis) % kPointsPerPass, t = i/(kMaxBasis*kPointsPerPass);
			const double v = phi[(((size_t)e*kFeatures+t)*kQuad+q0+q)*kMaxBasis+b];
			if (t == 0) sN[q][b] = v;
			else sG[t-1][q][b] = v;
		}
		if (tid < kPointsPerPass) sW[tid] = qdata[((size_t)e*kQuad+q0+tid)*kQData];
		__syncthreads();
		{
			// Warp `warp` owns point q0 + warp: interpolated velocity, tau, T_a and u.grad N_a
			// (IgaCudaKernels.cuh:189-205, TransportElement.hpp:222-233).
			const int q = warp;
			double u[3];
			#pragma unroll
			for (int d = 0; d < 3; ++d) {
				double s = sN[q][lane]*sVel[lane][d]+sN[q][lane+32]*sVel[lane+32][d];
				#pragma unroll
				for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
				u[d] = s;
			}
			const double adv0 = u[0]*sG[0][q][lane]+u[1]*sG[1][q][lane]+u[2]*sG[2][q][lane];
			const double adv1 = u[0]*sG[0][q][lane+32]+u[1]*sG[1][q][lane+32]+u[2]*sG[2][q][lane+32];
			double inverse_length = fabs(adv0)+fabs(adv1);
			#pragma unroll
			for (int o = 16; o > 0; o >>= 1) inverse_length += __shfl_xor_sync(0xffffffffu, inverse_length, o);
			const double tau_space = inverse_length > 0.0 ? 1.0/inverse_length : 0.0;
			const double tau_time = c.dt/2.0;
			const double tau = tau_space > 0.0
				? 1.0/sqrt(1.0/(tau_space*tau_space)+1.0/(tau_time*tau_time)) : 0.0;
			sA[q][lane] = adv0;
			sA[q][lane+32] = adv1;
			sT[q][lane] = sN[q][lane]+tau*adv0;
			sT[q][lane+32] = sN[q][lane+32]+tau*adv1;
		}
		__syncthreads();
		#pragma unroll 1
		for (int q = 0; q < kPointsPerPass; ++q) {
			const double w = sW[q];
			const double wN = w*sN[q][a], wT = w*sT[q][a];
			const double ga0 = sG[0][q][a], ga1 = sG[1][q][a], ga2 = sG[2][q][a];
			#pragma unroll
			for (int j = 0; j < kPairsPerThread; ++j) {
				const int b = bset+4*j;
				const double Nb = sN[q][b];
				const double gg = ga0*sG[0][q][b]+ga1*sG[1][q][b]+ga2*sG[2][q][b];
				M[j] = fma(wN, Nb, M[j]);
				S[j] = fma(w, gg, S[j]);
				P[j] = fma(wT, Nb, P[j]);
				X[j] = fma(wT, c.dt*sA[q][b]+cad*gg, X[j]);
			}
		}
	}

	const double l00_mass = 1.0+c.dt*(c.kplus+c.kminus), l0p_mass = -c.detach_plus*c.dt;
	const double lp0_p = -c.kplus*c.dt, lpp_p = 1.0+c.dt*c.detach_plus, l00_s = c.dt*c.diffusion;
	const int32_t* blocks = element_blocks+(size_t)e*kMaxBasis*kMaxBasis+a*kMaxBasis;
	#pragma unroll
	for (int j = 0; j < kPairsPerThread; ++j) {
		const int block = blocks[bset+4*j];
		if (block < 0) continue;
		double* l = left+(size_t)block*4;
		double* p = previous+(size_t)block*4;
		atomicAdd(l, l00_mass*M[j]+l00_s*S[j]);
		atomicAdd(l+1, l0p_mass*M[j]);
		atomicAdd(l+2, lp0_p*P[j]);
		atomicAdd(l+3, lpp_p*P[j]+X[j]);
		atomicAdd(p, M[j]);
		atomicAdd(p+3, P[j]);
	}
}

// Elements with 65..80 basis functions, from their 80-wide tables: CTA per element, 256 threads.  A warp
// per point forms the interpolated velocity, tau and the point weight; then one task per (a, eight
// consecutive b) sums M, S, P and X over the 64 points (T_a and u.grad N formed on the fly) and adds
// the same 2x2 blocks as TransportAssemblyKernel.
constexpr int kLargeGroup = 8;

__global__ void __launch_bounds__(256) TransportAssemblyLargeKernel(DeviceMeshView mesh, int first,
	const double* __restrict__ phi, const double* __restrict__ qdata, const int32_t* __restrict__ element_blocks,
	const double* __restrict__ velocity, TransportCoefficients c, double* __restrict__ left,
	double* __restrict__ previous)
{
	constexpr int NP = kMaxBasisLarge;
	__shared__ double sVel[NP][3];
	__shared__ double sU[kQuad][3];
	__shared__ double sTau[kQuad], sW[kQuad];
	const int e = first+blockIdx.x;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	const double* P = phi+(size_t)(e-first)*kFeatures*kQuad*NP;
	for (int i = tid; i < NP*3; i += blockDim.x) {
		const int a = i/3, d = i-3*a;
		sVel[a][d] = a < nen ? velocity[3*(size_t)mesh.connectivity[begin+a]+d] : 0.0;
	}
	__syncthreads();
	for (int q = warp; q < kQuad; q += 8) {
		double u[3] = {0.0, 0.0, 0.0};
		for (int a = lane; a < NP; a += 32)
			for (int d = 0; d < 3; ++d) u[d] += P[(0*kQuad+q)*NP+a]*sVel[a][d];
		for (int d = 0; d < 3; ++d)
			for (int o = 16; o > 0; o >>= 1) u[d] += __shfl_xor_sync(0xffffffffu, u[d], o);
		double inverse_length = 0.0;
		for (int a = lane; a < NP; a += 32)
			inverse_length += fabs(u[0]*P[(1*kQuad+q)*NP+a]+u[1]*P[(2*kQuad+q)*NP+a]+u[2]*P[(3*kQuad+q)*NP+a]);
		for (int o = 16; o > 0; o >>= 1) inverse_length += __shfl_xor_sync(0xffffffffu, inverse_length, o);
		if (lane == 0) {
			const double tau_space = inverse_length > 0.0 ? 1.0/inverse_length : 0.0;
			const double tau_time = c.dt/2.0;
			sTau[q] = tau_space > 0.0 ? 1.0/sqrt(1.0/(tau_space*tau_space)+1.0/(tau_time*tau_time)) : 0.0;
			sW[q] = qdata[((size_t)e*kQuad+q)*kQData];
			for (int d = 0; d < 3; ++d) sU[q][d] = u[d];
		}
	}
	__syncthreads();
	const double cad = c.dt*c.vplus*c.artificial_diffusion;
	const double l00_mass = 1.0+c.dt*(c.kplus+c.kminus), l0p_mass = -c.detach_plus*c.dt;
	const double lp0_p = -c.kplus*c.dt, lpp_p = 1.0+c.dt*c.detach_plus, l00_s = c.dt*c.diffusion;
	const int32_t* EB = element_blocks+(size_t)(e-first)*NP*NP;
	constexpr int kGroups = NP/kLargeGroup;
	for (int task = tid; task < NP*kGroups; task += blockDim.x) {
		const int a = task/kGroups, b0 = (task%kGroups)*kLargeGroup;
		if (a >= nen || b0 >= nen) continue;
		double M[kLargeGroup], S[kLargeGroup], Pp[kLargeGroup], X[kLargeGroup];
		#pragma unroll
		for (int j = 0; j < kLargeGroup; ++j) { M[j] = 0.0; S[j] = 0.0; Pp[j] = 0.0; X[j] = 0.0; }
		for (int q = 0; q < kQuad; ++q) {
			const double w = sW[q], u0 = sU[q][0], u1 = sU[q][1], u2 = sU[q][2];
			const double na = P[(0*kQuad+q)*NP+a];
			const double ga0 = P[(1*kQuad+q)*NP+a], ga1 = P[(2*kQuad+q)*NP+a], ga2 = P[(3*kQuad+q)*NP+a];
			const double ta = na+sTau[q]*(u0*ga0+u1*ga1+u2*ga2);
			const double wN = w*na, wT = w*ta;
			#pragma unroll
			for (int j = 0; j < kLargeGroup; ++j) {
				const int b = b0+j;
				const double nb = P[(0*kQuad+q)*NP+b];
				const double gb0 = P[(1*kQuad+q)*NP+b], gb1 = P[(2*kQuad+q)*NP+b], gb2 = P[(3*kQuad+q)*NP+b];
				const double gg = ga0*gb0+ga1*gb1+ga2*gb2;
				M[j] = fma(wN, nb, M[j]);
				S[j] = fma(w, gg, S[j]);
				Pp[j] = fma(wT, nb, Pp[j]);
				X[j] = fma(wT, c.dt*(u0*gb0+u1*gb1+u2*gb2)+cad*gg, X[j]);
			}
		}
		#pragma unroll
		for (int j = 0; j < kLargeGroup; ++j) {
			const int b = b0+j;
			if (b >= nen) break;
			const int block = EB[a*NP+b];
			if (block < 0) continue;
			double* l = left+(size_t)block*4;
			double* p = previous+(size_t)block*4;
			atomicAdd(l, l00_mass*M[j]+l00_s*S[j]);
			atomicAdd(l+1, l0p_mass*M[j]);
			atomicAdd(l+2, lp0_p*Pp[j]);
			atomicAdd(l+3, lpp_p*Pp[j]+X[j]);
			atomicAdd(p, M[j]);
			atomicAdd(p+3, Pp[j]);
		}
	}
}

// Constrained rows (ApplyTransportBoundaryKernel, IgaCudaKernels.cuh:411-424): zero in both
// matrices, identity diagonal block in `left`.  A warp per constrained node.
__global__ void TransportBoundaryRowsKernel(DevicePatternView p, int count, const int32_t* __restrict__ nodes,
	double* __restrict__ left, double* __restrict__ previous)
{
	const int item = blockIdx.x*(blockDim.x >> 5)+(threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (item >= count) return;
	const int node = nodes[item];
	const long long lo = 4LL*p.row_offsets[node], hi = 4LL*p.row_offsets[node+1];
	for (long long k = lo+lane; k < hi; k += 32) { left[k] = 0.0; previous[k] = 0.0; }
	__syncwarp();
	if (lane == 0) {
		double* d = left+4LL*p.diagonal[node];
		d[0] = 1.0;
		d[3] = 1.0;
	}
}

// vector[2 node + (0, 1)] = (n0, n+) on constrained nodes (SetTransportBoundaryVectorKernel,
// IgaCudaKernels.cuh:426-434); a thread per constrained node.
__global__ void TransportBoundaryValuesKernel(int count, const int32_t* __restrict__ nodes,
	const double* __restrict__ n0, const double* __restrict__ nplus, double* __restrict__ vector)
{
	const int item = blockIdx.x*blockDim.x+threadIdx.x;
	if (item >= count) return;
	const size_t node = (size_t)nodes[item];
	vector[2*node] = n0[node];
	vector[2*node+1] = nplus[node];
}

// One 2x2 block (row-major) as doubles: two 16-byte loads (FP64) or one (FP32).
template <class T> struct Block2;
template <> struct Block2<double> {
	static __device__ __forceinline__ void Get(const double* values, int b, double a[4])
	{
		const double2* v = reinterpret_cast<const double2*>(values+4*(size_t)b);
		const double2 r0 = __ldg(v), r1 = __ldg(v+1);
		a[0] = r0.x; a[1] = r0.y; a[2] = r1.x; a[3] = r1.y;
	}
};
template <> struct Block2<float> {
	static __device__ __forceinline__ void Get(const float* values, int b, double a[4])
	{
		const float4 v = __ldg(reinterpret_cast<const float4*>(values+4*(size_t)b));
		a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
	}
};

// Returns (A x)[2 row + (lane & 1)] in every lane.
template <class T>
__device__ __forceinline__ double RowBlockDot2(const DevicePatternView& p, const T* __restrict__ values,
	const double* __restrict__ x, int row, int lane)
{
	double s0 = 0.0, s1 = 0.0;
	const int hi = p.row_offsets[row+1];
	int b = p.row_offsets[row]+lane;
	int col = b < hi ? p.columns[b] : 0;
	while (b < hi) {
		const int next = b+32;
		const int next_col = next < hi ? p.columns[next] : 0;
		double a[4];
		Block2<T>::Get(values, b, a);
		const double2 xv = __ldg(reinterpret_cast<const double2*>(x+2*(size_t)col));
		s0 = fma(a[0], xv.x, s0); s0 = fma(a[1], xv.y, s0);
		s1 = fma(a[2], xv.x, s1); s1 = fma(a[3], xv.y, s1);
		b = next;
		col = next_col;
	}
	#pragma unroll
	for (int o = 16; o >= 2; o >>= 1) {
		s0 += __shfl_xor_sync(0xffffffffu, s0, o);
		s1 += __shfl_xor_sync(0xffffffffu, s1, o);
	}
	const bool odd = (lane & 1) != 0;
	double keep = odd ? s1 : s0;
	const double give = odd ? s0 : s1;
	keep += __shfl_xor_sync(0xffffffffu, give, 1);
	return keep;
}

__global__ void __launch_bounds__(256) Spmv2Kernel(DevicePatternView p, const double* __restrict__ values,
	const double* __restrict__ x, double* __restrict__ y)
{
	const int row = blockIdx.x*8+(threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (row >= p.nodes) return;
	const double sum = RowBlockDot2(p, values, x, row, lane);
	if (lane < 2) y[2*(size_t)row+lane] = sum;
}

template <class T>
__global__ void __launch_bounds__(256) SpmvBlockJacobi2Kernel(DevicePatternView p, const T* __restrict__ values,
	const double* __restrict__ inverse, const double* __restrict__ x, const double* __restrict__ scale,
	double* __restrict__ y, const int* __restrict__ stop)
{
	if (stop != nullptr && *stop) return;
	const int row = blockIdx.x*8+(threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (row >= p.nodes) return;
	double sum = RowBlockDot2(p, values, x, row, lane);
	if (scale != nullptr) sum *= *scale;
	if (inverse == nullptr) {
		if (lane < 2) y[2*(size_t)row+lane] = sum;
		return;
	}
	const double y0 = __shfl_sync(0xffffffffu, sum, 0), y1 = __shfl_sync(0xffffffffu, sum, 1);
	if (lane < 2) {
		const double* d = inverse+(size_t)row*4+lane*2;
		y[2*(size_t)row+lane] = d[0]*y0+d[1]*y1;
	}
}

// Flow-line preconditioner apply: thread per line, forward substitution with the unit lower band,
// backward substitution with the upper band and the inverted diagonal blocks; the forward result
// is kept in y at the line's nodes (every node is on exactly one line).
__global__ void __launch_bounds__(128) LineApplyKernel(LinePreconditionerView v, const double* __restrict__ x,
	double* __restrict__ y, const int* __restrict__ stop)
{
	if (stop != nullptr && *stop) return;
	const int l = blockIdx.x*blockDim.x+threadIdx.x;
	if (l >= v.lines) return;
	const int lo = v.line_offsets[l], m = v.line_offsets[l+1]-lo, w = v.band_width[l], s = 2*w+1;
	const double* B = v.factors+v.band_offsets[l];
	const int32_t* nodes = v.line_nodes+lo;
	for (int p = 0; p < m; ++p) {
		const size_t i = 2*(size_t)nodes[p];
		double v0 = x[i], v1 = x[i+1];
		for (int q = p-w > 0 ? p-w : 0; q < p; ++q) {
			const double* L = B+4*((size_t)p*s+(q-p+w));
			const size_t j = 2*(size_t)nodes[q];
			const double y0 = y[j], y1 = y[j+1];
			v0 -= L[0]*y0+L[1]*y1;
			v1 -= L[2]*y0+L[3]*y1;
		}
		y[i] = v0;
		y[i+1] = v1;
	}
	for (int p = m-1; p >= 0; --p) {
		const size_t i = 2*(size_t)nodes[p];
		double v0 = y[i], v1 = y[i+1];
		for (int q = p+1; q <= p+w && q < m; ++q) {
			const double* U = B+4*((size_t)p*s+(q-p+w));
			const size_t j = 2*(size_t)nodes[q];
			const double x0 = y[j], x1 = y[j+1];
			v0 -= U[0]*x0+U[1]*x1;
			v1 -= U[2]*x0+U[3]*x1;
		}
		const double* D = B+4*((size_t)p*s+w);
		y[i] = D[0]*v0+D[1]*v1;
		y[i+1] = D[2]*v0+D[3]*v1;
	}
}

unsigned Grid(long long n, int per_block) { return (unsigned)((n+per_block-1)/per_block); }

} // namespace

void LaunchTransportAssembly(const DeviceMeshView& mesh, const double* phi, const double* qdata,
	const int32_t* element_blocks, const double* velocity, const TransportCoefficients& coefficients, double* left,
	double* previous, cudaStream_t stream)
{
	if (mesh.elements == 0) return;
	TransportAssemblyKernel<<<mesh.elements, 256, 0, stream>>>(mesh, phi, qdata, element_blocks, velocity,
		coefficients, left, previous);
	LaunchCheck("TransportAssemblyKernel");
}

void LaunchTransportAssemblyLarge(const DeviceMeshView& mesh, int first, int count, const double* phi,
	const double* qdata, const int32_t* element_blocks, const double* velocity,
	const TransportCoefficients& coefficients, double* left, double* previous, cudaStream_t stream)
{
	if (count == 0) return;
	TransportAssemblyLargeKernel<<<count, 256, 0, stream>>>(mesh, first, phi, qdata, element_blocks, velocity,
		coefficients, left, previous);
	LaunchCheck("TransportAssemblyLargeKernel");
}

void LaunchTransportBoundaryRows(const DevicePatternView& pattern, int count, const int32_t* nodes, double* left,
	double* previous, cudaStream_t stream)
{
	if (count == 0) return;
	TransportBoundaryRowsKernel<<<Grid(count, 8), 256, 0, stream>>>(pattern, count, nodes, left, previous);
	LaunchCheck("TransportBoundaryRowsKernel");
}

void LaunchTransportBoundaryValues(int count, const int32_t* nodes, const double* n0, const double* nplus,
	double* vector, cudaStream_t stream)
{
	if (count == 0) return;
	TransportBoundaryValuesKernel<<<Grid(count, 256), 256, 0, stream>>>(count, nodes, n0, nplus, vector);
	LaunchCheck("TransportBoundaryValuesKernel");
}

void LaunchSpmv2(const DevicePatternView& p, const double* values, const double* x, double* y, cudaStream_t stream)
{
	if (p.nodes == 0) return;
	Spmv2Kernel<<<Grid(p.nodes, 8), 256, 0, stream>>>(p, values, x, y);
	LaunchCheck("Spmv2Kernel");
}

template <class T>
void LaunchSpmvBlockJacobi2(const DevicePatternView& p, const T* values, const double* inverse,
	const double* x, const double* scale, double* y, const int* stop, cudaStream_t stream)
{
	if (p.nodes == 0) return;
	SpmvBlockJacobi2Kernel<T><<<Grid(p.nodes, 8), 256, 0, stream>>>(p, values, inverse, x, scale, y, stop);
	LaunchCheck("SpmvBlockJacobi2Kernel");
}

void LaunchLineApply(const LinePreconditionerView& view, const double* x, double* y, const int* stop,
	cudaStream_t stream)
{
	if (view.lines == 0) return;
	LineApplyKernel<<<Grid(view.lines, 128), 128, 0, stream>>>(view, x, y, stop);
	LaunchCheck("LineApplyKernel");
}

template void LaunchSpmvBlockJacobi2<double>(const DevicePatternView&, const double*, const double*, const double*,
	const double*, double*, const int*, cudaStream_t);
template void LaunchSpmvBlockJacobi2<float>(const DevicePatternView&, const float*, const double*, const double*,
	const double*, double*, const int*, cudaStream_t);

} // namespace tfiga
