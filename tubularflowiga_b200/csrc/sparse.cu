// Block-CSR (4x4) kernels: SpMV (optionally fused with the block-Jacobi
// apply), diagonal-block inverse, Dirichlet rows, boundary-face flows and
// tractions, and deterministic two-stage reductions.
//
// SpMV layout: one warp per block row (block_row.cuh).
#include "block_row.cuh"
#include "common.hpp"
#include "kernels.cuh"

namespace tfiga {
namespace {

constexpr int kReduceBlocks = 296;   // 2 CTAs per SM for the partial-sum stage

template <class T>
__global__ void __launch_bounds__(256) SpmvKernel(DevicePatternView p, const T* __restrict__ values,
	const double* __restrict__ x, double* __restrict__ y)
{
	const int row = blockIdx.x*8+(threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (row >= p.nodes) return;
	const double sum = RowBlockDot(p, values, x, row, lane);
	if (lane < 4) y[4*(size_t)row+lane] = sum;
}

template <class T>
__global__ void __launch_bounds__(256) SpmvBlockJacobiKernel(DevicePatternView p, const T* __restrict__ values,
	const double* __restrict__ inverse, const double* __restrict__ x, const double* __restrict__ scale,
	double* __restrict__ y, const int* __restrict__ stop)
{
	if (stop != nullptr && *stop) return;
	const int row = blockIdx.x*8+(threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (row >= p.nodes) return;
	double sum = RowBlockDot(p, values, x, row, lane);
	if (scale != nullptr) sum *= *scale;
	if (inverse == nullptr) {
		if (lane < 4) y[4*(size_t)row+lane] = sum;
		return;
	}
	const double y0 = __shfl_sync(0xffffffffu, sum, 0), y1 = __shfl_sync(0xffffffffu, sum, 1);
	const double y2 = __shfl_sync(0xffffffffu, sum, 2), y3 = __shfl_sync(0xffffffffu, sum, 3);
	if (lane < 4) {
		const double* d = inverse+(size_t)row*16+lane*4;
		y[4*(size_t)row+lane] = d[0]*y0+d[1]*y1+d[2]*y2+d[3]*y3;
	}
}

// Gauss-Jordan with partial pivoting and the singular fallback of
// BuildBlockInverseKernel (SparseKernels.cuh:42-89), for F x F diagonal blocks.
template <int F, class T>
__global__ void BlockInverseKernel(DevicePatternView p, const T* __restrict__ values,
	double* __restrict__ inverse, unsigned int* __restrict__ singular)
{
	const int node = blockIdx.x*blockDim.x+threadIdx.x;
	if (node >= p.nodes) return;
	const T* s = values+(size_t)p.diagonal[node]*F*F;
	double m[F][2*F];
	for (int i = 0; i < F; ++i)
		for (int j = 0; j < 2*F; ++j) m[i][j] = j < F ? s[i*F+j] : (j-F == i ? 1.0 : 0.0);
	bool failed = false;
	for (int pivot = 0; pivot < F; ++pivot) {
		int best = pivot;
		for (int r = pivot+1; r < F; ++r)
			if (fabs(m[r][pivot]) > fabs(m[best][pivot])) best = r;
		if (!isfinite(m[best][pivot]) || fabs(m[best][pivot]) < 1e-14) { failed = true; break; }
		if (best != pivot)
			for (int c = 0; c < 2*F; ++c) { const double t = m[pivot][c]; m[pivot][c] = m[best][c]; m[best][c] = t; }
		const double sc = 1.0/m[pivot][pivot];
		for (int c = 0; c < 2*F; ++c) m[pivot][c] *= sc;
		for (int r = 0; r < F; ++r) {
			if (r == pivot) continue;
			const double factor = m[r][pivot];
			for (int c = 0; c < 2*F; ++c) m[r][c] -= factor*m[pivot][c];
		}
	}
	double* d = inverse+(size_t)node*F*F;
	if (!failed) {
		for (int i = 0; i < F; ++i) for (int j = 0; j < F; ++j) d[i*F+j] = m[i][F+j];
	} else {
		atomicAdd(singular, 1u);
		for (int i = 0; i < F; ++i)
			for (int j = 0; j < F; ++j)
				d[i*F+j] = i == j && fabs(s[i*F+i]) > 1e-14 ? 1.0/s[i*F+i] : (i == j ? 1.0 : 0.0);
	}
}

template <int F>
__global__ void ApplyBlockInverseKernel(int nodes, const double* __restrict__ inverse, const double* __restrict__ x,
	double* __restrict__ y)
{
	const long long i = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (i >= (long long)F*nodes) return;
	const long long node = i/F;
	const int r = (int)(i-node*F);
	const double* d = inverse+node*F*F+r*F;
	const double* v = x+F*node;
	double s = d[0]*v[0];
	#pragma unroll
	for (int c = 1; c < F; ++c) s += d[c]*v[c];
	y[i] = s;
}

// state = prescribed value on every constrained entry (thread per constrained node).
__global__ void LiftDirichletKernel(int count, const int32_t* __restrict__ nodes, const int32_t* __restrict__ vmask,
	const int32_t* __restrict__ pmask, const double* __restrict__ velocity, const double* __restrict__ pressure,
	double* __restrict__ state)
{
	const int item = blockIdx.x*blockDim.x+threadIdx.x;
	if (item >= count) return;
	const size_t node = (size_t)nodes[item];
	if (vmask[node]) for (int d = 0; d < 3; ++d) state[4*node+d] = velocity[3*node+d];
	if (pmask[node]) state[4*node+3] = pressure[node];
}

// Dirichlet rows (IgaCudaKernels.cuh:436-463): a warp per constrained node.
template <class T>
__global__ void DirichletRowsKernel(DevicePatternView p, int count, const int32_t* __restrict__ nodes,
	const int32_t* __restrict__ vmask, const int32_t* __restrict__ pmask, const double* __restrict__ velocity,
	const double* __restrict__ pressure, const double* __restrict__ state, T* __restrict__ values,
	double* __restrict__ rhs)
{
	const int item = blockIdx.x*(blockDim.x >> 5)+(threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (item >= count) return;
	const int node = nodes[item];
	const bool cv = vmask[node] != 0, cp = pmask[node] != 0;
	if (values != nullptr) {
		const int lo = p.row_offsets[node], hi = p.row_offsets[node+1];
		for (int b = lo+lane; b < hi; b += 32) {
			T* blk = values+(size_t)b*16;
			if (cv) for (int k = 0; k < 12; ++k) blk[k] = T(0);
			if (cp) for (int k = 12; k < 16; ++k) blk[k] = T(0);
		}
		__syncwarp();
		if (lane == 0) {
			T* diag = values+(size_t)p.diagonal[node]*16;
			if (cv) { diag[0] = T(1); diag[5] = T(1); diag[10] = T(1); }
			if (cp) diag[15] = T(1);
		}
	}
	if (rhs != nullptr && lane < 4) {
		const bool c = lane < 3 ? cv : cp;
		if (c) {
			const double target = lane < 3 ? velocity[3*(size_t)node+lane] : pressure[node];
			rhs[4*(size_t)node+lane] = target-state[4*(size_t)node+lane];
		}
	}
}

// Outward flow of each boundary face: sum_a F[a].u_a (BoundaryFlow.hpp:165-200).
__global__ void __launch_bounds__(64) FaceFlowKernel(int faces, const int32_t* __restrict__ face_element,
	const double* __restrict__ coef, int stride, const int32_t* __restrict__ eo, const int32_t* __restrict__ conn,
	const double* __restrict__ state, double* __restrict__ out)
{
	const int face = blockIdx.x;
	const int e = face_element[face];
	const int begin = eo[e], nen = eo[e+1]-begin;
	double v = 0.0;
	for (int a = threadIdx.x; a < nen; a += 64) {
		const size_t node = (size_t)conn[begin+a];
		const double* F = coef+((size_t)face*stride+a)*3;
		v += F[0]*state[4*node]+F[1]*state[4*node+1]+F[2]*state[4*node+2];
	}
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	__shared__ double part[2];
	if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
	__syncthreads();
	if (threadIdx.x == 0) out[face] = part[0]+part[1];
}

// traction[4 node + c] -= p_face F[a][c] (IntegratePressureTractionForces, PressureTractionFlow.hpp:41-64).
__global__ void __launch_bounds__(64) FaceTractionKernel(int faces, const int32_t* __restrict__ face_element,
	const double* __restrict__ coef, int stride, const int32_t* __restrict__ eo, const int32_t* __restrict__ conn,
	const double* __restrict__ face_pressure, double* __restrict__ traction)
{
	const int face = blockIdx.x;
	const double pressure = face_pressure[face];
	if (pressure == 0.0) return;
	const int e = face_element[face];
	const int begin = eo[e], nen = eo[e+1]-begin;
	for (int a = threadIdx.x; a < nen; a += 64) {
		const size_t node = (size_t)conn[begin+a];
		const double* F = coef+((size_t)face*stride+a)*3;
		for (int c = 0; c < 3; ++c) atomicAdd(traction+4*node+c, -pressure*F[c]);
	}
}

__device__ __forceinline__ double BlockSum(double v, double* shared)
{
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (lane == 0) shared[warp] = v;
	__syncthreads();
	v = 0.0;
	if (warp == 0) {
		const int warps = blockDim.x >> 5;
		v = lane < warps ? shared[lane] : 0.0;
		for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	}
	__syncthreads();
	return v;
}

__global__ void __launch_bounds__(256) StridedPartialKernel(long long count, int stride, int offset,
	const double* __restrict__ x, double* __restrict__ partial)
{
	__shared__ double shared[8];
	double sq = 0.0, sum = 0.0;
	for (long long i = (long long)blockIdx.x*blockDim.x+threadIdx.x; i < count; i += (long long)gridDim.x*blockDim.x) {
		const double v = x[i*stride+offset];
		sq = fma(v, v, sq);
		sum += v;
	}
	sq = BlockSum(sq, shared);
	sum = BlockSum(sum, shared);
	if (threadIdx.x == 0) { partial[2*blockIdx.x] = sq; partial[2*blockIdx.x+1] = sum; }
}

__global__ void __launch_bounds__(256) FinalizeSumsKernel(int blocks, const double* __restrict__ partial,
	double* __restrict__ out, int take_sqrt)
{
	__shared__ double shared[8];
	double sq = 0.0, sum = 0.0;
	for (int i = threadIdx.x; i < blocks; i += blockDim.x) { sq += partial[2*i]; sum += partial[2*i+1]; }
	sq = BlockSum(sq, shared);
	sum = BlockSum(sum, shared);
	if (threadIdx.x == 0) { out[0] = take_sqrt ? sqrt(sq) : sq; out[1] = sum; }
}

__global__ void AxpyKernel(long long n, double alpha, const double* __restrict__ x, double* __restrict__ y)
{
	const long long i = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (i < n) y[i] = fma(alpha, x[i], y[i]);
}

__global__ void __launch_bounds__(256) SegmentSumKernel(const int32_t* __restrict__ segment_of, int items,
	const double* __restrict__ values, double* __restrict__ out)
{
	__shared__ double shared[8];
	const int seg = blockIdx.x;
	double v = 0.0;
	for (int i = threadIdx.x; i < items; i += blockDim.x)
		if (segment_of[i] == seg) v += values[i];
	v = BlockSum(v, shared);
	if (threadIdx.x == 0) out[seg] = v;
}

unsigned Blocks(long long n, int threads) { return (unsigned)((n+threads-1)/threads); }

__global__ void ToFloatKernel(long long n, const double* __restrict__ in, float* __restrict__ out)
{
	const long long i = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (i < n) out[i] = (float)in[i];
}

} // namespace

// out[k] = sum of x[i]^2 over [offsets[k], offsets[k+1]) -- one CTA per segment, fixed order.
__global__ void __launch_bounds__(256) SegmentSquaresKernel(const int64_t* __restrict__ offsets,
	const double* __restrict__ x, double* __restrict__ out)
{
	__shared__ double shared[8];
	const int64_t lo = offsets[blockIdx.x], hi = offsets[blockIdx.x+1];
	double sq = 0.0;
	for (long long i = lo+threadIdx.x; i < hi; i += blockDim.x) sq += x[i]*x[i];
	sq = BlockSum(sq, shared);
	if (threadIdx.x == 0) out[blockIdx.x] = sq;
}

// x[i] *= scale[k] over segment k's entries (scale 0 clears the segment).
__global__ void ScaleSegmentsKernel(int segments, const int64_t* __restrict__ offsets,
	const double* __restrict__ scale, double* __restrict__ x)
{
	const int k = blockIdx.y;
	if (k >= segments) return;
	const double s = scale[k];
	if (s == 1.0) return;
	const int64_t lo = offsets[k], hi = offsets[k+1];
	for (long long i = lo+(long long)blockIdx.x*blockDim.x+threadIdx.x; i < hi; i += (long long)gridDim.x*blockDim.x)
		x[i] = s == 0.0 ? 0.0 : s*x[i];
}

int PartialSlots() { return 2*kReduceBlocks; }

template <class T>
void LaunchSpmv(const DevicePatternView& p, const T* values, const double* x, double* y, cudaStream_t stream)
{
	if (p.nodes == 0) return;
	SpmvKernel<T><<<Blocks(p.nodes, 8), 256, 0, stream>>>(p, values, x, y);
	LaunchCheck("SpmvKernel");
}

// y = A x on the block rows of segments still open (node_seg[row] the row's segment, seg_stop[s] set
// once segment s has stopped: its rows are skipped and y there is left as it was).
template <class T>
__global__ void __launch_bounds__(256) SpmvMaskedKernel(DevicePatternView p, const T* __restrict__ values,
	const double* __restrict__ x, double* __restrict__ y, const int* __restrict__ stop,
	const int32_t* __restrict__ node_seg, const int* __restrict__ seg_stop)
{
	if (*stop) return;
	const int row = blockIdx.x*8+(threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (row >= p.nodes || seg_stop[node_seg[row]]) return;
	const double sum = RowBlockDot(p, values, x, row, lane);
	if (lane < 4) y[4*(size_t)row+lane] = sum;
}

template <class T>
void LaunchSpmvMasked(const DevicePatternView& p, const T* values, const double* x, double* y, const int* stop,
	const int32_t* node_seg, const int* seg_stop, cudaStream_t stream)
{
	if (p.nodes == 0) return;
	SpmvMaskedKernel<T><<<Blocks(p.nodes, 8), 256, 0, stream>>>(p, values, x, y, stop, node_seg, seg_stop);
	LaunchCheck("SpmvMaskedKernel");
}

template <class T>
void LaunchSpmvBlockJacobi(const DevicePatternView& p, const T* values, const double* inverse,
	const double* x, const double* scale, double* y, const int* stop, cudaStream_t stream)
{
	if (p.nodes == 0) return;
	SpmvBlockJacobiKernel<T><<<Blocks(p.nodes, 8), 256, 0, stream>>>(p, values, inverse, x, scale, y, stop);
	LaunchCheck("SpmvBlockJacobiKernel");
}

template <class T>
void LaunchBlockInverse(const DevicePatternView& p, const T* values, double* inverse, unsigned int* singular,
	cudaStream_t stream)
{
	if (p.nodes == 0) return;
	BlockInverseKernel<4, T><<<Blocks(p.nodes, 128), 128, 0, stream>>>(p, values, inverse, singular);
	LaunchCheck("BlockInverseKernel");
}

template void LaunchSpmv<double>(const DevicePatternView&, const double*, const double*, double*, cudaStream_t);
template void LaunchSpmv<float>(const DevicePatternView&, const float*, const double*, double*, cudaStream_t);
template void LaunchSpmvBlockJacobi<double>(const DevicePatternView&, const double*, const double*, const double*,
	const double*, double*, const int*, cudaStream_t);
template void LaunchSpmvMasked<double>(const DevicePatternView&, const double*, const double*, double*, const int*,
	const int32_t*, const int*, cudaStream_t);
template void LaunchSpmvMasked<float>(const DevicePatternView&, const float*, const double*, double*, const int*,
	const int32_t*, const int*, cudaStream_t);
template void LaunchSpmvBlockJacobi<float>(const DevicePatternView&, const float*, const double*, const double*,
	const double*, double*, const int*, cudaStream_t);
template void LaunchBlockInverse<double>(const DevicePatternView&, const double*, double*, unsigned int*, cudaStream_t);
template void LaunchBlockInverse<float>(const DevicePatternView&, const float*, double*, unsigned int*, cudaStream_t);

namespace {

// One thread per (table, point pair, function): two FP64 reads 64 apart, one 8-byte store.
__global__ void ToFloatPointPairsKernel(long long pairs, const double* __restrict__ in, float* __restrict__ out)
{
	const long long i = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (i >= pairs) return;
	const long long table = i >> 11, rest = i & 2047;          // 32 pairs x 64 functions per table
	const int pair = (int)(rest >> 6), b = (int)(rest & 63);
	const double* t = in+table*4096;
	reinterpret_cast<float2*>(out)[i] = make_float2((float)t[(2*pair)*64+b], (float)t[(2*pair+1)*64+b]);
}

} // namespace

void LaunchToFloatPointPairs(long long tables, const double* in, float* out, cudaStream_t stream)
{
	if (tables == 0) return;
	const long long pairs = tables*2048;
	ToFloatPointPairsKernel<<<Blocks(pairs, 256), 256, 0, stream>>>(pairs, in, out);
	LaunchCheck("ToFloatPointPairsKernel");
}

void LaunchToFloat(long long n, const double* in, float* out, cudaStream_t stream)
{
	if (n == 0) return;
	ToFloatKernel<<<Blocks(n, 256), 256, 0, stream>>>(n, in, out);
	LaunchCheck("ToFloatKernel");
}

void LaunchApplyBlockInverse(int nodes, const double* inverse, const double* x, double* y, cudaStream_t stream)
{
	if (nodes == 0) return;
	ApplyBlockInverseKernel<4><<<Blocks(4LL*nodes, 256), 256, 0, stream>>>(nodes, inverse, x, y);
	LaunchCheck("ApplyBlockInverseKernel");
}

void LaunchBlockInverse2(const DevicePatternView& p, const double* values, double* inverse, unsigned int* singular,
	cudaStream_t stream)
{
	if (p.nodes == 0) return;
	BlockInverseKernel<2, double><<<Blocks(p.nodes, 128), 128, 0, stream>>>(p, values, inverse, singular);
	LaunchCheck("BlockInverseKernel<2>");
}

void LaunchApplyBlockInverse2(int nodes, const double* inverse, const double* x, double* y, cudaStream_t stream)
{
	if (nodes == 0) return;
	ApplyBlockInverseKernel<2><<<Blocks(2LL*nodes, 256), 256, 0, stream>>>(nodes, inverse, x, y);
	LaunchCheck("ApplyBlockInverseKernel<2>");
}

template <class T>
void LaunchDirichletRows(const DevicePatternView& p, int count, const int32_t* nodes, const int32_t* vmask,
	const int32_t* pmask, const double* velocity, const double* pressure, const double* state, T* values,
	double* rhs, cudaStream_t stream)
{
	if (count == 0) return;
	DirichletRowsKernel<T><<<Blocks(count, 8), 256, 0, stream>>>(p, count, nodes, vmask, pmask, velocity, pressure,
		state, values, rhs);
	LaunchCheck("DirichletRowsKernel");
}

template void LaunchDirichletRows<double>(const DevicePatternView&, int, const int32_t*, const int32_t*,
	const int32_t*, const double*, const double*, const double*, double*, double*, cudaStream_t);
template void LaunchDirichletRows<float>(const DevicePatternView&, int, const int32_t*, const int32_t*,
	const int32_t*, const double*, const double*, const double*, float*, double*, cudaStream_t);

void LaunchLiftDirichlet(int count, const int32_t* nodes, const int32_t* vmask, const int32_t* pmask,
	const double* velocity, const double* pressure, double* state, cudaStream_t stream)
{
	if (count == 0) return;
	LiftDirichletKernel<<<(unsigned)((count+255)/256), 256, 0, stream>>>(count, nodes, vmask, pmask, velocity,
		pressure, state);
	LaunchCheck("LiftDirichletKernel");
}

void LaunchFaceFlows(int faces, const int32_t* face_element, const double* face_coef, int stride, const int32_t* eo,
	const int32_t* conn, const double* state, double* face_flow, cudaStream_t stream)
{
	if (faces == 0) return;
	FaceFlowKernel<<<faces, 64, 0, stream>>>(faces, face_element, face_coef, stride, eo, conn, state, face_flow);
	LaunchCheck("FaceFlowKernel");
}

void LaunchFaceTraction(int faces, const int32_t* face_element, const double* face_coef, int stride,
	const int32_t* eo, const int32_t* conn, const double* face_pressure, double* traction, cudaStream_t stream)
{
	if (faces == 0) return;
	FaceTractionKernel<<<faces, 64, 0, stream>>>(faces, face_element, face_coef, stride, eo, conn, face_pressure,
		traction);
	LaunchCheck("FaceTractionKernel");
}

void LaunchStridedSums(long long count, int stride, int offset, const double* x, double* partial, double* out,
	cudaStream_t stream)
{
	StridedPartialKernel<<<kReduceBlocks, 256, 0, stream>>>(count, stride, offset, x, partial);
	LaunchCheck("StridedPartialKernel");
	FinalizeSumsKernel<<<1, 256, 0, stream>>>(kReduceBlocks, partial, out, 0);
	LaunchCheck("FinalizeSumsKernel");
}

void LaunchNorm(long long n, const double* x, double* partial, double* out, cudaStream_t stream)
{
	StridedPartialKernel<<<kReduceBlocks, 256, 0, stream>>>(n, 1, 0, x, partial);
	LaunchCheck("StridedPartialKernel");
	FinalizeSumsKernel<<<1, 256, 0, stream>>>(kReduceBlocks, partial, out, 1);
	LaunchCheck("FinalizeSumsKernel");
}

void LaunchSegmentSquares(int segments, const int64_t* offsets, const double* x, double* out, cudaStream_t stream)
{
	if (segments == 0) return;
	SegmentSquaresKernel<<<segments, 256, 0, stream>>>(offsets, x, out);
	LaunchCheck("SegmentSquaresKernel");
}

void LaunchScaleSegments(int segments, const int64_t* offsets, const double* scale, double* x, cudaStream_t stream)
{
	if (segments == 0) return;
	ScaleSegmentsKernel<<<dim3(16, segments), 256, 0, stream>>>(segments, offsets, scale, x);
	LaunchCheck("ScaleSegmentsKernel");
}

void LaunchAxpy(long long n, double alpha, const double* x, double* y, cudaStream_t stream)
{
	if (n == 0) return;
	AxpyKernel<<<Blocks(n, 256), 256, 0, stream>>>(n, alpha, x, y);
	LaunchCheck("AxpyKernel");
}

void LaunchSegmentSums(int segments, const int32_t* segment_of, int items, const double* values, double* out,
	cudaStream_t stream)
{
	if (segments == 0) return;
	SegmentSumKernel<<<segments, 256, 0, stream>>>(segment_of, items, values, out);
	LaunchCheck("SegmentSumKernel");
}

} // namespace tfiga
