// One 4x4 block row of A x, shared by the SpMV kernels and the AMG residual.
//
// A warp owns one block row; lane l multiplies whole blocks l, l+32, ...
// (16 FP32 values in four 128-bit loads, or 16 FP64 values in eight), so a
// warp keeps 32 blocks of values in flight, and the column index of a lane's
// next block is loaded one step ahead so that the x gather does not wait on
// it.  The four row sums are then reduced across the warp (three butterfly
// levels on all four, two reduce-scatter levels) so that lane r ends with row
// r.  This replaces the reference's thread-per-row BlockSpmvKernel
// (solvers/cuda/include/SparseKernels.cuh:25-40), whose loads are strided.
#pragma once

#include "kernels.cuh"

namespace tfiga {

template <class T> struct BlockLoad;
template <> struct BlockLoad<double> {
	static __device__ __forceinline__ void Get(const double* values, long long b, double a[16])
	{
		const double2* p = reinterpret_cast<const double2*>(values+(size_t)b*16);
		#pragma unroll
		for (int k = 0; k < 8; ++k) { const double2 v = __ldg(p+k); a[2*k] = v.x; a[2*k+1] = v.y; }
	}
};
template <> struct BlockLoad<float> {
	static __device__ __forceinline__ void Get(const float* values, long long b, double a[16])
	{
		const float4* p = reinterpret_cast<const float4*>(values+(size_t)b*16);
		#pragma unroll
		for (int k = 0; k < 4; ++k) {
			const float4 v = __ldg(p+k);
			a[4*k] = v.x; a[4*k+1] = v.y; a[4*k+2] = v.z; a[4*k+3] = v.w;
		}
	}
};

// Returns (A x)[4*row + r] in lane r = 0..3 of the warp (lane l holds row l & 3).
template <class T>
__device__ __forceinline__ double RowBlockDot(const DevicePatternView& p, const T* __restrict__ values,
	const double* __restrict__ x, int row, int lane)
{
	double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
	const int hi = p.row_offsets[row+1];
	int b = p.row_offsets[row]+lane;
	int col = b < hi ? p.columns[b] : 0;
	while (b < hi) {
		const int next = b+32;
		const int next_col = next < hi ? p.columns[next] : 0;
		double a[16];
		BlockLoad<T>::Get(values, b, a);
		const double2* xv = reinterpret_cast<const double2*>(x+4*(size_t)col);
		const double2 x01 = __ldg(xv), x23 = __ldg(xv+1);
		s0 = fma(a[0], x01.x, s0); s0 = fma(a[1], x01.y, s0); s0 = fma(a[2], x23.x, s0); s0 = fma(a[3], x23.y, s0);
		s1 = fma(a[4], x01.x, s1); s1 = fma(a[5], x01.y, s1); s1 = fma(a[6], x23.x, s1); s1 = fma(a[7], x23.y, s1);
		s2 = fma(a[8], x01.x, s2); s2 = fma(a[9], x01.y, s2); s2 = fma(a[10], x23.x, s2); s2 = fma(a[11], x23.y, s2);
		s3 = fma(a[12], x01.x, s3); s3 = fma(a[13], x01.y, s3); s3 = fma(a[14], x23.x, s3); s3 = fma(a[15], x23.y, s3);
		b = next;
		col = next_col;
	}
	#pragma unroll
	for (int o = 16; o >= 4; o >>= 1) {
		s0 += __shfl_xor_sync(0xffffffffu, s0, o);
		s1 += __shfl_xor_sync(0xffffffffu, s1, o);
		s2 += __shfl_xor_sync(0xffffffffu, s2, o);
		s3 += __shfl_xor_sync(0xffffffffu, s3, o);
	}
	const bool upper = (lane & 2) != 0;            // keeps rows 2, 3
	double k0 = upper ? s2 : s0, k1 = upper ? s3 : s1;
	const double g0 = upper ? s0 : s2, g1 = upper ? s1 : s3;
	k0 += __shfl_xor_sync(0xffffffffu, g0, 2);
	k1 += __shfl_xor_sync(0xffffffffu, g1, 2);
	const bool odd = (lane & 1) != 0;              // keeps rows 1, 3
	double keep = odd ? k1 : k0;
	const double give = odd ? k0 : k1;
	keep += __shfl_xor_sync(0xffffffffu, give, 1);
	return keep;
}

} // namespace tfiga
