// Device kernels and host driver of the block-Jacobi GMRES (see gmres.hpp).
#include "gmres.hpp"

#include <algorithm>
#include <cmath>
#include <type_traits>

namespace tfiga {
namespace {

constexpr int kBlocks = 592;          // 4 CTAs per SM for the streaming passes
constexpr int kThreads = 256;
constexpr int kWarps = kThreads/32;
constexpr int kBatch = 8;             // Arnoldi steps launched per host wait

// Two consecutive basis entries as doubles (the basis is FP64, or FP32 in the
// reduced-precision modes).
template <class B> struct BasisPair;
template <> struct BasisPair<double> {
	static __device__ __forceinline__ double2 Load(const double* p, long long k2)
	{
		return reinterpret_cast<const double2*>(p)[k2];
	}
	static __device__ __forceinline__ void Store(double* p, long long k2, double2 v)
	{
		reinterpret_cast<double2*>(p)[k2] = v;
	}
};
template <> struct BasisPair<float> {
	static __device__ __forceinline__ double2 Load(const float* p, long long k2)
	{
		const float2 v = reinterpret_cast<const float2*>(p)[k2];
		return make_double2(v.x, v.y);
	}
	static __device__ __forceinline__ void Store(float* p, long long k2, double2 v)
	{
		reinterpret_cast<float2*>(p)[k2] = make_float2((float)v.x, (float)v.y);
	}
};

// partial[i*blocks + cta] = scale[i] * <V_i, w> over this CTA's chunk.  The
// chunk is a multiple of 128 doubles and n is even, so every row slice is
// 16-byte aligned: a warp streams two basis vectors at once with 16-byte
// loads, two steps per iteration, to keep enough bytes in flight for HBM.
template <class B>
__global__ void __launch_bounds__(kThreads) MultiDotKernel(const B* __restrict__ V, long long n,
	const double* __restrict__ scale, int count, const double* __restrict__ w, double* __restrict__ partial,
	int chunk, const int* __restrict__ stop)
{
	if (*stop) return;
	extern __shared__ double wchunk[];
	double2* w2 = reinterpret_cast<double2*>(wchunk);
	const long long lo = (long long)blockIdx.x*chunk;
	const long long rest = n-lo;
	const int len2 = (rest <= 0 ? 0 : (rest < chunk ? (int)rest : chunk)) >> 1;
	const double2* win = reinterpret_cast<const double2*>(w+lo);
	for (int k = threadIdx.x; k < len2; k += blockDim.x) w2[k] = win[k];
	__syncthreads();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const double2 zero = make_double2(0.0, 0.0);
	for (int i0 = warp; i0 < count; i0 += 2*kWarps) {
		const int i1 = i0+kWarps;
		const bool two = i1 < count;
		const B* a = V+(size_t)i0*n+lo;
		const B* b = V+(size_t)(two ? i1 : i0)*n+lo;
		double sa = 0.0, sb = 0.0, ta = 0.0, tb = 0.0;
		for (int k = lane; k < len2; k += 64) {
			const bool more = k+32 < len2;
			const double2 x0 = BasisPair<B>::Load(a, k), y0 = BasisPair<B>::Load(b, k);
			const double2 x1 = more ? BasisPair<B>::Load(a, k+32) : zero;
			const double2 y1 = more ? BasisPair<B>::Load(b, k+32) : zero;
			const double2 w0 = w2[k], w1 = more ? w2[k+32] : zero;
			sa = fma(x0.x, w0.x, sa); sa = fma(x0.y, w0.y, sa);
			sb = fma(y0.x, w0.x, sb); sb = fma(y0.y, w0.y, sb);
			ta = fma(x1.x, w1.x, ta); ta = fma(x1.y, w1.y, ta);
			tb = fma(y1.x, w1.x, tb); tb = fma(y1.y, w1.y, tb);
		}
		double u = sa+ta, v = sb+tb;
		for (int o = 16; o > 0; o >>= 1) {
			u += __shfl_xor_sync(0xffffffffu, u, o);
			v += __shfl_xor_sync(0xffffffffu, v, o);
		}
		if (lane == 0) {
			partial[(size_t)i0*gridDim.x+blockIdx.x] = u*scale[i0];
			if (two) partial[(size_t)i1*gridDim.x+blockIdx.x] = v*scale[i1];
		}
	}
}

// hpass[i] = sum over CTAs; H[i][j] = (pass == 0 ? hpass : H + hpass).
__global__ void __launch_bounds__(kThreads) DotFinalizeKernel(const double* __restrict__ partial, int blocks,
	int count, double* __restrict__ hpass, double* __restrict__ H, int restart, int j, int pass,
	const int* __restrict__ stop)
{
	if (*stop) return;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int i = blockIdx.x*(kThreads/32)+warp;   // a warp per basis vector, spread over CTAs
	if (i < count) {
		double s = 0.0;
		for (int b = lane; b < blocks; b += 32) s += partial[(size_t)i*blocks+b];
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) {
			hpass[i] = s;
			double& h = H[(size_t)i*restart+j];
			h = pass == 0 ? s : h+s;
		}
	}
}

// out = w - sum_i scale_i hpass_i V_i; norm_partial[cta] = sum out^2 (if non-null).
// out may alias w.  One CTA per tile of 32 entry pairs: its 8 warps split the
// basis (a contiguous slice each, four vectors per step) so that many
// independent loads are in flight, and warp 0 adds the 8 slice sums to w in
// a fixed order.
template <class B, class O>
__global__ void __launch_bounds__(kThreads) UpdateKernel(const B* __restrict__ V, long long n,
	const double* __restrict__ scale, int count, const double* __restrict__ hpass, const double* win, O* out,
	double* __restrict__ norm_partial, const int* __restrict__ stop)
{
	if (*stop) return;
	extern __shared__ double coef[];
	__shared__ double2 part[kWarps][32];
	for (int i = threadIdx.x; i < count; i += blockDim.x) coef[i] = scale[i]*hpass[i];
	__syncthreads();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long n2 = n >> 1;
	const long long k = (long long)blockIdx.x*32+lane;
	const int per = (count+kWarps-1)/kWarps;
	const int lo = warp*per, hi = min(count, lo+per);
	double2 acc = make_double2(0.0, 0.0);
	if (k < n2) {
		int i = lo;
		for (; i+3 < hi; i += 4) {
			const double2 a0 = BasisPair<B>::Load(V+(size_t)i*n, k), a1 = BasisPair<B>::Load(V+(size_t)(i+1)*n, k);
			const double2 a2 = BasisPair<B>::Load(V+(size_t)(i+2)*n, k), a3 = BasisPair<B>::Load(V+(size_t)(i+3)*n, k);
			acc.x = fma(-coef[i], a0.x, acc.x); acc.y = fma(-coef[i], a0.y, acc.y);
			acc.x = fma(-coef[i+1], a1.x, acc.x); acc.y = fma(-coef[i+1], a1.y, acc.y);
			acc.x = fma(-coef[i+2], a2.x, acc.x); acc.y = fma(-coef[i+2], a2.y, acc.y);
			acc.x = fma(-coef[i+3], a3.x, acc.x); acc.y = fma(-coef[i+3], a3.y, acc.y);
		}
		for (; i < hi; ++i) {
			const double2 a0 = BasisPair<B>::Load(V+(size_t)i*n, k);
			acc.x = fma(-coef[i], a0.x, acc.x); acc.y = fma(-coef[i], a0.y, acc.y);
		}
	}
	part[warp][lane] = acc;
	__syncthreads();
	if (warp != 0) return;
	double sq = 0.0;
	if (k < n2) {
		double2 v = reinterpret_cast<const double2*>(win)[k];
		#pragma unroll
		for (int w = 0; w < kWarps; ++w) { v.x += part[w][lane].x; v.y += part[w][lane].y; }
		BasisPair<O>::Store(out, k, v);
		sq = fma(v.x, v.x, v.y*v.y);
	}
	if (norm_partial == nullptr) return;
	for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
	if (lane == 0) norm_partial[blockIdx.x] = sq;
}

// Classical Gram-Schmidt twice, first pass's update and second pass's dots in one sweep over the
// basis: this CTA's chunk of every basis vector is staged in shared memory once (cp.async), then
// w <- w - sum_i scale_i hpass_i V_i on the chunk and partial[i*blocks + cta] = scale_i <V_i, w> on
// the updated chunk.  The chunk is a multiple of 32 entries and n a multiple of 4, so every slice is
// 16-byte aligned; the basis is read once where the separate passes read it twice.
template <class B>
__global__ void __launch_bounds__(kThreads) UpdateDotKernel(const B* __restrict__ V, long long n,
	const double* __restrict__ scale, int count, const double* __restrict__ hpass, double* __restrict__ w,
	double* __restrict__ partial, int chunk, const int* __restrict__ stop)
{
	if (*stop) return;
	extern __shared__ __align__(16) double fused[];
	double* coef = fused;                                        // [count], padded to an even length
	double* ws = coef+((count+1) & ~1);                          // [chunk] updated w
	B* Vs = reinterpret_cast<B*>(ws+chunk);                      // [count][chunk]
	const long long lo = (long long)blockIdx.x*chunk;
	const int len = (int)min((long long)chunk, n-lo);
	constexpr int kPer = 16/(int)sizeof(B);                      // entries per 16-byte copy
	const int units = len/kPer;
	for (int idx = threadIdx.x; idx < count*units; idx += blockDim.x) {
		const int i = idx/units, u = idx-i*units;
		const uint32_t dst = (uint32_t)__cvta_generic_to_shared(Vs+(size_t)i*chunk+u*kPer);
		asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(V+(size_t)i*n+lo+u*kPer)
			: "memory");
	}
	asm volatile("cp.async.commit_group;" ::: "memory");
	for (int i = threadIdx.x; i < count; i += blockDim.x) coef[i] = scale[i]*hpass[i];
	asm volatile("cp.async.wait_group 0;" ::: "memory");
	__syncthreads();
	for (int k = threadIdx.x; k < len; k += blockDim.x) {
		double acc = 0.0;
		for (int i = 0; i < count; ++i) acc = fma(-coef[i], (double)Vs[(size_t)i*chunk+k], acc);
		const double v = w[lo+k]+acc;
		w[lo+k] = v;
		ws[k] = v;
	}
	__syncthreads();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	for (int i = warp; i < count; i += kWarps) {
		const B* vi = Vs+(size_t)i*chunk;
		double sum = 0.0;
		for (int k = lane; k < len; k += 32) sum = fma((double)vi[k], ws[k], sum);
		for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
		if (lane == 0) partial[(size_t)i*gridDim.x+blockIdx.x] = sum*scale[i];
	}
}

// y += sum_k coef_k (g_k . x) g_k over sparse g_k; one CTA per outlet k (the dot in a fixed order;
// the scatter by atomic adds, as two outlets' vectors may share unknowns).
__global__ void __launch_bounds__(kThreads) LowRankKernel(const int* __restrict__ ptr,
	const int* __restrict__ idx, const double* __restrict__ val, const double* __restrict__ coef,
	const double* __restrict__ x, double* __restrict__ y, const int* __restrict__ stop)
{
	if (stop && *stop) return;
	__shared__ double part[kWarps];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int k = blockIdx.x;
	const int lo = ptr[k], hi = ptr[k+1];
	double s = 0.0;
	for (int j = lo+threadIdx.x; j < hi; j += blockDim.x) s = fma(val[j], x[idx[j]], s);
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	if (lane == 0) part[warp] = s;
	__syncthreads();
	double dot = 0.0;
	#pragma unroll
	for (int w = 0; w < kWarps; ++w) dot += part[w];
	const double scale = coef[k]*dot;
	for (int j = lo+threadIdx.x; j < hi; j += blockDim.x) atomicAdd(y+idx[j], scale*val[j]);
}

// Column j of the Hessenberg matrix: norm, previous rotations, new rotation,
// residual estimate (Gmres.hpp:272-305).  One warp stages the column and the
// rotations in shared memory; lane 0 then applies the rotations sequentially.
__global__ void ArnoldiFinalizeKernel(const double* __restrict__ norm_partial, int blocks, double* __restrict__ H,
	int restart, int j, double* __restrict__ cs, double* __restrict__ sn, double* __restrict__ g,
	double* __restrict__ scale, int* __restrict__ state, double* __restrict__ residual, double tolerance)
{
	extern __shared__ double sh[];
	double* col = sh;                 // [restart+1]
	double* c = col+restart+1;        // [restart]
	double* s_ = c+restart;           // [restart]
	__shared__ double red[kWarps];
	if (state[0]) return;
	// eight independent running sums per thread (loads in flight, fixed order: deterministic)
	double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
	int b = threadIdx.x;
	for (; b+7*(int)blockDim.x < blocks; b += 8*blockDim.x) {
		#pragma unroll
		for (int u = 0; u < 8; ++u) acc[u] += norm_partial[b+u*blockDim.x];
	}
	for (int u = 0; b < blocks; b += blockDim.x, ++u) acc[u & 7] += norm_partial[b];
	double s = ((acc[0]+acc[1])+(acc[2]+acc[3]))+((acc[4]+acc[5])+(acc[6]+acc[7]));
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x >= 32) return;
	s = threadIdx.x < kWarps ? red[threadIdx.x] : 0.0;
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	const double next = sqrt(s);
	for (int i = threadIdx.x; i <= j; i += 32) col[i] = H[(size_t)i*restart+j];
	for (int i = threadIdx.x; i < j; i += 32) { c[i] = cs[i]; s_[i] = sn[i]; }
	__syncwarp();
	if (threadIdx.x == 0) {
		col[j+1] = next;
		for (int i = 0; i < j; ++i) {
			const double a = col[i], b = col[i+1];
			col[i] = c[i]*a+s_[i]*b;
			col[i+1] = -s_[i]*a+c[i]*b;
		}
		const double a = col[j], b = col[j+1];
		const double mag = hypot(a, b);
		const double cj = mag > 0.0 ? a/mag : 1.0, sj = mag > 0.0 ? b/mag : 0.0;
		cs[j] = cj; sn[j] = sj;
		col[j] = mag; col[j+1] = 0.0;
		const double old = g[j];
		g[j] = cj*old;
		g[j+1] = -sj*old;
		const double res = fabs(g[j+1]);
		residual[0] = res;
		scale[j+1] = next > 1e-30 ? 1.0/next : 0.0;
		state[1] = j+1;
		if (res <= tolerance || next <= 1e-30) state[0] = 1;
	}
	__syncwarp();
	for (int i = threadIdx.x; i <= j+1; i += 32) H[(size_t)i*restart+j] = col[i];
}

// Cycle start: g = beta e_0, scale_0 = 1/beta, flags cleared.
__global__ void CycleInitKernel(const double* __restrict__ beta, double* __restrict__ g, int restart,
	double* __restrict__ scale, int* __restrict__ state)
{
	for (int i = threadIdx.x; i <= restart; i += blockDim.x) g[i] = 0.0;
	if (threadIdx.x == 0) {
		g[0] = beta[0];
		scale[0] = beta[0] > 0.0 ? 1.0/beta[0] : 0.0;
		state[0] = 0; state[1] = 0; state[2] = 0;
	}
}

// Back substitution of the least-squares system (Gmres.hpp:308-315), column
// oriented: y_row = b_row / H_row,row, then every earlier right-hand side
// entry drops its H_t,row y_row term in parallel (one CTA, right-hand side in
// shared memory).
__global__ void __launch_bounds__(256) BackSolveKernel(const double* __restrict__ H, const double* __restrict__ g,
	int restart, const int* __restrict__ state, double* __restrict__ y, int* __restrict__ error_flag)
{
	extern __shared__ double rhs[];
	__shared__ double current;
	const int used = state[1];
	for (int i = threadIdx.x; i < used; i += blockDim.x) rhs[i] = g[i];
	__syncthreads();
	for (int row = used-1; row >= 0; --row) {
		if (threadIdx.x == 0) {
			const double d = H[(size_t)row*restart+row];
			double v = 0.0;
			if (fabs(d) < 1e-30) *error_flag = 1;
			else v = rhs[row]/d;
			y[row] = v;
			current = v;
		}
		__syncthreads();
		const double v = current;
		for (int t = threadIdx.x; t < row; t += blockDim.x) rhs[t] -= H[(size_t)t*restart+row]*v;
		__syncthreads();
	}
}

// x += sum_i y_i scale_i V_i over the columns of this cycle.
__global__ void __launch_bounds__(kThreads) SolutionUpdateKernel(const double* __restrict__ V, long long n,
	const double* __restrict__ scale, const double* __restrict__ y, const int* __restrict__ state,
	double* __restrict__ x)
{
	extern __shared__ double coef[];
	const int used = state[1];
	for (int i = threadIdx.x; i < used; i += blockDim.x) coef[i] = scale != nullptr ? y[i]*scale[i] : y[i];
	__syncthreads();
	for (long long k = (long long)blockIdx.x*blockDim.x+threadIdx.x; k < n; k += (long long)gridDim.x*blockDim.x) {
		double v = x[k];
		for (int i = 0; i < used; ++i) v = fma(coef[i], V[(size_t)i*n+k], v);
		x[k] = v;
	}
}

// out = scale[j] * in (materialise a lazily normalised Krylov vector).
template <class B>
__global__ void ScaleCopyKernel(long long n, const B* __restrict__ in, const double* __restrict__ scale,
	double* __restrict__ out, const int* __restrict__ stop)
{
	if (*stop) return;
	const double s = *scale;
	for (long long k = (long long)blockIdx.x*blockDim.x+threadIdx.x; k < n; k += (long long)gridDim.x*blockDim.x)
		out[k] = s*in[k];
}

__global__ void ResidualKernel(long long n, const double* __restrict__ rhs, const double* __restrict__ ax,
	double* __restrict__ r)
{
	const long long i = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (i < n) r[i] = rhs[i]-ax[i];
}

// Bytes classical Gram-Schmidt twice moves over one cycle of `used` Arnoldi
// steps: step j reads the j+1 basis vectors and w in each multi-dot, reads
// them again and writes w in each update, two passes: 8 n (4 (j+1) + 6).
double OrthoBytes(long long n, int used, int basis_bytes, bool fused)
{
	// step j, separate passes: both passes read the j+1 basis vectors twice (dot, update): 4 (j+1) sB n;
	// the FP64 work vector is read four times and written once, and the new basis vector is written:
	// (40 + sB) n.  Fused sweep: the basis three times (3 (j+1) sB n), the work vector read three times
	// and written once, the new vector written: (32 + sB) n.
	const double reads = fused ? 3.0 : 4.0, work = fused ? 32.0 : 40.0;
	return (double)n*(reads*basis_bytes*0.5*used*(used+1.0)+(work+basis_bytes)*used);
}

// The algorithmic bytes of the same steps: s_v n (2j + 7) per step with s_v the basis
// entry size, plus 8 n for the stored FP64 preconditioned vector of FGMRES.
double ArnoldiBytes(long long n, int used, int basis_bytes, bool flexible)
{
	return (double)n*(basis_bytes*(used*(used-1.0)+7.0*used)+(flexible ? 8.0*used : 0.0));
}

} // namespace

void Gmres::AddLowRank(const double* x, double* y, const int* stop)
{
	LowRankKernel<<<low_.count, kThreads, 0, stream_>>>(low_.ptr, low_.idx, low_.val, low_.coef, x, y, stop);
	LaunchCheck("LowRankKernel");
	launches_ += 1;
}

Gmres::Gmres(int nodes, int restart, cudaStream_t stream, int fields)
	: nodes_(nodes), fields_(fields), n_(fields*nodes), restart_(restart), blocks_(kBlocks), stream_(stream)
{
	if (nodes <= 0 || restart <= 0) Fail(-1, "GMRES workspace dimensions must be positive");
	if (fields != 2 && fields != 4) Fail(-7, "GMRES supports 2x2 and 4x4 blocks");
	// multi-dot chunk per CTA: a multiple of 128 doubles (16-byte aligned row slices, two-step unroll)
	chunk_ = (int)((((long long)n_+blocks_-1)/blocks_+127)/128*128);
	V_.Allocate((size_t)(restart+1)*n_);
	w_.Allocate(n_); r_.Allocate(n_); tmp_.Allocate(n_);
	inverse_.Allocate((size_t)nodes*fields*fields);
	partial_.Allocate((size_t)(restart+1)*blocks_);
	hpass_.Allocate(restart+1);
	H_.Allocate((size_t)(restart+1)*restart);
	cs_.Allocate(restart); sn_.Allocate(restart); g_.Allocate(restart+1); y_.Allocate(restart);
	scale_.Allocate(restart+1);
	update_blocks_ = (int)(((long long)n_/2+31)/32);
	norm_partial_.Allocate(std::max(std::max(PartialSlots(), blocks_), update_blocks_));
	scalar_.Allocate(2);
	state_.Allocate(4);
	residual_.Allocate(1);
	singular_.Allocate(1);
	CudaCheck(cudaMallocHost(reinterpret_cast<void**>(&host_), sizeof(HostStatus)), "pinned GMRES status");
	if ((size_t)chunk_*sizeof(double) > 48*1024) {
		CudaCheck(cudaFuncSetAttribute(MultiDotKernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)((size_t)chunk_*sizeof(double))), "multi-dot shared memory");
		CudaCheck(cudaFuncSetAttribute(MultiDotKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)((size_t)chunk_*sizeof(double))), "multi-dot shared memory");
	}
	if ((size_t)(restart+1)*sizeof(double) > 48*1024) {
		const int coef = (int)((size_t)(restart+1)*sizeof(double));
		CudaCheck(cudaFuncSetAttribute(UpdateKernel<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			coef), "update shared memory");
		CudaCheck(cudaFuncSetAttribute(UpdateKernel<float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			coef), "update shared memory");
		CudaCheck(cudaFuncSetAttribute(UpdateKernel<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			coef), "update shared memory");
		CudaCheck(cudaFuncSetAttribute(SolutionUpdateKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)((size_t)(restart+1)*sizeof(double))), "solution update shared memory");
	}
	if ((size_t)chunk_*sizeof(double) > 227*1024) Fail(-7, "GMRES vector too long for the multi-dot chunking");
	if ((size_t)(restart+1)*sizeof(double) > 48*1024)
		CudaCheck(cudaFuncSetAttribute(BackSolveKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)((size_t)(restart+1)*sizeof(double))), "back substitution shared memory");
	// fused sweep: chunks that keep a CTA's staged basis near 36 KiB (six CTAs per SM, so that loads of
	// some CTAs overlap the arithmetic of others; at 100 KiB, two CTAs per SM, the sweep was slower than
	// the separate passes); restarts too long for a 64-entry chunk keep the separate passes
	for (int b = 0; b < 2; ++b) {
		const size_t entry = b ? sizeof(double) : sizeof(float);
		const size_t budget = 36*1024-(size_t)(restart+2)*sizeof(double);
		int chunk = (int)(budget/((restart+1)*entry+sizeof(double)))/32*32;
		chunk = std::min(chunk, 2048);
		if (chunk < 64 || (b == 0 && n_ % 4 != 0)) continue;      // 16-byte slices of an FP32 basis
		fused_chunk_[b] = chunk;
		fused_blocks_[b] = (int)(((long long)n_+chunk-1)/chunk);
		fused_smem_[b] = (size_t)(((restart+1)+1) & ~1)*sizeof(double)+(size_t)chunk*sizeof(double)
			+(size_t)(restart+1)*chunk*entry;
	}
	if (fused_chunk_[0] || fused_chunk_[1]) {
		fused_partial_.Allocate((size_t)(restart+1)*std::max(fused_blocks_[0], fused_blocks_[1]));
		if (fused_chunk_[0])
			CudaCheck(cudaFuncSetAttribute(UpdateDotKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)fused_smem_[0]), "fused Gram-Schmidt shared memory");
		if (fused_chunk_[1])
			CudaCheck(cudaFuncSetAttribute(UpdateDotKernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)fused_smem_[1]), "fused Gram-Schmidt shared memory");
	}
	finalize_smem_ = (size_t)(3*restart+1)*sizeof(double);
	if (finalize_smem_ > 48*1024)
		CudaCheck(cudaFuncSetAttribute(ArnoldiFinalizeKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)finalize_smem_), "Arnoldi finalize shared memory");
}

Gmres::~Gmres()
{
	ReleaseSegmentGraphs();
	if (host_) cudaFreeHost(host_);
}

std::size_t Gmres::bytes() const
{
	return V_.bytes()+w_.bytes()+r_.bytes()+tmp_.bytes()+inverse_.bytes()+partial_.bytes()+H_.bytes();
}

template <class T>
void Gmres::Step(const DevicePatternView& pattern, const T* values, int j)
{
	const int* stop = state_.get();
	if (profiler_) profiler_->Begin(Profiler::kSpmv, stream_);
	if (fields_ == 2 && line_on_) {
		LaunchSpmvBlockJacobi2(pattern, values, static_cast<const double*>(nullptr), V_.get()+(size_t)j*n_,
			scale_.get()+j, tmp_.get(), stop, stream_);
		LaunchLineApply(line_, tmp_.get(), w_.get(), stop, stream_);
		launches_ += 1;
	} else if (fields_ == 2)
		LaunchSpmvBlockJacobi2(pattern, values, inverse_.get(), V_.get()+(size_t)j*n_, scale_.get()+j, w_.get(),
			stop, stream_);
	else
		LaunchSpmvBlockJacobi(pattern, values, inverse_.get(), V_.get()+(size_t)j*n_, scale_.get()+j, w_.get(), stop,
			stream_);
	if (profiler_) profiler_->End(stream_);
	launches_ += 1;
	Orthogonalize<double>(j, V_.get());
}

template <class B>
void Gmres::Orthogonalize(int j, B* basis)
{
	const int count = j+1;
	const int* stop = state_.get();
	const size_t dot_smem = (size_t)chunk_*sizeof(double);
	const size_t coef_smem = (size_t)(restart_+1)*sizeof(double);
	if (profiler_) profiler_->Begin(Profiler::kOrtho, stream_);
	const int fb = std::is_same<B, double>::value ? 1 : 0;
	if (fused_chunk_[fb]) {
		// first pass's dots; its update fused with the second pass's dots; the second pass's update
		MultiDotKernel<B><<<blocks_, kThreads, dot_smem, stream_>>>(basis, n_, scale_.get(), count, w_.get(),
			partial_.get(), chunk_, stop);
		LaunchCheck("MultiDotKernel");
		DotFinalizeKernel<<<(count+kThreads/32-1)/(kThreads/32), kThreads, 0, stream_>>>(partial_.get(), blocks_,
			count, hpass_.get(), H_.get(), restart_, j, 0, stop);
		LaunchCheck("DotFinalizeKernel");
		UpdateDotKernel<B><<<fused_blocks_[fb], kThreads, fused_smem_[fb], stream_>>>(basis, n_, scale_.get(), count,
			hpass_.get(), w_.get(), fused_partial_.get(), fused_chunk_[fb], stop);
		LaunchCheck("UpdateDotKernel");
		DotFinalizeKernel<<<(count+kThreads/32-1)/(kThreads/32), kThreads, 0, stream_>>>(fused_partial_.get(),
			fused_blocks_[fb], count, hpass_.get(), H_.get(), restart_, j, 1, stop);
		LaunchCheck("DotFinalizeKernel");
		UpdateKernel<B, B><<<update_blocks_, kThreads, coef_smem, stream_>>>(basis, n_, scale_.get(), count,
			hpass_.get(), w_.get(), basis+(size_t)(j+1)*n_, norm_partial_.get(), stop);
		LaunchCheck("UpdateKernel");
		ArnoldiFinalizeKernel<<<1, kThreads, finalize_smem_, stream_>>>(norm_partial_.get(), update_blocks_,
			H_.get(), restart_, j, cs_.get(), sn_.get(), g_.get(), scale_.get(), state_.get(), residual_.get(),
			tolerance_);
		LaunchCheck("ArnoldiFinalizeKernel");
		if (profiler_) profiler_->End(stream_);
		launches_ += 6;
		return;
	}
	for (int pass = 0; pass < 2; ++pass) {
		MultiDotKernel<B><<<blocks_, kThreads, dot_smem, stream_>>>(basis, n_, scale_.get(), count, w_.get(),
			partial_.get(), chunk_, stop);
		LaunchCheck("MultiDotKernel");
		DotFinalizeKernel<<<(count+kThreads/32-1)/(kThreads/32), kThreads, 0, stream_>>>(partial_.get(), blocks_,
			count, hpass_.get(), H_.get(), restart_, j, pass, stop);
		LaunchCheck("DotFinalizeKernel");
		if (pass == 0)
			UpdateKernel<B, double><<<update_blocks_, kThreads, coef_smem, stream_>>>(basis, n_, scale_.get(), count,
				hpass_.get(), w_.get(), w_.get(), nullptr, stop);
		else
			UpdateKernel<B, B><<<update_blocks_, kThreads, coef_smem, stream_>>>(basis, n_, scale_.get(), count,
				hpass_.get(), w_.get(), basis+(size_t)(j+1)*n_, norm_partial_.get(), stop);
		LaunchCheck("UpdateKernel");
	}
	ArnoldiFinalizeKernel<<<1, kThreads, finalize_smem_, stream_>>>(norm_partial_.get(), update_blocks_, H_.get(),
		restart_, j, cs_.get(), sn_.get(), g_.get(), scale_.get(), state_.get(), residual_.get(), tolerance_);
	LaunchCheck("ArnoldiFinalizeKernel");
	if (profiler_) profiler_->End(stream_);
	launches_ += 8;
}

template <> double* Gmres::Basis<double>() { return V_.get(); }
template <> float* Gmres::Basis<float>()
{
	if (V32_.size() == 0) V32_.Allocate((size_t)(restart_+1)*n_);
	return V32_.get();
}

template <class T, class B>
void Gmres::FlexibleStep(const DevicePatternView& pattern, const T* values, int j, Amg& M)
{
	const int* stop = state_.get();
	B* basis = Basis<B>();
	if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
	ScaleCopyKernel<B><<<blocks_, kThreads, 0, stream_>>>(n_, basis+(size_t)j*n_, scale_.get()+j, r_.get(), stop);
	LaunchCheck("ScaleCopyKernel");
	if (profiler_) profiler_->End(stream_);
	launches_ += 1;
	double* z = Z_.get()+(size_t)j*n_;
	M.Apply(values, r_.get(), z, stop);
	if (learned_ != nullptr) {
		// z += N(D^{-1} r) on the unit residual r
		LaunchApplyBlockInverse(nodes_, M.fine_inverse(), r_.get(), tmp_.get(), stream_);
		learned_->Apply(tmp_.get(), z, stop);
		launches_ += 1+3+learned_->layers();
	}
	if (profiler_) profiler_->Begin(Profiler::kSpmv, stream_);
	LaunchSpmvBlockJacobi<T>(pattern, values, nullptr, z, nullptr, w_.get(), stop, stream_);
	if (low_on_) AddLowRank(z, w_.get(), stop);
	if (profiler_) profiler_->End(stream_);
	launches_ += 1;
	if (collector_ != nullptr && j%kBatch == 0) {
		if (pair_dinv_.size() == 0) { pair_dinv_.Allocate(n_); pair_amg_.Allocate(n_); pair_aamg_.Allocate(n_); }
		LaunchApplyBlockInverse(nodes_, M.fine_inverse(), w_.get(), pair_dinv_.get(), stream_);
		M.Apply(values, w_.get(), pair_amg_.get(), stop);
		LaunchSpmv<T>(pattern, values, pair_amg_.get(), pair_aamg_.get(), stream_);
		collector_->AddKrylovPair(pair_dinv_.get(), z, pair_amg_.get(), w_.get(), pair_aamg_.get(), stop);
		launches_ += 6;
	}
	Orthogonalize<B>(j, basis);
}

template <class T, class B>
double Gmres::TrueResidualPlain(const DevicePatternView& pattern, const T* values, const double* rhs,
	const double* x)
{
	// v_0 = b - A x (FP64), stored in the basis precision; beta from the FP64 vector
	if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
	LaunchSpmv<T>(pattern, values, x, tmp_.get(), stream_);
	if (low_on_) AddLowRank(x, tmp_.get(), nullptr);
	double* r = std::is_same<B, double>::value ? V_.get() : r_.get();
	ResidualKernel<<<(unsigned)((n_+255)/256), 256, 0, stream_>>>(n_, rhs, tmp_.get(), r);
	LaunchCheck("ResidualKernel");
	LaunchNorm(n_, r, norm_partial_.get(), scalar_.get(), stream_);
	launches_ += 4;
	if (!std::is_same<B, double>::value) {
		LaunchToFloat(n_, r, reinterpret_cast<float*>(Basis<B>()), stream_);
		launches_ += 1;
	}
	if (profiler_) profiler_->End(stream_);
	scalar_.Download(host_->beta, 1, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "FGMRES residual");
	return host_->beta[0];
}

template <class T>
GmresResult Gmres::SolveFlexible(const DevicePatternView& pattern, const T* values, const double* rhs,
	double* x, double rtol, int max_iterations, Amg& M, long long* launches, bool fp64_basis)
{
	if (fields_ != 4) Fail(-7, "the flexible GMRES with AMG needs 4x4 blocks");
	if (fp64_basis || std::is_same<T, double>::value)
		return SolveFlexibleImpl<T, double>(pattern, values, rhs, x, rtol, max_iterations, M, launches);
	return SolveFlexibleImpl<T, float>(pattern, values, rhs, x, rtol, max_iterations, M, launches);
}

template <class T, class B>
GmresResult Gmres::SolveFlexibleImpl(const DevicePatternView& pattern, const T* values, const double* rhs,
	double* x, double rtol, int max_iterations, Amg& M, long long* launches)
{
	launches_ = 0;
	const long long amg0 = M.launches();
	if (Z_.size() == 0) Z_.Allocate((size_t)(restart_+1)*n_);
	GmresResult result;
	double beta = TrueResidualPlain<T, B>(pattern, values, rhs, x);
	result.residual = beta;
	if (!std::isfinite(beta)) Fail(-6, "FGMRES initial residual is not finite");
	if (beta == 0.0) {
		result.converged = true;
		if (launches) *launches += launches_;
		return result;
	}
	const double tolerance = std::max(1e-30, rtol*beta);
	tolerance_ = tolerance;
	while (result.iterations < max_iterations) {
		if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
		CycleInitKernel<<<1, 256, 0, stream_>>>(scalar_.get(), g_.get(), restart_, scale_.get(), state_.get());
		LaunchCheck("CycleInitKernel");
		H_.Zero(stream_);
		if (profiler_) profiler_->End(stream_);
		launches_ += 1;
		const int cap = std::min(restart_, max_iterations-result.iterations);
		for (int j = 0; j < cap;) {
			const int batch = std::min(kBatch, cap-j);
			for (int b = 0; b < batch; ++b) FlexibleStep<T, B>(pattern, values, j+b, M);
			j += batch;
			state_.Download(&host_->stop, 3, stream_);
			residual_.Download(&host_->residual, 1, stream_);
			CudaCheck(cudaStreamSynchronize(stream_), "FGMRES batch");
			if (host_->stop) break;
		}
		const int used = host_->used;
		result.iterations += used;
		if (profiler_) {
			profiler_->AddBytes(Profiler::kOrtho, ArnoldiBytes(n_, used, (int)sizeof(B), true));
			profiler_->AddMovedBytes(Profiler::kOrtho, OrthoBytes(n_, used, (int)sizeof(B),
				fused_chunk_[std::is_same<B, double>::value ? 1 : 0] != 0));
		}
		if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
		BackSolveKernel<<<1, 256, (size_t)(restart_+1)*sizeof(double), stream_>>>(H_.get(), g_.get(), restart_, state_.get(), y_.get(), state_.get()+2);
		LaunchCheck("BackSolveKernel");
		SolutionUpdateKernel<<<blocks_, kThreads, (size_t)(restart_+1)*sizeof(double), stream_>>>(Z_.get(), n_,
			nullptr, y_.get(), state_.get(), x);
		LaunchCheck("SolutionUpdateKernel");
		if (profiler_) profiler_->End(stream_);
		launches_ += 2;
		beta = TrueResidualPlain<T, B>(pattern, values, rhs, x);
		state_.Download(&host_->stop, 3, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "FGMRES restart");
		if (host_->error) Fail(-6, "FGMRES Hessenberg matrix is singular");
		result.residual = beta;
		if (!std::isfinite(beta)) Fail(-6, "FGMRES residual is not finite");
		if (beta <= tolerance) { result.converged = true; break; }
		if (used == 0) break;
	}
	if (launches) *launches += launches_+(M.launches()-amg0);
	return result;
}

double Gmres::TrueResidual(const DevicePatternView& pattern, const double* values, const double* rhs,
	const double* x)
{
	if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
	if (fields_ == 2) LaunchSpmv2(pattern, values, x, tmp_.get(), stream_);
	else LaunchSpmv(pattern, values, x, tmp_.get(), stream_);
	ResidualKernel<<<(unsigned)((n_+255)/256), 256, 0, stream_>>>(n_, rhs, tmp_.get(), r_.get());
	LaunchCheck("ResidualKernel");
	if (fields_ == 2 && line_on_) LaunchLineApply(line_, r_.get(), V_.get(), nullptr, stream_);
	else if (fields_ == 2) LaunchApplyBlockInverse2(nodes_, inverse_.get(), r_.get(), V_.get(), stream_);
	else LaunchApplyBlockInverse(nodes_, inverse_.get(), r_.get(), V_.get(), stream_);
	LaunchNorm(n_, V_.get(), norm_partial_.get(), scalar_.get(), stream_);
	if (profiler_) profiler_->End(stream_);
	launches_ += 5;
	scalar_.Download(host_->beta, 1, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "GMRES residual");
	return host_->beta[0];
}

GmresResult Gmres::Solve(const DevicePatternView& pattern, const double* values, const double* rhs, double* x,
	double rtol, int max_iterations, long long* launches, bool rebuild_preconditioner, const float* krylov_values)
{
	launches_ = 0;
	GmresResult result;
	if (rebuild_preconditioner) {
		singular_.Zero(stream_);
		if (fields_ == 2) LaunchBlockInverse2(pattern, values, inverse_.get(), singular_.get(), stream_);
		else LaunchBlockInverse(pattern, values, inverse_.get(), singular_.get(), stream_);
		launches_ += 1;
		singular_.Download(&host_->singular, 1, stream_);
	}
	double beta = TrueResidual(pattern, values, rhs, x);
	if (rebuild_preconditioner) singular_count_ = host_->singular;
	result.singular_blocks = singular_count_;
	result.residual = beta;
	if (!std::isfinite(beta)) Fail(-6, "GMRES initial residual is not finite");
	if (beta == 0.0) {
		result.converged = true;
		if (launches) *launches += launches_;
		return result;
	}
	const double tolerance = std::max(1e-30, rtol*beta);
	tolerance_ = tolerance;
	const size_t coef_smem = (size_t)(restart_+1)*sizeof(double);
	while (result.iterations < max_iterations) {
		if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
		CycleInitKernel<<<1, 256, 0, stream_>>>(scalar_.get(), g_.get(), restart_, scale_.get(), state_.get());
		LaunchCheck("CycleInitKernel");
		H_.Zero(stream_);
		if (profiler_) profiler_->End(stream_);
		launches_ += 1;
		const int cap = std::min(restart_, max_iterations-result.iterations);
		for (int j = 0; j < cap;) {
			const int batch = std::min(kBatch, cap-j);
			for (int b = 0; b < batch; ++b) {
				if (krylov_values) Step(pattern, krylov_values, j+b);
				else Step(pattern, values, j+b);
			}
			j += batch;
			state_.Download(&host_->stop, 3, stream_);
			residual_.Download(&host_->residual, 1, stream_);
			CudaCheck(cudaStreamSynchronize(stream_), "GMRES batch");
			if (host_->stop) break;
		}
		const int used = host_->used;
		result.iterations += used;
		if (profiler_) {
			profiler_->AddBytes(Profiler::kOrtho, ArnoldiBytes(n_, used, 8, false));
			profiler_->AddMovedBytes(Profiler::kOrtho, OrthoBytes(n_, used, 8, fused_chunk_[1] != 0));
		}
		result.residual = host_->residual;
		if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
		BackSolveKernel<<<1, 256, (size_t)(restart_+1)*sizeof(double), stream_>>>(H_.get(), g_.get(), restart_, state_.get(), y_.get(),
			state_.get()+2);
		LaunchCheck("BackSolveKernel");
		SolutionUpdateKernel<<<blocks_, kThreads, coef_smem, stream_>>>(V_.get(), n_, scale_.get(), y_.get(),
			state_.get(), x);
		LaunchCheck("SolutionUpdateKernel");
		if (profiler_) profiler_->End(stream_);
		launches_ += 2;
		beta = TrueResidual(pattern, values, rhs, x);
		state_.Download(&host_->stop, 3, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "GMRES restart");
		if (host_->error) Fail(-6, "GMRES Hessenberg matrix is singular");
		result.residual = beta;
		if (!std::isfinite(beta)) Fail(-6, "GMRES residual is not finite");
		if (beta <= tolerance) { result.converged = true; break; }
		if (used == 0) break;
	}
	if (launches) *launches += launches_;
	return result;
}

template GmresResult Gmres::SolveFlexible<double>(const DevicePatternView&, const double*, const double*, double*,
	double, int, Amg&, long long*, bool);
template GmresResult Gmres::SolveFlexible<float>(const DevicePatternView&, const float*, const double*, double*,
	double, int, Amg&, long long*, bool);

} // namespace tfiga
