// Flexible GMRES over independent segments of the unknowns (the tubes of a batched mesh): one Krylov
// iteration advances every segment's own Arnoldi process at once.  The preconditioner (AMG) and the
// operator (SpMV) run over the union -- the matrix is block diagonal over the segments and the AMG's
// aggregates never cross them -- while every segment keeps its own Gram-Schmidt coefficients,
// normalisation, Hessenberg matrix, Givens rotations, residual estimate and tolerance
// rtol * ||b_k - A_k x_k||, and stops on its own.  A stopped segment's next vector is zero, the SpMV
// skips its block rows and the Gram-Schmidt kernels its chunks, and the union's iteration ends when
// every segment has stopped.
// The single-system solver's tolerance definition (true residual at every restart) is kept per segment.
//
// Grids are two-dimensional: blockIdx.y is the segment, blockIdx.x a chunk of it (CTAs past the end of
// a short segment write zero partial sums and return), so no CTA straddles two segments and every
// reduction is per segment, in a fixed order.
#include "gmres.hpp"

#include <algorithm>
#include <cmath>
#include <type_traits>

namespace tfiga {
namespace {

constexpr int kSegThreads = 256;
constexpr int kSegWarps = kSegThreads/32;
constexpr int kDotChunk = 2048;              // entries per multi-dot CTA (the work vector chunk in shared memory)
constexpr int kVecChunk = 2*kSegThreads;     // entries per element-wise CTA (an entry pair per thread)
constexpr int kSegBatch = 8;                 // Arnoldi steps launched per host wait

template <class B> __device__ __forceinline__ double2 LoadPair(const B* p, long long k2);
template <> __device__ __forceinline__ double2 LoadPair<double>(const double* p, long long k2)
{
	return reinterpret_cast<const double2*>(p)[k2];
}
template <> __device__ __forceinline__ double2 LoadPair<float>(const float* p, long long k2)
{
	const float2 v = reinterpret_cast<const float2*>(p)[k2];
	return make_double2(v.x, v.y);
}
template <class B> __device__ __forceinline__ void StorePair(B* p, long long k2, double2 v);
template <> __device__ __forceinline__ void StorePair<double>(double* p, long long k2, double2 v)
{
	reinterpret_cast<double2*>(p)[k2] = v;
}
template <> __device__ __forceinline__ void StorePair<float>(float* p, long long k2, double2 v)
{
	reinterpret_cast<float2*>(p)[k2] = make_float2((float)v.x, (float)v.y);
}

// Per-segment state: stop[s] (1 once the segment has converged or broken down), used[s] (Arnoldi
// columns of the current cycle), and the union's flags all[0] (every segment stopped), all[1]
// (largest used), all[2] (singular Hessenberg).

// out = scale[s][j] V_j on segment s (zero on a stopped segment, whatever V_j holds there).
template <class B>
__global__ void __launch_bounds__(kSegThreads) SegScaleCopyKernel(const int64_t* __restrict__ off,
	const B* __restrict__ v, const double* __restrict__ scale, int stride, int j, double* __restrict__ out,
	const int* __restrict__ all)
{
	if (all[0]) return;
	const int s = blockIdx.y;
	const long long lo = off[s], hi = off[s+1];
	const long long k2 = (lo >> 1)+(long long)blockIdx.x*kSegThreads+threadIdx.x;
	if (2*k2 >= hi) return;
	const double c = scale[(size_t)s*stride+j];
	const double2 x = c == 0.0 ? make_double2(0.0, 0.0) : LoadPair<B>(v, k2);
	reinterpret_cast<double2*>(out)[k2] = make_double2(c*x.x, c*x.y);
}

// partial[(s stride + i) cx + bx] = scale[s][i] <V_i, w> over this CTA's chunk of segment s.
template <class B>
__global__ void __launch_bounds__(kSegThreads) SegMultiDotKernel(const int64_t* __restrict__ off,
	const B* __restrict__ V, long long n, const double* __restrict__ scale, int stride, int count,
	const double* __restrict__ w, double* __restrict__ partial, const int* __restrict__ stop,
	const int* __restrict__ all)
{
	if (all[0]) return;
	__shared__ double2 ws[kDotChunk/2];
	const int s = blockIdx.y, cx = gridDim.x, bx = blockIdx.x;
	const long long lo = off[s]+(long long)bx*kDotChunk, hi = off[s+1];
	const int len2 = (stop[s] || lo >= hi) ? 0 : (int)(min((long long)kDotChunk, hi-lo) >> 1);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (len2 == 0) {
		for (int i = threadIdx.x; i < count; i += blockDim.x) partial[((size_t)s*stride+i)*cx+bx] = 0.0;
		return;
	}
	const double2* win = reinterpret_cast<const double2*>(w+lo);
	for (int k = threadIdx.x; k < len2; k += blockDim.x) ws[k] = win[k];
	__syncthreads();
	for (int i = warp; i < count; i += kSegWarps) {
		const B* a = V+(size_t)i*n+lo;
		double t0 = 0.0, t1 = 0.0;
		for (int k = lane; k < len2; k += 32) {
			const double2 x = LoadPair<B>(a, k), y = ws[k];
			t0 = fma(x.x, y.x, t0);
			t1 = fma(x.y, y.y, t1);
		}
		double t = t0+t1;
		for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
		if (lane == 0) partial[((size_t)s*stride+i)*cx+bx] = t*scale[(size_t)s*stride+i];
	}
}

// hpass[s][i] = sum over the segment's CTAs; H[s][i][j] = (pass == 0 ? hpass : H + hpass).  A warp per
// (segment, i).
__global__ void __launch_bounds__(kSegThreads) SegDotFinalizeKernel(const double* __restrict__ partial, int cx,
	int segments, int stride, int count, double* __restrict__ hpass, double* __restrict__ H, int restart, int j,
	int pass, const int* __restrict__ stop, const int* __restrict__ all)
{
	if (all[0]) return;
	const int task = blockIdx.x*kSegWarps+(threadIdx.x >> 5), lane = threadIdx.x & 31;
	if (task >= segments*count) return;
	const int s = task/count, i = task%count;
	if (stop[s]) return;
	double t = 0.0;
	for (int b = lane; b < cx; b += 32) t += partial[((size_t)s*stride+i)*cx+b];
	for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
	if (lane == 0) {
		hpass[(size_t)s*stride+i] = t;
		double& h = H[((size_t)s*(restart+1)+i)*restart+j];
		h = pass == 0 ? t : h+t;
	}
}

// out = w - sum_i scale[s][i] hpass[s][i] V_i on segment s; norm_partial[s ux + bx] = sum out^2 (if
// non-null).  out may alias w.  Stopped segments are left alone.
template <class B, class O>
__global__ void __launch_bounds__(kSegThreads) SegUpdateKernel(const int64_t* __restrict__ off,
	const B* __restrict__ V, long long n, const double* __restrict__ scale, const double* __restrict__ hpass,
	int stride, int count, const double* win, O* out, double* __restrict__ norm_partial, const int* __restrict__ stop,
	const int* __restrict__ all)
{
	if (all[0]) return;
	__shared__ double coef[129];
	__shared__ double red[kSegWarps];
	const int s = blockIdx.y, ux = gridDim.x, bx = blockIdx.x;
	const long long lo = off[s], hi = off[s+1];
	const long long k2 = (lo >> 1)+(long long)bx*kSegThreads+threadIdx.x;
	const bool live = !stop[s] && lo+(long long)bx*kVecChunk < hi;
	if (!live) {
		if (norm_partial != nullptr && threadIdx.x == 0) norm_partial[(size_t)s*ux+bx] = 0.0;
		return;
	}
	for (int i = threadIdx.x; i < count; i += blockDim.x) coef[i] = scale[(size_t)s*stride+i]*hpass[(size_t)s*stride+i];
	__syncthreads();
	double sq = 0.0;
	if (2*k2 < hi) {
		double2 v = reinterpret_cast<const double2*>(win)[k2];
		for (int i = 0; i < count; ++i) {
			const double2 a = LoadPair<B>(V+(size_t)i*n, k2);
			v.x = fma(-coef[i], a.x, v.x);
			v.y = fma(-coef[i], a.y, v.y);
		}
		StorePair<O>(out, k2, v);
		sq = fma(v.x, v.x, v.y*v.y);
	}
	if (norm_partial == nullptr) return;
	for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		#pragma unroll
		for (int w = 0; w < kSegWarps; ++w) t += red[w];
		norm_partial[(size_t)s*ux+bx] = t;
	}
}

// Column j of every open segment's Hessenberg matrix: norm, previous rotations, new rotation,
// residual estimate; a segment stops when its estimate reaches its tolerance or its new vector
// vanishes.  One thread per segment.
__global__ void SegArnoldiFinalizeKernel(const double* __restrict__ norm_partial, int ux, int segments,
	double* __restrict__ H, int restart, int j, double* __restrict__ cs, double* __restrict__ sn,
	double* __restrict__ g, double* __restrict__ scale, int stride, const double* __restrict__ tolerance,
	int* __restrict__ stop, int* __restrict__ used, double* __restrict__ residual, int* __restrict__ all)
{
	if (all[0]) return;
	const int s = blockIdx.x*blockDim.x+threadIdx.x;
	bool stopped = true;
	if (s < segments) {
		stopped = stop[s] != 0;
		if (!stopped) {
			double t = 0.0;
			for (int b = 0; b < ux; ++b) t += norm_partial[(size_t)s*ux+b];
			const double next = sqrt(t);
			double* Hs = H+(size_t)s*(restart+1)*restart;
			double* c = cs+(size_t)s*restart;
			double* sv = sn+(size_t)s*restart;
			double* gs = g+(size_t)s*stride;
			for (int i = 0; i < j; ++i) {
				const double a = Hs[(size_t)i*restart+j], b = Hs[(size_t)(i+1)*restart+j];
				Hs[(size_t)i*restart+j] = c[i]*a+sv[i]*b;
				Hs[(size_t)(i+1)*restart+j] = -sv[i]*a+c[i]*b;
			}
			const double a = Hs[(size_t)j*restart+j], b = next;
			const double mag = hypot(a, b);
			const double cj = mag > 0.0 ? a/mag : 1.0, sj = mag > 0.0 ? b/mag : 0.0;
			c[j] = cj; sv[j] = sj;
			Hs[(size_t)j*restart+j] = mag;
			Hs[(size_t)(j+1)*restart+j] = 0.0;
			const double old = gs[j];
			gs[j] = cj*old;
			gs[j+1] = -sj*old;
			const double res = fabs(gs[j+1]);
			residual[s] = res;
			used[s] = j+1;
			stopped = res <= tolerance[s] || next <= 1e-30;
			scale[(size_t)s*stride+j+1] = (!stopped && next > 1e-30) ? 1.0/next : 0.0;
			if (stopped) stop[s] = 1;
		}
	}
	// every segment stopped: the union's iteration ends (one CTA covers all segments)
	const int open = __syncthreads_count(!stopped);
	if (threadIdx.x == 0) {
		if (open == 0) all[0] = 1;
		all[1] = j+1;
	}
}

// Cycle start per segment: g = beta e_0, scale_0 = 1/beta, rotations cleared, stopped when the segment
// already meets its tolerance.
__global__ void SegCycleInitKernel(const double* __restrict__ beta, const double* __restrict__ tolerance,
	int segments, int restart, int stride, double* __restrict__ g, double* __restrict__ scale, int* __restrict__ stop,
	int* __restrict__ used, int* __restrict__ all)
{
	const int s = blockIdx.x*blockDim.x+threadIdx.x;
	bool stopped = true;
	if (s < segments) {
		for (int i = 0; i <= restart; ++i) { g[(size_t)s*stride+i] = 0.0; scale[(size_t)s*stride+i] = 0.0; }
		const double b = beta[s];
		stopped = !(b > tolerance[s]);
		g[(size_t)s*stride] = b;
		scale[(size_t)s*stride] = stopped ? 0.0 : 1.0/b;
		stop[s] = stopped ? 1 : 0;
		used[s] = 0;
	}
	const int open = __syncthreads_count(!stopped);
	if (threadIdx.x == 0) { all[0] = open == 0 ? 1 : 0; all[1] = 0; all[2] = 0; }
}

// Back substitution per segment (one CTA each), over the segment's used columns.
__global__ void __launch_bounds__(256) SegBackSolveKernel(const double* __restrict__ H, const double* __restrict__ g,
	int restart, int stride, const int* __restrict__ used, double* __restrict__ y, int* __restrict__ all)
{
	extern __shared__ double rhs[];
	__shared__ double current;
	const int s = blockIdx.x;
	const int u = used[s];
	const double* Hs = H+(size_t)s*(restart+1)*restart;
	double* ys = y+(size_t)s*stride;
	for (int i = threadIdx.x; i < u; i += blockDim.x) rhs[i] = g[(size_t)s*stride+i];
	__syncthreads();
	for (int row = u-1; row >= 0; --row) {
		if (threadIdx.x == 0) {
			const double d = Hs[(size_t)row*restart+row];
			double v = 0.0;
			if (fabs(d) < 1e-30) all[2] = 1;
			else v = rhs[row]/d;
			ys[row] = v;
			current = v;
		}
		__syncthreads();
		const double v = current;
		for (int t = threadIdx.x; t < row; t += blockDim.x) rhs[t] -= Hs[(size_t)t*restart+row]*v;
		__syncthreads();
	}
}

// x += sum_{i < used[s]} y[s][i] Z_i on segment s.
__global__ void __launch_bounds__(kSegThreads) SegSolutionUpdateKernel(const int64_t* __restrict__ off,
	const double* __restrict__ Z, long long n, const double* __restrict__ y, int stride, const int* __restrict__ used,
	double* __restrict__ x)
{
	const int s = blockIdx.y;
	const long long lo = off[s], hi = off[s+1];
	const long long k2 = (lo >> 1)+(long long)blockIdx.x*kSegThreads+threadIdx.x;
	const int u = used[s];
	if (u == 0 || 2*k2 >= hi) return;
	double2 v = reinterpret_cast<const double2*>(x)[k2];
	for (int i = 0; i < u; ++i) {
		const double c = y[(size_t)s*stride+i];
		const double2 z = reinterpret_cast<const double2*>(Z+(size_t)i*n)[k2];
		v.x = fma(c, z.x, v.x);
		v.y = fma(c, z.y, v.y);
	}
	reinterpret_cast<double2*>(x)[k2] = v;
}

__global__ void SegResidualKernel(long long n, const double* __restrict__ rhs, const double* __restrict__ ax,
	double* __restrict__ r)
{
	const long long i = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (i < n) r[i] = rhs[i]-ax[i];
}

template <class B>
__global__ void SegStoreBasisKernel(long long n, const double* __restrict__ r, B* __restrict__ v)
{
	const long long i = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (i < n) v[i] = (B)r[i];
}

} // namespace

void Gmres::SetSegments(const std::vector<int64_t>& entry_offsets, const std::vector<int64_t>& blocks)
{
	ReleaseSegmentGraphs();
	const int count = (int)entry_offsets.size()-1;
	if (count <= 0) { segments_ = 0; return; }
	if (count > 1024) Fail(-7, "at most 1024 segments per flexible solve");
	if (entry_offsets[0] != 0 || entry_offsets[count] != n_) Fail(-1, "segments must cover the unknowns");
	for (int k = 0; k <= count; ++k)
		if (entry_offsets[k] % fields_) Fail(-1, "segments must hold whole nodes");
	int64_t longest = 0;
	for (int k = 0; k < count; ++k) {
		if (entry_offsets[k+1] <= entry_offsets[k] || (entry_offsets[k] & 1)) Fail(-1, "bad segment offsets");
		longest = std::max<int64_t>(longest, entry_offsets[k+1]-entry_offsets[k]);
	}
	if (restart_+1 > 129) Fail(-7, "segmented flexible GMRES supports restarts up to 128");
	segments_ = count;
	seg_dot_cx_ = (int)((longest+kDotChunk-1)/kDotChunk);
	seg_len_.resize(count);
	for (int k = 0; k < count; ++k) seg_len_[k] = entry_offsets[k+1]-entry_offsets[k];
	seg_vec_cx_ = (int)((longest+kVecChunk-1)/kVecChunk);
	const int stride = restart_+1;
	seg_off_.Allocate(count+1);
	seg_off_.Upload(entry_offsets.data(), count+1, stream_);
	std::vector<int32_t> node_seg(n_/fields_);
	for (int k = 0; k < count; ++k)
		for (int64_t e = entry_offsets[k]/fields_; e < entry_offsets[k+1]/fields_; ++e) node_seg[e] = k;
	seg_node_.Allocate(node_seg.size());
	seg_node_.Upload(node_seg.data(), node_seg.size(), stream_);
	seg_H_.Allocate((size_t)count*(restart_+1)*restart_);
	seg_cs_.Allocate((size_t)count*restart_);
	seg_sn_.Allocate((size_t)count*restart_);
	seg_g_.Allocate((size_t)count*stride);
	seg_y_.Allocate((size_t)count*stride);
	seg_scale_.Allocate((size_t)count*stride);
	seg_hpass_.Allocate((size_t)count*stride);
	seg_partial_.Allocate((size_t)count*stride*seg_dot_cx_);
	seg_norm_partial_.Allocate((size_t)count*seg_vec_cx_);
	seg_tol_.Allocate(count);
	seg_beta_.Allocate(count);
	seg_sq_.Allocate(count);
	seg_residual_.Allocate(count);
	seg_stop_.Allocate(count);
	seg_used_.Allocate(count);
	seg_all_.Allocate(4);
	seg_host_beta_.assign(count, 0.0);
	seg_host_tol_.assign(count, 0.0);
	seg_host_flags_.assign(4, 0);
	seg_host_stop_.assign(count, 0);
	seg_blocks_ = blocks;
	CudaCheck(cudaStreamSynchronize(stream_), "segments");
}

template <class T, class B>
void Gmres::SegTrueResidual(const DevicePatternView& pattern, const T* values, const double* rhs, const double* x)
{
	if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
	LaunchSpmv<T>(pattern, values, x, tmp_.get(), stream_);
	if (low_on_) AddLowRank(x, tmp_.get(), nullptr);
	SegResidualKernel<<<(unsigned)((n_+255)/256), 256, 0, stream_>>>(n_, rhs, tmp_.get(), r_.get());
	LaunchCheck("SegResidualKernel");
	SegStoreBasisKernel<B><<<(unsigned)((n_+255)/256), 256, 0, stream_>>>(n_, r_.get(), Basis<B>());
	LaunchCheck("SegStoreBasisKernel");
	LaunchSegmentSquares(segments_, seg_off_.get(), r_.get(), seg_sq_.get(), stream_);
	launches_ += 4;
	if (profiler_) profiler_->End(stream_);
	seg_sq_.Download(seg_host_beta_.data(), segments_, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "segmented FGMRES residual");
	for (double& b : seg_host_beta_) b = std::sqrt(b);
	seg_beta_.Upload(seg_host_beta_.data(), segments_, stream_);
}

template <class T, class B>
void Gmres::SegFlexibleStep(const DevicePatternView& pattern, const T* values, int j, Amg& M)
{
	const int* all = seg_all_.get();
	const int stride = restart_+1, count = j+1;
	B* basis = Basis<B>();
	const dim3 vec_grid(seg_vec_cx_, segments_), dot_grid(seg_dot_cx_, segments_);
	if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
	SegScaleCopyKernel<B><<<vec_grid, kSegThreads, 0, stream_>>>(seg_off_.get(), basis+(size_t)j*n_, seg_scale_.get(),
		stride, j, r_.get(), all);
	LaunchCheck("SegScaleCopyKernel");
	if (profiler_) profiler_->End(stream_);
	double* z = Z_.get()+(size_t)j*n_;
	M.Apply(values, r_.get(), z, all, seg_stop_.get());   // stopped tubes' nodes and aggregates skipped
	if (profiler_) profiler_->Begin(Profiler::kSpmv, stream_);
	// the rows of stopped segments are skipped: nothing reads their w again in this cycle
	LaunchSpmvMasked<T>(pattern, values, z, w_.get(), all, seg_node_.get(), seg_stop_.get(), stream_);
	if (low_on_) AddLowRank(z, w_.get(), all);
	if (profiler_) profiler_->End(stream_);
	launches_ += 2;
	// classical Gram-Schmidt twice, per segment
	if (profiler_) profiler_->Begin(Profiler::kOrtho, stream_);
	const unsigned fin_blocks = (unsigned)((segments_*count+kSegWarps-1)/kSegWarps);
	for (int pass = 0; pass < 2; ++pass) {
		SegMultiDotKernel<B><<<dot_grid, kSegThreads, 0, stream_>>>(seg_off_.get(), basis, n_, seg_scale_.get(), stride,
			count, w_.get(), seg_partial_.get(), seg_stop_.get(), all);
		LaunchCheck("SegMultiDotKernel");
		SegDotFinalizeKernel<<<fin_blocks, kSegThreads, 0, stream_>>>(seg_partial_.get(), seg_dot_cx_, segments_, stride,
			count, seg_hpass_.get(), seg_H_.get(), restart_, j, pass, seg_stop_.get(), all);
		LaunchCheck("SegDotFinalizeKernel");
		if (pass == 0)
			SegUpdateKernel<B, double><<<vec_grid, kSegThreads, 0, stream_>>>(seg_off_.get(), basis, n_, seg_scale_.get(),
				seg_hpass_.get(), stride, count, w_.get(), w_.get(), nullptr, seg_stop_.get(), all);
		else
			SegUpdateKernel<B, B><<<vec_grid, kSegThreads, 0, stream_>>>(seg_off_.get(), basis, n_, seg_scale_.get(),
				seg_hpass_.get(), stride, count, w_.get(), basis+(size_t)(j+1)*n_, seg_norm_partial_.get(), seg_stop_.get(),
				all);
		LaunchCheck("SegUpdateKernel");
	}
	SegArnoldiFinalizeKernel<<<1, 1024, 0, stream_>>>(seg_norm_partial_.get(), seg_vec_cx_, segments_, seg_H_.get(),
		restart_, j, seg_cs_.get(), seg_sn_.get(), seg_g_.get(), seg_scale_.get(), stride, seg_tol_.get(),
		seg_stop_.get(), seg_used_.get(), seg_residual_.get(), seg_all_.get());
	LaunchCheck("SegArnoldiFinalizeKernel");
	if (profiler_) profiler_->End(stream_);
	launches_ += 8;
}

void Gmres::ReleaseSegmentGraphs()
{
	for (auto& g : seg_graphs_)
		if (g) cudaGraphExecDestroy(g);
	seg_graphs_.clear();
	seg_graph_launches_.clear();
	seg_graph_amg_launches_.clear();
	seg_graph_values_ = nullptr;
	seg_graph_amg_ = nullptr;
}

template <class T, class B>
void Gmres::SegStep(const DevicePatternView& pattern, const T* values, int j, Amg& M)
{
	const bool profiling = profiler_ != nullptr && profiler_->enabled();
	if (!seg_graphs_ok_ || profiling || low_on_ || learned_ != nullptr) {
		SegFlexibleStep<T, B>(pattern, values, j, M);
		return;
	}
	if (seg_graph_values_ != static_cast<const void*>(values) || seg_graph_amg_ != static_cast<const void*>(&M))
		ReleaseSegmentGraphs();
	if ((int)seg_graphs_.size() < restart_) {
		seg_graphs_.resize(restart_, nullptr);
		seg_graph_launches_.resize(restart_, 0);
		seg_graph_amg_launches_.resize(restart_, 0);
	}
	seg_graph_values_ = values;
	seg_graph_amg_ = &M;
	if (seg_graphs_[j] == nullptr) {
		const long long own0 = launches_, amg0 = M.launches();
		cudaGraph_t graph = nullptr;
		if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
			(void)cudaGetLastError();
			seg_graphs_ok_ = false;
			SegFlexibleStep<T, B>(pattern, values, j, M);
			return;
		}
		SegFlexibleStep<T, B>(pattern, values, j, M);
		const cudaError_t end = cudaStreamEndCapture(stream_, &graph);
		cudaGraphExec_t exec = nullptr;
		const bool ok = end == cudaSuccess && graph != nullptr
			&& cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
		if (graph) cudaGraphDestroy(graph);
		if (!ok) {
			// nothing of the step ran while it was being captured: run it directly from now on
			(void)cudaGetLastError();
			seg_graphs_ok_ = false;
			launches_ = own0;
			SegFlexibleStep<T, B>(pattern, values, j, M);
			return;
		}
		seg_graphs_[j] = exec;
		seg_graph_launches_[j] = launches_-own0;
		seg_graph_amg_launches_[j] = M.launches()-amg0;
		launches_ = own0;
		M.count_launches(-seg_graph_amg_launches_[j]);
	}
	CudaCheck(cudaGraphLaunch(seg_graphs_[j], stream_), "segmented FGMRES step graph");
	launches_ += seg_graph_launches_[j];
	M.count_launches(seg_graph_amg_launches_[j]);
}

template <class T>
GmresResult Gmres::SolveFlexibleSegments(const DevicePatternView& pattern, const T* values, const double* rhs,
	double* x, double rtol, int max_iterations, Amg& M, long long* launches, bool fp64_basis)
{
	if (fields_ != 4) Fail(-7, "the flexible GMRES with AMG needs 4x4 blocks");
	if (segments_ == 0) Fail(-1, "segmented flexible GMRES without segments");
	if (fp64_basis || std::is_same<T, double>::value)
		return SolveFlexibleSegmentsImpl<T, double>(pattern, values, rhs, x, rtol, max_iterations, M, launches);
	return SolveFlexibleSegmentsImpl<T, float>(pattern, values, rhs, x, rtol, max_iterations, M, launches);
}

template <class T, class B>
GmresResult Gmres::SolveFlexibleSegmentsImpl(const DevicePatternView& pattern, const T* values, const double* rhs,
	double* x, double rtol, int max_iterations, Amg& M, long long* launches)
{
	launches_ = 0;
	const long long amg0 = M.launches();
	if (Z_.size() == 0) Z_.Allocate((size_t)(restart_+1)*n_);
	const int stride = restart_+1;
	GmresResult result;
	SegTrueResidual<T, B>(pattern, values, rhs, x);
	double total = 0.0;
	for (int k = 0; k < segments_; ++k) {
		const double b = seg_host_beta_[k];
		if (!std::isfinite(b)) Fail(-6, "FGMRES initial residual is not finite");
		seg_host_tol_[k] = std::max(1e-300, rtol*b);
		total += b*b;
	}
	result.residual = std::sqrt(total);
	seg_tol_.Upload(seg_host_tol_.data(), segments_, stream_);
	auto all_met = [&]() {
		for (int k = 0; k < segments_; ++k)
			if (!(seg_host_beta_[k] <= seg_host_tol_[k])) return false;
		return true;
	};
	if (all_met()) {
		result.converged = true;
		if (launches) *launches += launches_;
		return result;
	}
	const unsigned init_threads = (unsigned)std::max(32, (segments_+31)/32*32);
	while (result.iterations < max_iterations) {
		if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
		SegCycleInitKernel<<<1, init_threads, 0, stream_>>>(seg_beta_.get(), seg_tol_.get(), segments_, restart_, stride,
			seg_g_.get(), seg_scale_.get(), seg_stop_.get(), seg_used_.get(), seg_all_.get());
		LaunchCheck("SegCycleInitKernel");
		seg_H_.Zero(stream_);
		if (profiler_) profiler_->End(stream_);
		launches_ += 1;
		const int cap = std::min(restart_, max_iterations-result.iterations);
		int used = 0;
		for (int j = 0; j < cap;) {
			const int batch = std::min(kSegBatch, cap-j);
			for (int b = 0; b < batch; ++b) SegStep<T, B>(pattern, values, j+b, M);
			seg_all_.Download(seg_host_flags_.data(), 3, stream_);
			if (profiler_) seg_stop_.Download(seg_host_stop_.data(), segments_, stream_);
			CudaCheck(cudaStreamSynchronize(stream_), "segmented FGMRES batch");
			if (profiler_) {
				// the work of the segments still open at the end of the batch (a lower bound: a segment
				// that stopped inside the batch did part of it): SpMV blocks and vectors, and the
				// Gram-Schmidt traffic of steps j .. j + batch - 1 over their entries
				double entries = 0.0, blocks = 0.0;
				for (int k = 0; k < segments_; ++k)
					if (!seg_host_stop_[k]) {
						const double len = (double)(seg_len_[k]);
						entries += len;
						if ((size_t)k < seg_blocks_.size()) blocks += (double)seg_blocks_[k];
					}
				const double basis = (double)sizeof(B), vb = sizeof(T) == 4 ? 68.0 : 132.0;
				profiler_->AddBytes(Profiler::kSpmv, batch*(blocks*vb+entries*(8.0+8.0)));
				double algo = 0.0, moved = 0.0;
				for (int s = j; s < j+batch; ++s) {
					algo += entries*(basis*(2.0*s+7.0)+8.0);
					moved += entries*(4.0*basis*(s+1.0)+40.0+basis);
				}
				profiler_->AddBytes(Profiler::kOrtho, algo);
				profiler_->AddMovedBytes(Profiler::kOrtho, moved);
			}
			j += batch;
			used = seg_host_flags_[1];
			if (seg_host_flags_[0]) break;
		}
		result.iterations += used;
		if (profiler_) profiler_->Begin(Profiler::kVector, stream_);
		SegBackSolveKernel<<<segments_, 256, (size_t)(restart_+1)*sizeof(double), stream_>>>(seg_H_.get(), seg_g_.get(),
			restart_, stride, seg_used_.get(), seg_y_.get(), seg_all_.get());
		LaunchCheck("SegBackSolveKernel");
		SegSolutionUpdateKernel<<<dim3(seg_vec_cx_, segments_), kSegThreads, 0, stream_>>>(seg_off_.get(), Z_.get(), n_,
			seg_y_.get(), stride, seg_used_.get(), x);
		LaunchCheck("SegSolutionUpdateKernel");
		if (profiler_) profiler_->End(stream_);
		launches_ += 2;
		SegTrueResidual<T, B>(pattern, values, rhs, x);
		seg_all_.Download(seg_host_flags_.data(), 3, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "segmented FGMRES restart");
		if (seg_host_flags_[2]) Fail(-6, "FGMRES Hessenberg matrix is singular");
		total = 0.0;
		for (int k = 0; k < segments_; ++k) {
			if (!std::isfinite(seg_host_beta_[k])) Fail(-6, "FGMRES residual is not finite");
			total += seg_host_beta_[k]*seg_host_beta_[k];
		}
		result.residual = std::sqrt(total);
		if (all_met()) { result.converged = true; break; }
		if (used == 0) break;
	}
	if (launches) *launches += launches_+(M.launches()-amg0);
	return result;
}

template GmresResult Gmres::SolveFlexibleSegments<float>(const DevicePatternView&, const float*, const double*,
	double*, double, int, Amg&, long long*, bool);
template GmresResult Gmres::SolveFlexibleSegments<double>(const DevicePatternView&, const double*, const double*,
	double*, double, int, Amg&, long long*, bool);

} // namespace tfiga
