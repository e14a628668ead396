// Point-block aggregation AMG: host setup, device refresh and V-cycle (see amg.hpp).
#include "amg.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace tfiga {

struct Amg::Level {
	int nodes = 0;
	long long blocks = 0;
	std::vector<int32_t> h_rows, h_cols, h_diag;     // pattern of this level's operator
	std::vector<double> h_mask;                      // [4*nodes] 1 = free DOF
	DeviceArray<int32_t> rows, cols, diag;
	DeviceArray<double> values, inverse, mask, x, b, r;
	DeviceArray<unsigned> singular;
	// transfer to the next level
	std::vector<int32_t> h_agg;
	DeviceArray<int32_t> agg, agg_order, agg_offsets, gal_order, gal_offsets, block_row;
	// A P (this level's operator times the masked prolongation): block rows of the fine
	// nodes, block columns of the coarse nodes, and the fixed-order fine-block lists
	long long ap_blocks = 0;
	DeviceArray<int32_t> ap_rows, ap_cols, ap_order, ap_offsets;
	DeviceArray<double> ap_values;      // A P with an FP64 fine matrix
	DeviceArray<float> ap_values32;     // A P with an FP32 fine matrix (stored in its precision)
	// coarsest level
	int dense_n = 0;
	DeviceArray<double> dense, column;
	DeviceArray<double> panel;          // blocked Gauss-Jordan: two n x 32 panel copies + the 32 x 32 pivot-block inverse
	DeviceArray<int> dense_flag, pivots;
	DevicePatternView view() const { return {nodes, blocks, rows.get(), cols.get(), diag.get()}; }
};

namespace {

constexpr int kThreads = 256;
constexpr int kPanel = 32;          // pivot columns per blocked Gauss-Jordan panel

unsigned Grid(long long n, int per) { return (unsigned)((n+per-1)/per); }

template <class T>
__global__ void StrengthKernel(long long blocks, const T* __restrict__ values, double* __restrict__ s)
{
	const long long b = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (b >= blocks) return;
	const T* v = values+b*16;
	s[b] = fabs((double)v[0])+fabs((double)v[5])+fabs((double)v[10]);
}

// Coarse block = masked sum of its fine blocks: one CTA per coarse block, each
// thread accumulating a strided subset of the fine blocks, then a fixed-order
// reduction in shared memory (deterministic).
template <class T>
__global__ void __launch_bounds__(128) GalerkinKernel(long long coarse_blocks, const int32_t* __restrict__ order,
	const int32_t* __restrict__ offsets, const int32_t* __restrict__ block_row, const int32_t* __restrict__ fine_cols,
	const double* __restrict__ fine_mask, const T* __restrict__ fine_values, double* __restrict__ coarse_values)
{
	const long long B = blockIdx.x;
	double acc[16];
	#pragma unroll
	for (int e = 0; e < 16; ++e) acc[e] = 0.0;
	for (int k = offsets[B]+threadIdx.x; k < offsets[B+1]; k += blockDim.x) {
		const int fb = order[k];
		const double* mr = fine_mask+4*(size_t)block_row[fb];
		const double* mc = fine_mask+4*(size_t)fine_cols[fb];
		const T* v = fine_values+(size_t)fb*16;
		#pragma unroll
		for (int e = 0; e < 16; ++e) acc[e] += mr[e >> 2]*mc[e & 3]*(double)v[e];
	}
	__shared__ double red[16][129];
	#pragma unroll
	for (int e = 0; e < 16; ++e) red[e][threadIdx.x] = acc[e];
	__syncthreads();
	for (int stride = 64; stride > 0; stride >>= 1) {
		if ((int)threadIdx.x < stride)
			#pragma unroll
			for (int e = 0; e < 16; ++e) red[e][threadIdx.x] += red[e][threadIdx.x+stride];
		__syncthreads();
	}
	if (threadIdx.x < 16) coarse_values[B*16+threadIdx.x] = red[threadIdx.x][0];
}

// Masked-out coarse DOFs are decoupled: unit diagonal.
__global__ void UnitDiagonalKernel(int nodes, const int32_t* __restrict__ diag, const double* __restrict__ mask,
	double* __restrict__ values)
{
	const int i = blockIdx.x*blockDim.x+threadIdx.x;
	if (i >= 4*nodes) return;
	const int node = i >> 2, c = i & 3;
	if (mask[i] == 0.0) values[(size_t)diag[node]*16+c*4+c] = 1.0;
}

// (A P)[i, I] = sum over the fine blocks (i, j) with j in aggregate I of
// A[i, j] diag(mask_j): a warp per A P block, lanes = (slot, entry), fixed
// order (deterministic); summed in FP64, stored in the fine matrix's precision.
template <class T>
__global__ void __launch_bounds__(256) ApKernel(long long ap_blocks, const int32_t* __restrict__ order,
	const int32_t* __restrict__ offsets, const int32_t* __restrict__ fine_cols, const double* __restrict__ mask,
	const T* __restrict__ values, T* __restrict__ ap)
{
	const long long B = ((long long)blockIdx.x*blockDim.x+threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (B >= ap_blocks) return;
	const int e = lane & 15, slot = lane >> 4;
	double acc = 0.0;
	for (int k = offsets[B]+slot; k < offsets[B+1]; k += 2) {
		const int fb = order[k];
		acc += mask[4*(size_t)fine_cols[fb]+(e & 3)]*(double)values[(size_t)fb*16+e];
	}
	acc += __shfl_xor_sync(0xffffffffu, acc, 16);
	if (lane < 16) ap[B*16+lane] = T(acc);
}

template <class A> struct ApRow;
template <> struct ApRow<double> {
	static __device__ __forceinline__ void Load(const double* p, double v[4])
	{
		const double2 a01 = reinterpret_cast<const double2*>(p)[0], a23 = reinterpret_cast<const double2*>(p)[1];
		v[0] = a01.x; v[1] = a01.y; v[2] = a23.x; v[3] = a23.y;
	}
};
template <> struct ApRow<float> {
	static __device__ __forceinline__ void Load(const float* p, double v[4])
	{
		const float4 a = *reinterpret_cast<const float4*>(p);
		v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
	}
};

// The fine-level half of the two-level application, four threads per fine
// node (one per field row): t = P x_c (masked), r = b - (A P) x_c,
// z = t + omega D^{-1} r, the node's four residual entries exchanged within
// the lane quad.  Equal to prolongation, residual and block-Jacobi step on the
// full operator, but it reads the few A P blocks of the row instead of the
// row of A.
template <class A>
__global__ void __launch_bounds__(256) CoarseCorrectionKernel(int nodes, const int32_t* __restrict__ agg,
	const double* __restrict__ mask, const double* __restrict__ xc, const int32_t* __restrict__ ap_rows,
	const int32_t* __restrict__ ap_cols, const A* __restrict__ ap, const double* __restrict__ b,
	const double* __restrict__ inverse, double omega, double* __restrict__ z, const int* __restrict__ stop,
	const int32_t* __restrict__ node_seg, const int* __restrict__ seg_stop)
{
	if (*stop) return;
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	const int i = (int)(t >> 2), row = (int)(t & 3);
	// a node of a stopped segment takes no work (the lane quad stays together for the shuffles)
	const bool active = i < nodes && (seg_stop == nullptr || !seg_stop[node_seg[i]]);
	double r = 0.0;
	if (active) {
		r = b[t];
		for (int k = ap_rows[i]; k < ap_rows[i+1]; ++k) {
			double a[4];
			ApRow<A>::Load(ap+(size_t)k*16+row*4, a);
			const double2* xv = reinterpret_cast<const double2*>(xc+4*(size_t)ap_cols[k]);
			const double2 x01 = xv[0], x23 = xv[1];
			r -= a[0]*x01.x+a[1]*x01.y+a[2]*x23.x+a[3]*x23.y;
		}
	}
	const int base = threadIdx.x & ~3;
	const double r0 = __shfl_sync(0xffffffffu, r, base & 31), r1 = __shfl_sync(0xffffffffu, r, (base+1) & 31);
	const double r2 = __shfl_sync(0xffffffffu, r, (base+2) & 31), r3 = __shfl_sync(0xffffffffu, r, (base+3) & 31);
	if (!active) return;
	const double2* dinv = reinterpret_cast<const double2*>(inverse+(size_t)i*16+row*4);
	const double2 d01 = dinv[0], d23 = dinv[1];
	z[t] = mask[t]*xc[4*(size_t)agg[i]+row]+omega*(d01.x*r0+d01.y*r1+d23.x*r2+d23.y*r3);
}

// b_c[I,c] = sum_{i in I} mask_i[c] r[i,c]: one CTA per aggregate, fixed-order reduction.
__global__ void __launch_bounds__(128) RestrictKernel(int coarse_nodes, const int32_t* __restrict__ order,
	const int32_t* __restrict__ offsets, const double* __restrict__ mask, const double* __restrict__ r,
	double* __restrict__ bc, const int* __restrict__ stop, const int32_t* __restrict__ agg_seg,
	const int* __restrict__ seg_stop)
{
	if (*stop) return;
	const int I = blockIdx.x;
	if (seg_stop != nullptr && seg_stop[agg_seg[I]]) {
		if (threadIdx.x < 4) bc[4*I+threadIdx.x] = 0.0;   // a stopped segment's coarse rows
		return;
	}
	double acc[4] = {0.0, 0.0, 0.0, 0.0};
	for (int k = offsets[I]+threadIdx.x; k < offsets[I+1]; k += blockDim.x) {
		const size_t i = (size_t)order[k];
		const double2* m = reinterpret_cast<const double2*>(mask+4*i);
		const double2* v = reinterpret_cast<const double2*>(r+4*i);
		const double2 m01 = m[0], m23 = m[1], v01 = v[0], v23 = v[1];
		acc[0] += m01.x*v01.x; acc[1] += m01.y*v01.y; acc[2] += m23.x*v23.x; acc[3] += m23.y*v23.y;
	}
	__shared__ double red[4][129];
	for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = acc[c];
	__syncthreads();
	for (int stride = 64; stride > 0; stride >>= 1) {
		if ((int)threadIdx.x < stride)
			for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x+stride];
		__syncthreads();
	}
	if (threadIdx.x < 4) bc[4*I+threadIdx.x] = red[threadIdx.x][0];
}


__global__ void DenseScatterKernel(DevicePatternView p, const double* __restrict__ values, int n, double* __restrict__ dense)
{
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= p.blocks*16) return;
	const long long k = t >> 4;
	const int e = (int)(t & 15), r = e >> 2, c = e & 3;
	// row of block k: binary search in row offsets
	int lo = 0, hi = p.nodes;
	while (hi-lo > 1) {
		const int mid = (lo+hi)/2;
		if (p.row_offsets[mid] <= k) lo = mid; else hi = mid;
	}
	const size_t row = 4*(size_t)lo+r, col = 4*(size_t)p.columns[k]+c;
	dense[row*(size_t)(2*n)+col] = values[t];
}

// Gauss-Jordan inverse with partial pivoting on the augmented [A | I] (n x 2n,
// row-major), one pivot per pair of launches so every step uses the whole GPU:
// GaussJordanPivotKernel (one CTA) selects and swaps the pivot row, scales it
// and saves column k; GaussJordanEliminateKernel (grid) removes column k from
// every other row.  A vanishing pivot decouples its unknown (unit row) and
// raises *flag.
__global__ void AugmentIdentityKernel(int n, double* __restrict__ a)
{
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= (long long)n*n) return;
	const int i = (int)(t/n), j = (int)(t%n);
	a[(size_t)i*(2*n)+n+j] = i == j ? 1.0 : 0.0;
}

__global__ void __launch_bounds__(1024) GaussJordanPivotKernel(int n, int k, double* __restrict__ a,
	double* __restrict__ column, int* __restrict__ flag)
{
	const int ld = 2*n;
	__shared__ double best_val[32];
	__shared__ int best_idx[32];
	__shared__ int pivot_row;
	__shared__ double pivot_inv;
	double bv = -1.0; int bi = k;
	for (int i = k+threadIdx.x; i < n; i += blockDim.x) {
		const double v = fabs(a[(size_t)i*ld+k]);
		if (v > bv) { bv = v; bi = i; }
	}
	for (int o = 16; o > 0; o >>= 1) {
		const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
		const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
		if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
	}
	if ((threadIdx.x & 31) == 0) { best_val[threadIdx.x >> 5] = bv; best_idx[threadIdx.x >> 5] = bi; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double v = -1.0; int idx = k;
		for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
			if (best_val[w] > v) { v = best_val[w]; idx = best_idx[w]; }
		pivot_row = (v > 1e-300) ? idx : -1;
		if (pivot_row < 0) *flag = 1;
	}
	__syncthreads();
	const int pr = pivot_row;
	if (pr < 0) {
		for (int j = threadIdx.x; j < ld; j += blockDim.x) a[(size_t)k*ld+j] = (j == k || j == n+k) ? 1.0 : 0.0;
	} else if (pr != k) {
		for (int j = threadIdx.x; j < ld; j += blockDim.x) {
			const double t = a[(size_t)k*ld+j];
			a[(size_t)k*ld+j] = a[(size_t)pr*ld+j];
			a[(size_t)pr*ld+j] = t;
		}
	}
	__syncthreads();
	if (threadIdx.x == 0) pivot_inv = 1.0/a[(size_t)k*ld+k];
	__syncthreads();
	for (int j = threadIdx.x; j < ld; j += blockDim.x) a[(size_t)k*ld+j] *= pivot_inv;
	for (int i = threadIdx.x; i < n; i += blockDim.x) column[i] = i == k ? 0.0 : a[(size_t)i*ld+k];
}

__global__ void GaussJordanEliminateKernel(int n, int k, double* __restrict__ a, const double* __restrict__ column)
{
	const int ld = 2*n;
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= (long long)n*ld) return;
	const int i = (int)(t/ld), j = (int)(t%ld);
	const double f = column[i];
	if (f == 0.0) return;
	a[(size_t)i*ld+j] = j == k ? 0.0 : a[(size_t)i*ld+j]-f*a[(size_t)k*ld+j];
}

// Blocked Gauss-Jordan on the augmented [A | I] (n x 2n, row-major): 32 pivot columns per pair of
// launches instead of one.  For the panel of columns k0 .. k0 + b - 1 (b <= 32):
//   GaussJordanPanelKernel (one CTA): copies the panel's n x b columns twice (W, O), runs Gauss-Jordan
//     with partial pivoting on W alone (pivot rows searched below k0 + jj, swaps applied to W and O), so
//     that O ends up as the row-permuted original panel and the pivot block A_RR = O[k0 .. k0 + b) is
//     factorable in natural order; inverts A_RR in shared memory (Gauss-Jordan without further
//     pivoting: its pivots are the panel's) and records the swaps;
//   GaussJordanUpdateKernel (CTA per 16 columns of all 2n): applies the swaps, then
//     rows R = k0 .. k0 + b - 1  <-  Z = A_RR^{-1} Y_R,   every other row i  <-  Y_i - O_i Z,
//   which is what the b single-column eliminations do to those columns.
// A vanishing pivot (|max| <= 1e-300) raises *flag; the caller then redoes the inverse column by column.
constexpr int kPanelThreads = 1024;
constexpr int kUpdateColumns = 16;

__global__ void __launch_bounds__(kPanelThreads) GaussJordanPanelKernel(int n, int k0, int b,
	const double* __restrict__ a, double* __restrict__ panel, int* __restrict__ pivots, int* __restrict__ flag)
{
	const int ld = 2*n;
	double* W = panel;                      // [n][b]
	double* O = panel+(size_t)n*kPanel;     // [n][b]
	double* Ainv = panel+(size_t)2*n*kPanel; // [b][b]
	__shared__ double best_val[32];
	__shared__ int best_idx[32];
	__shared__ int pivot_row;
	__shared__ double pivot_value;
	__shared__ double block[kPanel][2*kPanel+1];
	const int tid = threadIdx.x;
	for (long long idx = tid; idx < (long long)n*b; idx += kPanelThreads) {
		const int i = (int)(idx/b), j = (int)(idx%b);
		const double v = a[(size_t)i*ld+k0+j];
		W[(size_t)i*b+j] = v;
		O[(size_t)i*b+j] = v;
	}
	__syncthreads();
	for (int jj = 0; jj < b; ++jj) {
		const int j = k0+jj;
		double bv = -1.0; int bi = j;
		for (int i = j+tid; i < n; i += kPanelThreads) {
			const double v = fabs(W[(size_t)i*b+jj]);
			if (v > bv) { bv = v; bi = i; }
		}
		for (int o = 16; o > 0; o >>= 1) {
			const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
			const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
			if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
		}
		if ((tid & 31) == 0) { best_val[tid >> 5] = bv; best_idx[tid >> 5] = bi; }
		__syncthreads();
		if (tid == 0) {
			double v = -1.0; int idx = j;
			for (int w = 0; w < kPanelThreads/32; ++w)
				if (best_val[w] > v || (best_val[w] == v && best_idx[w] < idx)) { v = best_val[w]; idx = best_idx[w]; }
			if (!(v > 1e-300)) { *flag = 1; idx = j; }
			pivot_row = idx;
			pivots[jj] = idx;
		}
		__syncthreads();
		const int pr = pivot_row;
		if (pr != j)
			for (int c = tid; c < b; c += kPanelThreads) {
				double t = W[(size_t)j*b+c]; W[(size_t)j*b+c] = W[(size_t)pr*b+c]; W[(size_t)pr*b+c] = t;
				t = O[(size_t)j*b+c]; O[(size_t)j*b+c] = O[(size_t)pr*b+c]; O[(size_t)pr*b+c] = t;
			}
		__syncthreads();
		if (tid == 0) {
			const double v = W[(size_t)j*b+jj];
			pivot_value = v != 0.0 ? v : 1.0;
		}
		__syncthreads();
		const double inv = 1.0/pivot_value;
		// eliminate column jj of the panel from every other row (row j scaled in place afterwards)
		for (long long idx = tid; idx < (long long)n*b; idx += kPanelThreads) {
			const int i = (int)(idx/b), c = (int)(idx%b);
			if (i == j || c <= jj) continue;
			const double f = W[(size_t)i*b+jj]*inv;
			if (f != 0.0) W[(size_t)i*b+c] -= f*W[(size_t)j*b+c];
		}
		__syncthreads();
		for (long long i = tid; i < n; i += kPanelThreads)
			if (i != j) W[(size_t)i*b+jj] = 0.0;
		for (int c = tid; c < b; c += kPanelThreads) W[(size_t)j*b+c] *= inv;
		__syncthreads();
	}
	// inverse of the pivot block A_RR = O[k0 .. k0 + b) by Gauss-Jordan in natural order
	for (int idx = tid; idx < b*2*b; idx += kPanelThreads) {
		const int r = idx/(2*b), c = idx%(2*b);
		block[r][c] = c < b ? O[(size_t)(k0+r)*b+c] : (c-b == r ? 1.0 : 0.0);
	}
	__syncthreads();
	for (int jj = 0; jj < b; ++jj) {
		if (tid == 0) {
			const double v = block[jj][jj];
			pivot_value = v != 0.0 ? v : 1.0;
		}
		__syncthreads();
		const double inv = 1.0/pivot_value;
		for (int idx = tid; idx < b*2*b; idx += kPanelThreads) {
			const int r = idx/(2*b), c = idx%(2*b);
			if (r == jj || c == jj) continue;
			const double f = block[r][jj]*inv;
			if (f != 0.0) block[r][c] -= f*block[jj][c];
		}
		__syncthreads();
		for (int r = tid; r < b; r += kPanelThreads) if (r != jj) block[r][jj] = 0.0;
		for (int c = tid; c < 2*b; c += kPanelThreads) block[jj][c] *= inv;
		__syncthreads();
	}
	for (int idx = tid; idx < b*b; idx += kPanelThreads) Ainv[idx] = block[idx/b][b+idx%b];
}

__global__ void __launch_bounds__(256) GaussJordanUpdateKernel(int n, int k0, int b, double* __restrict__ a,
	const double* __restrict__ panel, const int* __restrict__ pivots)
{
	const int ld = 2*n;
	const double* O = panel+(size_t)n*kPanel;
	const double* Ainv = panel+(size_t)2*n*kPanel;
	__shared__ double sA[kPanel][kPanel+1];
	__shared__ double sY[kPanel][kUpdateColumns];
	__shared__ double sZ[kPanel][kUpdateColumns];
	__shared__ int sP[kPanel];
	const int tid = threadIdx.x;
	const int c0 = blockIdx.x*kUpdateColumns;
	const int cols = min(kUpdateColumns, ld-c0);
	for (int idx = tid; idx < b*b; idx += blockDim.x) sA[idx/b][idx%b] = Ainv[idx];
	if (tid < b) sP[tid] = pivots[tid];
	__syncthreads();
	// the panel's row swaps, in order, one thread per column of the tile
	if (tid < cols)
		for (int jj = 0; jj < b; ++jj) {
			const int j = k0+jj, p = sP[jj];
			if (p != j) {
				const double t = a[(size_t)j*ld+c0+tid];
				a[(size_t)j*ld+c0+tid] = a[(size_t)p*ld+c0+tid];
				a[(size_t)p*ld+c0+tid] = t;
			}
		}
	__syncthreads();
	for (int idx = tid; idx < b*kUpdateColumns; idx += blockDim.x) {
		const int r = idx/kUpdateColumns, c = idx%kUpdateColumns;
		sY[r][c] = c < cols ? a[(size_t)(k0+r)*ld+c0+c] : 0.0;
	}
	__syncthreads();
	for (int idx = tid; idx < b*kUpdateColumns; idx += blockDim.x) {
		const int r = idx/kUpdateColumns, c = idx%kUpdateColumns;
		double z = 0.0;
		for (int k = 0; k < b; ++k) z = fma(sA[r][k], sY[k][c], z);
		sZ[r][c] = z;
		if (c < cols) a[(size_t)(k0+r)*ld+c0+c] = z;
	}
	__syncthreads();
	// every other row: Y_i -= O_i Z (threads: 16 columns x 16 row lanes)
	const int c = tid % kUpdateColumns, lane = tid / kUpdateColumns;
	if (c < cols)
		for (int i = lane; i < n; i += blockDim.x/kUpdateColumns) {
			if (i >= k0 && i < k0+b) continue;
			const double* o = O+(size_t)i*b;
			double s = 0.0;
			for (int k = 0; k < b; ++k) s = fma(o[k], sZ[k][c], s);
			a[(size_t)i*ld+c0+c] -= s;
		}
}

// x = A^{-1} b with the inverse in the right half of the augmented matrix; warp per row.
__global__ void DenseApplyKernel(int n, const double* __restrict__ a, const double* __restrict__ b,
	double* __restrict__ x, const int* __restrict__ stop)
{
	if (*stop) return;
	const int row = blockIdx.x*(blockDim.x >> 5)+(threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (row >= n) return;
	const double* ar = a+(size_t)row*(2*n)+n;
	double s = 0.0;
	for (int j = lane; j < n; j += 32) s = fma(ar[j], b[j], s);
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	if (lane == 0) x[row] = s;
}

} // namespace

Amg::Amg(const DevicePatternView& fine, const std::vector<int32_t>& row_offsets, const std::vector<int32_t>& columns,
	cudaStream_t stream, AmgOptions options)
	: fine_(fine), fine_rows_(row_offsets), fine_columns_(columns), stream_(stream), options_(options)
{
}

Amg::~Amg() = default;

std::vector<int> Amg::level_nodes() const
{
	std::vector<int> out;
	for (const auto& l : levels_) out.push_back(l->nodes);
	return out;
}

const double* Amg::fine_inverse() const
{
	return levels_.empty() ? nullptr : levels_[0]->inverse.get();
}

long long Amg::transfer_blocks() const
{
	return levels_.empty() ? 0 : levels_[0]->ap_blocks;
}

std::vector<long long> Amg::level_blocks() const
{
	std::vector<long long> out;
	for (const auto& l : levels_) out.push_back(l->blocks);
	return out;
}

void Amg::SetMasks(const std::vector<int32_t>& velocity_mask, const std::vector<int32_t>& pressure_mask)
{
	vmask_ = velocity_mask;
	pmask_ = pressure_mask;
	masks_dirty_ = true;
}

namespace {

// Vanek-style greedy aggregation on the symmetrised strength graph.
std::vector<int32_t> Aggregate(int nodes, const std::vector<int32_t>& rows, const std::vector<int32_t>& cols,
	const std::vector<int32_t>& diag, const std::vector<double>& s, double theta, int& coarse)
{
	// symmetrised strength: s_ij^sym = (s_ij + s_ji)/2
	std::vector<std::vector<int32_t>> strong(nodes);
	for (int i = 0; i < nodes; ++i) {
		const double sii = s[diag[i]];
		for (int k = rows[i]; k < rows[i+1]; ++k) {
			const int j = cols[k];
			if (j == i) continue;
			const auto it = std::lower_bound(cols.begin()+rows[j], cols.begin()+rows[j+1], i);
			const double sji = (it != cols.begin()+rows[j+1] && *it == i) ? s[it-cols.begin()] : 0.0;
			const double sij = 0.5*(s[k]+sji);
			const double sjj = s[diag[j]];
			if (sij >= theta*std::sqrt(sii*sjj) && sij > 0.0) strong[i].push_back(j);
		}
	}
	std::vector<int32_t> agg(nodes, -1);
	int count = 0;
	for (int i = 0; i < nodes; ++i) {           // phase 1: whole free neighbourhoods
		if (agg[i] >= 0 || strong[i].empty()) continue;
		bool free_nbhd = true;
		for (int j : strong[i]) if (agg[j] >= 0) { free_nbhd = false; break; }
		if (!free_nbhd) continue;
		agg[i] = count;
		for (int j : strong[i]) agg[j] = count;
		++count;
	}
	std::vector<int32_t> phase1 = agg;
	for (int i = 0; i < nodes; ++i) {           // phase 2: join a neighbouring phase-1 aggregate
		if (agg[i] >= 0) continue;
		for (int j : strong[i]) if (phase1[j] >= 0) { agg[i] = phase1[j]; break; }
	}
	for (int i = 0; i < nodes; ++i) {           // phase 3: the rest
		if (agg[i] >= 0) continue;
		agg[i] = count;
		for (int j : strong[i]) if (agg[j] < 0) agg[j] = count;
		++count;
	}
	coarse = count;
	return agg;
}

} // namespace

template <class T>
void Amg::Build(const T* values)
{
	std::vector<double> s(fine_.blocks);
	{
		DeviceArray<double> ds(fine_.blocks);
		StrengthKernel<T><<<Grid(fine_.blocks, 256), 256, 0, stream_>>>(fine_.blocks, values, ds.get());
		LaunchCheck("StrengthKernel");
		ds.Download(s.data(), s.size(), stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "AMG strength");
	}
	BuildFromStrength(std::move(s));
}

template void Amg::Build<double>(const double*);
template void Amg::Build<float>(const float*);

void Amg::BuildFromStrength(std::vector<double> s)
{
	levels_.clear();
	auto fine = std::make_unique<Level>();
	fine->nodes = fine_.nodes;
	fine->blocks = fine_.blocks;
	fine->h_rows = fine_rows_;
	fine->h_cols = fine_columns_;
	fine->h_diag.resize(fine_.nodes);
	for (int i = 0; i < fine_.nodes; ++i) {
		const auto it = std::lower_bound(fine_columns_.begin()+fine_rows_[i], fine_columns_.begin()+fine_rows_[i+1], i);
		fine->h_diag[i] = (int32_t)(it-fine_columns_.begin());
	}
	// Aggregate the strength graph repeatedly (aggregates of aggregates) until the
	// coarse space is small enough for a dense solve; compose the maps.
	std::vector<int32_t> compose(fine_.nodes);
	std::iota(compose.begin(), compose.end(), 0);
	std::vector<int32_t> rows = fine_rows_, cols = fine_columns_, diag = fine->h_diag;
	int nodes = fine_.nodes;
	for (int round = 0; round < options_.max_levels && nodes > options_.coarsest_nodes; ++round) {
		int nc = 0;
		const auto agg = Aggregate(nodes, rows, cols, diag, s, options_.strength, nc);
		if (nc >= (int)(0.9*nodes)) break;
		for (auto& c : compose) c = agg[c];
		// coarse strength graph = summed strengths
		std::vector<std::vector<std::pair<int32_t, double>>> crow(nc);
		for (int i = 0; i < nodes; ++i)
			for (int k = rows[i]; k < rows[i+1]; ++k) crow[agg[i]].push_back({agg[cols[k]], s[k]});
		std::vector<int32_t> nrows(nc+1, 0), ncols, ndiag(nc);
		std::vector<double> ns;
		for (int I = 0; I < nc; ++I) {
			auto& r = crow[I];
			std::sort(r.begin(), r.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
			for (size_t k = 0; k < r.size(); ++k) {
				if (!ncols.empty() && (int)ncols.size() > nrows[I] && ncols.back() == r[k].first) { ns.back() += r[k].second; continue; }
				if (r[k].first == I) ndiag[I] = (int32_t)ncols.size();
				ncols.push_back(r[k].first);
				ns.push_back(r[k].second);
			}
			nrows[I+1] = (int32_t)ncols.size();
		}
		rows.swap(nrows); cols.swap(ncols); diag.swap(ndiag); s.swap(ns);
		nodes = nc;
		coarse_history_.push_back(nc);
	}
	Level& L = *fine;
	L.h_agg = compose;
	const int nc = nodes;
	auto C = std::make_unique<Level>();
	C->nodes = nc;
	// coarse block pattern over the composite map and the fine-block -> coarse-block map
	std::vector<std::vector<int32_t>> crow(nc);
	for (int i = 0; i < L.nodes; ++i)
		for (int k = L.h_rows[i]; k < L.h_rows[i+1]; ++k) crow[compose[i]].push_back(compose[L.h_cols[k]]);
	C->h_rows.assign(nc+1, 0);
	for (int I = 0; I < nc; ++I) {
		auto& r = crow[I];
		std::sort(r.begin(), r.end());
		r.erase(std::unique(r.begin(), r.end()), r.end());
		C->h_rows[I+1] = C->h_rows[I]+(int32_t)r.size();
	}
	C->h_diag.resize(nc);
	for (int I = 0; I < nc; ++I) {
		const auto it = std::lower_bound(crow[I].begin(), crow[I].end(), I);
		C->h_diag[I] = C->h_rows[I]+(int32_t)(it-crow[I].begin());
		C->h_cols.insert(C->h_cols.end(), crow[I].begin(), crow[I].end());
	}
	C->blocks = C->h_rows[nc];
	std::vector<int32_t> target(L.blocks), block_row(L.blocks);
	for (int i = 0; i < L.nodes; ++i) {
		const int I = compose[i];
		for (int k = L.h_rows[i]; k < L.h_rows[i+1]; ++k) {
			const int J = compose[L.h_cols[k]];
			const auto it = std::lower_bound(C->h_cols.begin()+C->h_rows[I], C->h_cols.begin()+C->h_rows[I+1], J);
			target[k] = (int32_t)(it-C->h_cols.begin());
			block_row[k] = i;
		}
	}
	std::vector<int32_t> goff(C->blocks+1, 0), gorder(L.blocks);
	for (long long k = 0; k < L.blocks; ++k) ++goff[target[k]+1];
	for (long long B = 0; B < C->blocks; ++B) goff[B+1] += goff[B];
	{
		std::vector<int32_t> fill(goff.begin(), goff.end()-1);
		for (long long k = 0; k < L.blocks; ++k) gorder[fill[target[k]]++] = (int32_t)k;
	}
	// A P: per fine row, the distinct aggregates of its column nodes (sorted); every fine block
	// feeds exactly one A P block
	std::vector<int32_t> ap_rows(L.nodes+1, 0), ap_cols, ap_target(L.blocks);
	{
		std::vector<int32_t> row;
		for (int i = 0; i < L.nodes; ++i) {
			row.clear();
			for (int k = L.h_rows[i]; k < L.h_rows[i+1]; ++k) row.push_back(compose[L.h_cols[k]]);
			std::sort(row.begin(), row.end());
			row.erase(std::unique(row.begin(), row.end()), row.end());
			const int32_t base = (int32_t)ap_cols.size();
			ap_cols.insert(ap_cols.end(), row.begin(), row.end());
			ap_rows[i+1] = (int32_t)ap_cols.size();
			for (int k = L.h_rows[i]; k < L.h_rows[i+1]; ++k)
				ap_target[k] = base+(int32_t)(std::lower_bound(row.begin(), row.end(), compose[L.h_cols[k]])-row.begin());
		}
	}
	L.ap_blocks = (long long)ap_cols.size();
	std::vector<int32_t> apoff(L.ap_blocks+1, 0), aporder(L.blocks);
	for (long long k = 0; k < L.blocks; ++k) ++apoff[ap_target[k]+1];
	for (long long B = 0; B < L.ap_blocks; ++B) apoff[B+1] += apoff[B];
	{
		std::vector<int32_t> fill(apoff.begin(), apoff.end()-1);
		for (long long k = 0; k < L.blocks; ++k) aporder[fill[ap_target[k]]++] = (int32_t)k;
	}
	std::vector<int32_t> aoff(nc+1, 0), aorder(L.nodes);
	for (int i = 0; i < L.nodes; ++i) ++aoff[compose[i]+1];
	for (int I = 0; I < nc; ++I) aoff[I+1] += aoff[I];
	{
		std::vector<int32_t> fill(aoff.begin(), aoff.end()-1);
		for (int i = 0; i < L.nodes; ++i) aorder[fill[compose[i]]++] = i;
	}
	auto up = [&](DeviceArray<int32_t>& d, const std::vector<int32_t>& h) { d.Allocate(h.size()); d.Upload(h.data(), h.size(), stream_); };
	up(L.agg, L.h_agg); up(L.agg_order, aorder); up(L.agg_offsets, aoff);
	up(L.gal_order, gorder); up(L.gal_offsets, goff); up(L.block_row, block_row);
	up(L.ap_rows, ap_rows); up(L.ap_cols, ap_cols); up(L.ap_order, aporder); up(L.ap_offsets, apoff);
	// A P storage follows the fine matrix's precision; allocated on the first refresh
	levels_.push_back(std::move(fine));
	levels_.push_back(std::move(C));
	if (nc > 2048) Fail(-7, "aggregation stalled: coarse space of "+std::to_string(nc)+" nodes is too large for the dense coarse solve");
	for (size_t l = 0; l < levels_.size(); ++l) {
		Level& V = *levels_[l];
		up(V.rows, V.h_rows); up(V.cols, V.h_cols); up(V.diag, V.h_diag);
		if (l > 0) V.values.Allocate((size_t)V.blocks*16);
		V.inverse.Allocate((size_t)V.nodes*16);
		V.singular.Allocate(1);
		V.mask.Allocate((size_t)4*V.nodes);
		V.x.Allocate((size_t)4*V.nodes); V.b.Allocate((size_t)4*V.nodes); V.r.Allocate((size_t)4*V.nodes);
		if (l+1 == levels_.size()) {
			V.dense_n = 4*V.nodes;
			V.dense.Allocate((size_t)V.dense_n*2*V.dense_n);
			V.column.Allocate((size_t)V.dense_n);
			V.dense_flag.Allocate(1);
			V.panel.Allocate((size_t)2*V.dense_n*kPanel+kPanel*kPanel);
			V.pivots.Allocate(kPanel);
		}
	}
	CudaCheck(cudaStreamSynchronize(stream_), "AMG setup");
	built_ = true;
	BuildSegmentMaps();
	masks_dirty_ = true;
}

template <> double* Amg::ApValues<double>(Level& L)
{
	if (L.ap_values.size() == 0) L.ap_values.Allocate((size_t)L.ap_blocks*16);
	return L.ap_values.get();
}

template <> float* Amg::ApValues<float>(Level& L)
{
	if (L.ap_values32.size() == 0) L.ap_values32.Allocate((size_t)L.ap_blocks*16);
	return L.ap_values32.get();
}

template <class T>
void Amg::Refresh(const T* values, bool coarse)
{
	if (!built_) Fail(-1, "AMG hierarchy has not been built");
	if (masks_dirty_ || !coarse_ready_) coarse = true;
	if (masks_dirty_) {
		std::vector<double> m(4*(size_t)levels_[0]->nodes, 1.0);
		if (!vmask_.empty())
			for (int i = 0; i < levels_[0]->nodes; ++i) {
				if (vmask_[i]) m[4*i] = m[4*i+1] = m[4*i+2] = 0.0;
				if (!pmask_.empty() && pmask_[i]) m[4*i+3] = 0.0;
			}
		for (size_t l = 0; l < levels_.size(); ++l) {
			Level& L = *levels_[l];
			L.h_mask = m;
			L.mask.Upload(m.data(), m.size(), stream_);
			if (l+1 < levels_.size()) {
				std::vector<double> mc(4*(size_t)levels_[l+1]->nodes, 0.0);
				for (int i = 0; i < L.nodes; ++i)
					for (int c = 0; c < 4; ++c)
						if (m[4*i+c] != 0.0) mc[4*(size_t)L.h_agg[i]+c] = 1.0;
				m.swap(mc);
			}
		}
		CudaCheck(cudaStreamSynchronize(stream_), "AMG masks");
		masks_dirty_ = false;
	}
	for (size_t l = 0; l+1 < levels_.size(); ++l) {
		Level& L = *levels_[l];
		Level& C = *levels_[l+1];
		if (coarse) {
			if (l == 0)
				GalerkinKernel<T><<<(unsigned)C.blocks, 128, 0, stream_>>>(C.blocks, L.gal_order.get(),
					L.gal_offsets.get(), L.block_row.get(), L.cols.get(), L.mask.get(), values, C.values.get());
			else
				GalerkinKernel<double><<<(unsigned)C.blocks, 128, 0, stream_>>>(C.blocks, L.gal_order.get(),
					L.gal_offsets.get(), L.block_row.get(), L.cols.get(), L.mask.get(), L.values.get(),
					C.values.get());
			LaunchCheck("GalerkinKernel");
			launches_ += 1;
		}
		if (l == 0) {
			T* ap = ApValues<T>(L);
			ApKernel<T><<<Grid(L.ap_blocks, 8), 256, 0, stream_>>>(L.ap_blocks, L.ap_order.get(), L.ap_offsets.get(),
				L.cols.get(), L.mask.get(), values, ap);
			LaunchCheck("ApKernel");
			launches_ += 1;
		}
		if (coarse) {
			UnitDiagonalKernel<<<Grid(4LL*C.nodes, 256), 256, 0, stream_>>>(C.nodes, C.diag.get(), C.mask.get(),
				C.values.get());
			LaunchCheck("UnitDiagonalKernel");
			launches_ += 1;
		}
	}
	for (size_t l = 0; l+1 < levels_.size(); ++l) {
		Level& L = *levels_[l];
		L.singular.Zero(stream_);
		if (l == 0) LaunchBlockInverse<T>(L.view(), values, L.inverse.get(), L.singular.get(), stream_);
		else LaunchBlockInverse<double>(L.view(), L.values.get(), L.inverse.get(), L.singular.get(), stream_);
		launches_ += 1;
	}
	Level& Z = *levels_.back();
	if (Z.dense_n == 0 || !coarse) return;
	coarse_ready_ = true;
	Z.dense.Zero(stream_);
	Z.dense_flag.Zero(stream_);
	DenseScatterKernel<<<Grid(Z.blocks*16, 256), 256, 0, stream_>>>(Z.view(), Z.values.get(), Z.dense_n, Z.dense.get());
	LaunchCheck("DenseScatterKernel");
	const int dn = Z.dense_n;
	AugmentIdentityKernel<<<Grid((long long)dn*dn, 256), 256, 0, stream_>>>(dn, Z.dense.get());
	LaunchCheck("AugmentIdentityKernel");
	launches_ += 2;
	for (int k0 = 0; k0 < dn; k0 += kPanel) {
		const int b = std::min(kPanel, dn-k0);
		GaussJordanPanelKernel<<<1, kPanelThreads, 0, stream_>>>(dn, k0, b, Z.dense.get(), Z.panel.get(),
			Z.pivots.get(), Z.dense_flag.get());
		GaussJordanUpdateKernel<<<Grid(2LL*dn, kUpdateColumns), 256, 0, stream_>>>(dn, k0, b, Z.dense.get(),
			Z.panel.get(), Z.pivots.get());
		launches_ += 2;
	}
	LaunchCheck("GaussJordanUpdateKernel");
	// a vanishing panel pivot: redo the inverse one column at a time (that path decouples the unknown)
	int flag = 0;
	Z.dense_flag.Download(&flag, 1, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "AMG coarse inverse");
	if (flag == 0) return;
	Z.dense.Zero(stream_);
	Z.dense_flag.Zero(stream_);
	DenseScatterKernel<<<Grid(Z.blocks*16, 256), 256, 0, stream_>>>(Z.view(), Z.values.get(), Z.dense_n, Z.dense.get());
	AugmentIdentityKernel<<<Grid((long long)dn*dn, 256), 256, 0, stream_>>>(dn, Z.dense.get());
	for (int k = 0; k < dn; ++k) {
		GaussJordanPivotKernel<<<1, 1024, 0, stream_>>>(dn, k, Z.dense.get(), Z.column.get(), Z.dense_flag.get());
		GaussJordanEliminateKernel<<<Grid((long long)dn*2*dn, 256), 256, 0, stream_>>>(dn, k, Z.dense.get(),
			Z.column.get());
	}
	LaunchCheck("GaussJordanEliminateKernel");
	launches_ += 2+2LL*dn;
}

template void Amg::Refresh<double>(const double*, bool);
template void Amg::Refresh<float>(const float*, bool);

template <class T>
void Amg::Cycle(int l, const T* A, const double* b, double* x, const int* stop, const int* seg_stop)
{
	// Two-level: x_c = Ac^{-1} P^T b, then x = P x_c + omega D^{-1} (b - (A P) x_c).
	Level& L = *levels_[l];
	Level& C = *levels_[l+1];
	const bool masked = seg_stop != nullptr && segment_maps_ && l == 0;
	RestrictKernel<<<C.nodes, 128, 0, stream_>>>(C.nodes, L.agg_order.get(), L.agg_offsets.get(),
		L.mask.get(), b, C.b.get(), stop, masked ? aggregate_segment_dev_.get() : nullptr, masked ? seg_stop : nullptr);
	LaunchCheck("RestrictKernel");
	DenseApplyKernel<<<Grid(C.dense_n, 8), 256, 0, stream_>>>(C.dense_n, C.dense.get(), C.b.get(), C.x.get(), stop);
	LaunchCheck("DenseApplyKernel");
	(void)A;      // the fine operator enters through A P, refreshed with it
	CoarseCorrectionKernel<T><<<Grid(4LL*L.nodes, 256), 256, 0, stream_>>>(L.nodes, L.agg.get(), L.mask.get(),
		C.x.get(), L.ap_rows.get(), L.ap_cols.get(), ApValues<T>(L), b, L.inverse.get(), options_.omega, x, stop,
		masked ? node_segment_dev_.get() : nullptr, masked ? seg_stop : nullptr);
	LaunchCheck("CoarseCorrectionKernel");
	launches_ += 3;
}

template <class T>
void Amg::Apply(const T* fine_values, const double* v, double* z, const int* stop, const int* seg_stop)
{
	if (profiler_) profiler_->Begin(Profiler::kOther, stream_);
	Cycle<T>(0, fine_values, v, z, stop, seg_stop);
	if (profiler_) profiler_->End(stream_);
}

template void Amg::Apply<double>(const double*, const double*, double*, const int*, const int*);
template void Amg::Apply<float>(const float*, const double*, double*, const int*, const int*);

void Amg::SetSegments(const std::vector<int32_t>& node_segment)
{
	node_segment_ = node_segment;
	segment_maps_ = false;
	if (built_) BuildSegmentMaps();
}

// Device maps of the masked application: each fine node's segment, and each level-1 aggregate's
// (taken from any of its nodes; aggregates never cross segments, the matrix having no coupling
// between them).
void Amg::BuildSegmentMaps()
{
	segment_maps_ = false;
	if (node_segment_.empty() || levels_.size() < 2) return;
	const Level& L = *levels_[0];
	if ((int)node_segment_.size() != L.nodes) Fail(-1, "AMG segment map does not match the fine level");
	std::vector<int32_t> agg_seg(levels_[1]->nodes, -1);
	for (int i = 0; i < L.nodes; ++i) {
		const int32_t I = L.h_agg[i];
		if (agg_seg[I] < 0) agg_seg[I] = node_segment_[i];
		else if (agg_seg[I] != node_segment_[i]) Fail(-1, "an AMG aggregate spans two segments");
	}
	for (auto& v : agg_seg) if (v < 0) v = 0;
	node_segment_dev_.Allocate(node_segment_.size());
	node_segment_dev_.Upload(node_segment_.data(), node_segment_.size(), stream_);
	aggregate_segment_dev_.Allocate(agg_seg.size());
	aggregate_segment_dev_.Upload(agg_seg.data(), agg_seg.size(), stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "AMG segment maps");
	segment_maps_ = true;
}

} // namespace tfiga
