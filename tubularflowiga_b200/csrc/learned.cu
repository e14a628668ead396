// Learned FGMRES preconditioner stage (see learned.hpp): graph setup on the
// host, forward / backward / Adam kernels on the device.
#include "learned.hpp"
#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <random>
#include <tuple>

namespace tfiga {
namespace {

constexpr int H = LearnedPreconditioner::kHidden;
constexpr int kIn = LearnedPreconditioner::kInputs;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads/32;
constexpr int kChunk = 256;                 // elements per weight-gradient partial
// act(v) = v for v > 0, slope v otherwise (slope 0.1; slope 1 makes the network linear).
__device__ __forceinline__ float Act(float v, float slope) { return v > 0.f ? v : slope*v; }
__device__ __forceinline__ float DAct(float v, float slope) { return v > 0.f ? 1.f : slope; }
__device__ __forceinline__ float ToF(float v) { return v; }
__device__ __forceinline__ float ToF(__nv_bfloat16 v) { return __bfloat162float(v); }

unsigned Grid(long long n, int per) { return (unsigned)((n+per-1)/per); }

// X[e][4a + c] = s_in[c] x[4 conn[e][a] + c] (zero for padded a); thread per (element, a).
__global__ void GatherKernel(long long E, const int32_t* __restrict__ conn, const double* __restrict__ x,
	const double* __restrict__ scales, float* __restrict__ X, const int* __restrict__ stop)
{
	if (stop != nullptr && *stop) return;
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= E*64) return;
	const int node = conn[t];
	float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
	if (node >= 0) {
		const double* xv = x+4*(size_t)node;
		v = make_float4((float)(scales[0]*xv[0]), (float)(scales[1]*xv[1]), (float)(scales[2]*xv[2]),
			(float)(scales[3]*xv[3]));
	}
	reinterpret_cast<float4*>(X)[t] = v;
}

// h0 = act(X Win^T + bin): a warp per element, lane j -> outputs j, j + 32; Win transposed in shared memory.
template <class W>
__global__ void __launch_bounds__(kThreads) EncodeKernel(long long E, const float* __restrict__ X,
	const W* __restrict__ Win, const W* __restrict__ bin, float* __restrict__ z0, float* __restrict__ h0,
	float slope, const int* __restrict__ stop)
{
	if (stop != nullptr && *stop) return;
	extern __shared__ float sm[];
	float* WT = sm;                                    // [kIn][H]
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	float* xs = sm+kIn*H+warp*kIn;
	for (int idx = threadIdx.x; idx < H*kIn; idx += blockDim.x) WT[(idx%kIn)*H+idx/kIn] = ToF(Win[idx]);
	__syncthreads();
	const float b0 = ToF(bin[lane]), b1 = ToF(bin[lane+32]);
	for (long long e = (long long)blockIdx.x*kWarps+warp; e < E; e += (long long)gridDim.x*kWarps) {
		const float4* xr = reinterpret_cast<const float4*>(X+e*kIn);
		reinterpret_cast<float4*>(xs)[lane] = xr[lane];
		reinterpret_cast<float4*>(xs)[lane+32] = xr[lane+32];
		__syncwarp();
		float a0 = b0, a1 = b1;
		#pragma unroll 8
		for (int k = 0; k < kIn; ++k) {
			const float xk = xs[k];
			a0 = fmaf(WT[k*H+lane], xk, a0);
			a1 = fmaf(WT[k*H+lane+32], xk, a1);
		}
		if (z0 != nullptr) { z0[e*H+lane] = a0; z0[e*H+lane+32] = a1; }
		h0[e*H+lane] = Act(a0, slope);
		h0[e*H+lane+32] = Act(a1, slope);
		__syncwarp();
	}
}

// h_out = h + act(h Ws^T + mean_nb(h) Wn^T + b).
template <class W>
__global__ void __launch_bounds__(kThreads) LayerKernel(long long E, const int32_t* __restrict__ nb,
	const float* __restrict__ h, const W* __restrict__ Ws, const W* __restrict__ Wn, const W* __restrict__ b,
	float* __restrict__ m_out, float* __restrict__ z_out, float* __restrict__ h_out, float slope,
	const int* __restrict__ stop)
{
	if (stop != nullptr && *stop) return;
	extern __shared__ float sm[];
	float* WsT = sm;                                   // [H][H] transposed
	float* WnT = sm+H*H;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	float* hs = sm+2*H*H+warp*2*H;
	float* ms = hs+H;
	for (int idx = threadIdx.x; idx < H*H; idx += blockDim.x) {
		WsT[(idx%H)*H+idx/H] = ToF(Ws[idx]);
		WnT[(idx%H)*H+idx/H] = ToF(Wn[idx]);
	}
	__syncthreads();
	const float b0 = ToF(b[lane]), b1 = ToF(b[lane+32]);
	for (long long e = (long long)blockIdx.x*kWarps+warp; e < E; e += (long long)gridDim.x*kWarps) {
		const float h0 = h[e*H+lane], h1 = h[e*H+lane+32];
		float m0 = 0.f, m1 = 0.f;
		int cnt = 0;
		#pragma unroll
		for (int f = 0; f < 6; ++f) {
			const int n2 = nb[e*6+f];
			if (n2 >= 0) { m0 += h[(long long)n2*H+lane]; m1 += h[(long long)n2*H+lane+32]; ++cnt; }
		}
		if (cnt > 0) { m0 /= (float)cnt; m1 /= (float)cnt; }
		hs[lane] = h0; hs[lane+32] = h1; ms[lane] = m0; ms[lane+32] = m1;
		if (m_out != nullptr) { m_out[e*H+lane] = m0; m_out[e*H+lane+32] = m1; }
		__syncwarp();
		float a0 = b0, a1 = b1;
		#pragma unroll 8
		for (int k = 0; k < H; ++k) {
			const float hk = hs[k], mk = ms[k];
			a0 = fmaf(WsT[k*H+lane], hk, fmaf(WnT[k*H+lane], mk, a0));
			a1 = fmaf(WsT[k*H+lane+32], hk, fmaf(WnT[k*H+lane+32], mk, a1));
		}
		if (z_out != nullptr) { z_out[e*H+lane] = a0; z_out[e*H+lane+32] = a1; }
		h_out[e*H+lane] = h0+Act(a0, slope);
		h_out[e*H+lane+32] = h1+Act(a1, slope);
		__syncwarp();
	}
}

// y = h Wout^T + bout: lane -> outputs lane + 32 q.
template <class W>
__global__ void __launch_bounds__(kThreads) DecodeKernel(long long E, const float* __restrict__ h,
	const W* __restrict__ Wout, const W* __restrict__ bout, float* __restrict__ y, const int* __restrict__ stop)
{
	if (stop != nullptr && *stop) return;
	extern __shared__ float sm[];
	float* WoT = sm;                                   // [H][kIn] transposed
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	float* hs = sm+H*kIn+warp*H;
	for (int idx = threadIdx.x; idx < kIn*H; idx += blockDim.x) WoT[(idx%H)*kIn+idx/H] = ToF(Wout[idx]);
	__syncthreads();
	float bias[8];
	#pragma unroll
	for (int q = 0; q < 8; ++q) bias[q] = ToF(bout[lane+32*q]);
	for (long long e = (long long)blockIdx.x*kWarps+warp; e < E; e += (long long)gridDim.x*kWarps) {
		hs[lane] = h[e*H+lane]; hs[lane+32] = h[e*H+lane+32];
		__syncwarp();
		float acc[8];
		#pragma unroll
		for (int q = 0; q < 8; ++q) acc[q] = bias[q];
		for (int k = 0; k < H; ++k) {
			const float hk = hs[k];
			#pragma unroll
			for (int q = 0; q < 8; ++q) acc[q] = fmaf(WoT[k*kIn+lane+32*q], hk, acc[q]);
		}
		#pragma unroll
		for (int q = 0; q < 8; ++q) y[e*kIn+lane+32*q] = acc[q];
		__syncwarp();
	}
}

// out[4i + c] (+)= s_out[c] / deg(i) sum over the node's (element, a) entries of y; thread per (node, field).
__global__ void NodeOutKernel(int nodes, const int32_t* __restrict__ offsets, const int32_t* __restrict__ entries,
	const float* __restrict__ y, const double* __restrict__ scales, double* __restrict__ out, int accumulate,
	const int* __restrict__ stop)
{
	if (stop != nullptr && *stop) return;
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= 4LL*nodes) return;
	const int i = (int)(t >> 2), c = (int)(t & 3);
	const int lo = offsets[i], hi = offsets[i+1];
	float s = 0.f;
	for (int k = lo; k < hi; ++k) s += y[(size_t)entries[k]*4+c];
	const double v = hi > lo ? scales[4+c]*(double)s/(double)(hi-lo) : 0.0;
	out[t] = accumulate ? out[t]+v : v;
}

// Loss sum w_c (o - t)^2 / (4n) (block partials) and dL/do scaled by s_out / deg (the transpose of NodeOut).
__global__ void __launch_bounds__(kThreads) LossKernel(int nodes, const int32_t* __restrict__ offsets,
	const double* __restrict__ o, const double* __restrict__ target, const double* __restrict__ scales,
	float* __restrict__ node_do, double* __restrict__ partial)
{
	__shared__ double red[kWarps];
	const long long n4 = 4LL*nodes;
	double sq = 0.0;
	for (long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x; t < n4; t += (long long)gridDim.x*blockDim.x) {
		const int c = (int)(t & 3), i = (int)(t >> 2);
		const double d = o[t]-target[t];
		const double w = scales[8+c];
		sq += w*d*d;
		const int deg = offsets[i+1]-offsets[i];
		node_do[t] = deg > 0 ? (float)(2.0*w*d/(double)n4*scales[4+c]/(double)deg) : 0.f;
	}
	for (int k = 16; k > 0; k >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, k);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
	__syncthreads();
	if (threadIdx.x == 0) {
		double s = 0.0;
		for (int w = 0; w < kWarps; ++w) s += red[w];
		partial[blockIdx.x] = s;
	}
}

__global__ void LossFinalizeKernel(int count, const double* __restrict__ partial, double scale, double* __restrict__ out)
{
	__shared__ double red[kWarps];
	double s = 0.0;
	for (int i = threadIdx.x; i < count; i += blockDim.x) s += partial[i];
	for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < kWarps; ++w) t += red[w];
		*out = t*scale;
	}
}

// dy[e][4a + c] = node_do[4 conn[e][a] + c].
__global__ void DyGatherKernel(long long E, const int32_t* __restrict__ conn, const float* __restrict__ node_do,
	float* __restrict__ dy)
{
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= E*64) return;
	const int node = conn[t];
	float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
	if (node >= 0) v = reinterpret_cast<const float4*>(node_do)[node];
	reinterpret_cast<float4*>(dy)[t] = v;
}

// dh[e][k] = sum_o Wout[o][k] dy[e][o].
__global__ void __launch_bounds__(kThreads) DecodeBackKernel(long long E, const float* __restrict__ dy,
	const float* __restrict__ Wout, float* __restrict__ dh)
{
	extern __shared__ float sm[];
	float* Wo = sm;                                    // [kIn][H] natural
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	float* ds = sm+kIn*H+warp*kIn;
	for (int idx = threadIdx.x; idx < kIn*H; idx += blockDim.x) Wo[idx] = Wout[idx];
	__syncthreads();
	for (long long e = (long long)blockIdx.x*kWarps+warp; e < E; e += (long long)gridDim.x*kWarps) {
		const float4* dr = reinterpret_cast<const float4*>(dy+e*kIn);
		reinterpret_cast<float4*>(ds)[lane] = dr[lane];
		reinterpret_cast<float4*>(ds)[lane+32] = dr[lane+32];
		__syncwarp();
		float a0 = 0.f, a1 = 0.f;
		#pragma unroll 8
		for (int o = 0; o < kIn; ++o) {
			const float d = ds[o];
			a0 = fmaf(Wo[o*H+lane], d, a0);
			a1 = fmaf(Wo[o*H+lane+32], d, a1);
		}
		dh[e*H+lane] = a0;
		dh[e*H+lane+32] = a1;
		__syncwarp();
	}
}

// dz = dout act'(z); dprev = dout + Ws^T dz; dm = Wn^T dz / |nb(e)|.
__global__ void __launch_bounds__(kThreads) LayerBackKernel(long long E, const int32_t* __restrict__ nb,
	const float* __restrict__ dout, const float* __restrict__ z, const float* __restrict__ Ws,
	const float* __restrict__ Wn, float* __restrict__ dz, float* __restrict__ dprev, float* __restrict__ dm, float slope)
{
	extern __shared__ float sm[];
	float* S = sm;                                     // Ws [j][k] natural
	float* N = sm+H*H;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	float* zs = sm+2*H*H+warp*H;
	for (int idx = threadIdx.x; idx < H*H; idx += blockDim.x) { S[idx] = Ws[idx]; N[idx] = Wn[idx]; }
	__syncthreads();
	for (long long e = (long long)blockIdx.x*kWarps+warp; e < E; e += (long long)gridDim.x*kWarps) {
		const float d0 = dout[e*H+lane]*DAct(z[e*H+lane], slope);
		const float d1 = dout[e*H+lane+32]*DAct(z[e*H+lane+32], slope);
		zs[lane] = d0; zs[lane+32] = d1;
		dz[e*H+lane] = d0; dz[e*H+lane+32] = d1;
		int cnt = 0;
		#pragma unroll
		for (int f = 0; f < 6; ++f) cnt += nb[e*6+f] >= 0 ? 1 : 0;
		__syncwarp();
		float p0 = dout[e*H+lane], p1 = dout[e*H+lane+32], n0 = 0.f, n1 = 0.f;
		#pragma unroll 8
		for (int j = 0; j < H; ++j) {
			const float g = zs[j];
			p0 = fmaf(S[j*H+lane], g, p0); p1 = fmaf(S[j*H+lane+32], g, p1);
			n0 = fmaf(N[j*H+lane], g, n0); n1 = fmaf(N[j*H+lane+32], g, n1);
		}
		dprev[e*H+lane] = p0; dprev[e*H+lane+32] = p1;
		const float inv = cnt > 0 ? 1.f/(float)cnt : 0.f;
		dm[e*H+lane] = n0*inv; dm[e*H+lane+32] = n1*inv;
		__syncwarp();
	}
}

// dh[e] = dprev[e] + sum over the neighbours e' of e of dm[e'] (the adjacency is symmetric).
__global__ void NeighbourGatherKernel(long long E, const int32_t* __restrict__ nb, const float* __restrict__ dprev,
	const float* __restrict__ dm, float* __restrict__ dh)
{
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= E*H) return;
	const long long e = t/H;
	const int k = (int)(t%H);
	float s = dprev[t];
	#pragma unroll
	for (int f = 0; f < 6; ++f) {
		const int n2 = nb[e*6+f];
		if (n2 >= 0) s += dm[(long long)n2*H+k];
	}
	dh[t] = s;
}

__global__ void ActBackKernel(long long n, const float* __restrict__ dh, const float* __restrict__ z,
	float* __restrict__ dz, float slope)
{
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t < n) dz[t] = dh[t]*DAct(z[t], slope);
}

// partial[s][r][c] = sum over the elements of chunk s of A[e][r] B[e][c]; column C holds sum A[e][r].
// Block: 32 x 32 output tile, 256 threads x 4 outputs; chunk of kChunk elements staged 32 at a time.
__global__ void __launch_bounds__(kThreads) WeightGradKernel(long long E, const float* __restrict__ A, int R,
	const float* __restrict__ B, int C, float* __restrict__ partial)
{
	__shared__ float As[32][33], Bs[32][33];
	const int r0 = blockIdx.x*32, c0 = blockIdx.y*32;
	const long long e_lo = (long long)blockIdx.z*kChunk, e_hi = min(E, e_lo+kChunk);
	const int tr = threadIdx.x >> 3, tc = (threadIdx.x & 7)*4;
	float acc[4] = {0.f, 0.f, 0.f, 0.f}, bias = 0.f;
	for (long long e0 = e_lo; e0 < e_hi; e0 += 32) {
		for (int idx = threadIdx.x; idx < 32*32; idx += blockDim.x) {
			const int ee = idx >> 5, cc = idx & 31;
			const long long e = e0+ee;
			As[ee][cc] = e < e_hi ? A[e*R+r0+cc] : 0.f;
			Bs[ee][cc] = e < e_hi ? B[e*C+c0+cc] : 0.f;
		}
		__syncthreads();
		#pragma unroll 8
		for (int ee = 0; ee < 32; ++ee) {
			const float a = As[ee][tr];
			#pragma unroll
			for (int q = 0; q < 4; ++q) acc[q] = fmaf(a, Bs[ee][tc+q], acc[q]);
			bias += a;
		}
		__syncthreads();
	}
	float* out = partial+((size_t)blockIdx.z*R+r0+tr)*(C+1);
	#pragma unroll
	for (int q = 0; q < 4; ++q) out[c0+tc+q] = acc[q];
	if (blockIdx.y == 0 && tc == 0) out[C] = bias;
}

// grad[w_off + r C + c] = sum_s partial[s][r][c]; grad[b_off + r] = sum_s partial[s][r][C] (b_off >= 0).
__global__ void WeightGradReduceKernel(int chunks, int R, int C, const float* __restrict__ partial,
	float* __restrict__ grad, long long w_off, long long b_off)
{
	const int t = blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= R*(C+1)) return;
	const int r = t/(C+1), c = t%(C+1);
	if (c == C && b_off < 0) return;
	float s = 0.f;
	for (int k = 0; k < chunks; ++k) s += partial[((size_t)k*R+r)*(C+1)+c];
	if (c < C) grad[w_off+(long long)r*C+c] = s;
	else grad[b_off+r] = s;
}

__global__ void AdamKernel(long long n, float* __restrict__ theta, const float* __restrict__ g,
	float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= n) return;
	const float gt = g[t];
	const float mt = b1*m[t]+(1.f-b1)*gt, vt = b2*v[t]+(1.f-b2)*gt*gt;
	m[t] = mt; v[t] = vt;
	theta[t] -= lr*(mt/c1)/(sqrtf(vt/c2)+eps);
}

// Weighted inner products over one pair: partial sums of w_c o t and w_c o o (block partials).
__global__ void __launch_bounds__(kThreads) GainKernel(long long n4, const double* __restrict__ o,
	const double* __restrict__ t, const double* __restrict__ scales, double* __restrict__ partial)
{
	__shared__ double red[2][kWarps];
	double ot = 0.0, oo = 0.0;
	for (long long k = (long long)blockIdx.x*blockDim.x+threadIdx.x; k < n4; k += (long long)gridDim.x*blockDim.x) {
		const double w = scales[8+(k & 3)];
		ot += w*o[k]*t[k];
		oo += w*o[k]*o[k];
	}
	for (int s = 16; s > 0; s >>= 1) {
		ot += __shfl_xor_sync(0xffffffffu, ot, s);
		oo += __shfl_xor_sync(0xffffffffu, oo, s);
	}
	if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = ot; red[1][threadIdx.x >> 5] = oo; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double a = 0.0, b = 0.0;
		for (int w = 0; w < kWarps; ++w) { a += red[0][w]; b += red[1][w]; }
		partial[2*blockIdx.x] = a;
		partial[2*blockIdx.x+1] = b;
	}
}

// Krylov pair of the flexible GMRES (w = A z): x = D^{-1} w, t = z - M(w), q = w - A M(w) (skipped
// once the solve has stopped).
__global__ void KrylovPairKernel(long long n, const double* __restrict__ dinv_w, const double* __restrict__ z,
	const double* __restrict__ amg_w, const double* __restrict__ w, const double* __restrict__ a_amg_w,
	double* __restrict__ x, double* __restrict__ t, double* __restrict__ q, const int* __restrict__ stop)
{
	if (*stop) return;
	const long long k = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (k >= n) return;
	x[k] = dinv_w[k];
	t[k] = z[k]-amg_w[k];
	q[k] = w[k]-a_amg_w[k];
}

// Newton pair (J delta = b), scaled by 1 / |b|: x = D^{-1} b, t = delta - M(b), q = b - A M(b).
__global__ void SolvedPairKernel(long long n, const double* __restrict__ dinv_b, const double* __restrict__ delta,
	const double* __restrict__ amg_b, const double* __restrict__ b, const double* __restrict__ a_amg_b, double inv,
	double* __restrict__ x, double* __restrict__ t, double* __restrict__ q)
{
	const long long k = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (k >= n) return;
	x[k] = dinv_b[k]*inv;
	t[k] = (delta[k]-amg_b[k])*inv;
	q[k] = (b[k]-a_amg_b[k])*inv;
}

// Residual loss sum w_c (r - q)^2 / (4n) (block partials) and g = 2 w_c (r - q) / (4n).
__global__ void __launch_bounds__(kThreads) ResidualLossKernel(long long n4, const double* __restrict__ r,
	const double* __restrict__ q, const double* __restrict__ scales, double* __restrict__ g, double* __restrict__ partial)
{
	__shared__ double red[kWarps];
	double sq = 0.0;
	for (long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x; t < n4; t += (long long)gridDim.x*blockDim.x) {
		const double w = scales[8+(t & 3)];
		const double d = r[t]-q[t];
		sq += w*d*d;
		g[t] = 2.0*w*d/(double)n4;
	}
	for (int k = 16; k > 0; k >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, k);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
	__syncthreads();
	if (threadIdx.x == 0) {
		double s = 0.0;
		for (int w = 0; w < kWarps; ++w) s += red[w];
		partial[blockIdx.x] = s;
	}
}

// out += A^T v over the 4x4 block pattern: a warp per block row, FP64 atomics on the columns (training
// only; the summation order of the atomics varies from run to run).
template <class T>
__global__ void __launch_bounds__(256) TransposeSpmvKernel(DevicePatternView p, const T* __restrict__ values,
	const double* __restrict__ v, double* __restrict__ out)
{
	const int row = (int)(((long long)blockIdx.x*blockDim.x+threadIdx.x) >> 5);
	const int lane = threadIdx.x & 31;
	if (row >= p.nodes) return;
	const double v0 = v[4*(size_t)row], v1 = v[4*(size_t)row+1], v2 = v[4*(size_t)row+2], v3 = v[4*(size_t)row+3];
	for (int k = p.row_offsets[row]+lane; k < p.row_offsets[row+1]; k += 32) {
		const T* a = values+(size_t)k*16;
		double* o = out+4*(size_t)p.columns[k];
		#pragma unroll
		for (int c = 0; c < 4; ++c)
			atomicAdd(o+c, (double)a[c]*v0+(double)a[4+c]*v1+(double)a[8+c]*v2+(double)a[12+c]*v3);
	}
}

// node_do[4i + c] = g[4i + c] s_out[c] / deg(i) (the transpose of the node averaging).
__global__ void NodeDoKernel(int nodes, const int32_t* __restrict__ offsets, const double* __restrict__ g,
	const double* __restrict__ scales, float* __restrict__ node_do)
{
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t >= 4LL*nodes) return;
	const int i = (int)(t >> 2);
	const int deg = offsets[i+1]-offsets[i];
	node_do[t] = deg > 0 ? (float)(g[t]*scales[4+(t & 3)]/(double)deg) : 0.f;
}

__global__ void ToBf16Kernel(long long n, const float* __restrict__ in, __nv_bfloat16* __restrict__ out)
{
	const long long t = (long long)blockIdx.x*blockDim.x+threadIdx.x;
	if (t < n) out[t] = __float2bfloat16_rn(in[t]);
}

// Offsets of the flat parameter vector (the oracle's layout).
long long OffWin() { return 0; }
long long OffBin() { return (long long)H*kIn; }
long long OffLayer(int l) { return OffBin()+H+(long long)l*(2*H*H+H); }
long long OffWout(int layers) { return OffLayer(layers); }
long long OffBout(int layers) { return OffWout(layers)+(long long)kIn*H; }

constexpr size_t kEncodeSmem = sizeof(float)*(kIn*H+kWarps*kIn);
constexpr size_t kLayerSmem = sizeof(float)*(2*H*H+kWarps*2*H);
constexpr size_t kDecodeSmem = sizeof(float)*(H*kIn+kWarps*H);
constexpr size_t kDecodeBackSmem = sizeof(float)*(kIn*H+kWarps*kIn);
constexpr size_t kLayerBackSmem = sizeof(float)*(2*H*H+kWarps*H);

void ConfigureKernels()
{
	static bool done = false;
	if (done) return;
	CudaCheck(cudaFuncSetAttribute(EncodeKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEncodeSmem), "smem");
	CudaCheck(cudaFuncSetAttribute(EncodeKernel<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEncodeSmem), "smem");
	CudaCheck(cudaFuncSetAttribute(DecodeKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDecodeSmem), "smem");
	CudaCheck(cudaFuncSetAttribute(DecodeKernel<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDecodeSmem), "smem");
	CudaCheck(cudaFuncSetAttribute(DecodeBackKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDecodeBackSmem), "smem");
	CudaCheck(cudaFuncSetAttribute(LayerKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLayerSmem), "smem");
	CudaCheck(cudaFuncSetAttribute(LayerKernel<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLayerSmem), "smem");
	CudaCheck(cudaFuncSetAttribute(LayerBackKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLayerBackSmem), "smem");
	done = true;
}

unsigned PersistentGrid(long long E)
{
	return (unsigned)std::max<long long>(1, std::min<long long>(2*148, (E+kWarps-1)/kWarps));
}

} // namespace

// Face neighbours: two elements share a face when the four corner control points of one face of each
// coincide (after rounding to 1e-9 of the coordinate range).  Index of Bezier point (i, j, k): i + 4 j + 16 k.
static std::vector<int32_t> FaceNeighbours(const HostMesh& m)
{
	const long long E = m.elements();
	double scale = 0.0;
	for (double v : m.bezier_points) scale = std::max(scale, std::fabs(v));
	const double q = std::max(1e-9*scale, 1e-300);
	std::vector<int32_t> nb(6*E, -1);
	typedef std::tuple<long long, long long, long long> P3;
	std::map<std::vector<P3>, std::pair<long long, int>> open;
	for (long long e = 0; e < E; ++e) {
		const double* P = m.bezier_points.data()+e*192;
		for (int f = 0; f < 6; ++f) {
			const int axis = f/2, side = (f & 1) ? 3 : 0;
			const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
			std::vector<P3> key;
			for (int u : {0, 3})
				for (int v : {0, 3}) {
					int ijk[3];
					ijk[axis] = side; ijk[o1] = u; ijk[o2] = v;
					const int idx = ijk[0]+4*ijk[1]+16*ijk[2];
					key.emplace_back(std::llround(P[3*idx]/q), std::llround(P[3*idx+1]/q), std::llround(P[3*idx+2]/q));
				}
			std::sort(key.begin(), key.end());
			auto it = open.find(key);
			if (it == open.end()) open.emplace(std::move(key), std::make_pair(e, f));
			else {
				nb[6*e+f] = (int32_t)it->second.first;
				nb[6*it->second.first+it->second.second] = (int32_t)e;
				open.erase(it);
			}
		}
	}
	return nb;
}

LearnedPreconditioner::LearnedPreconditioner(const Mesh& mesh, int layers, unsigned long long seed,
	cudaStream_t stream, bool linear)
	: stream_(stream), layers_(layers), nodes_((int)mesh.nodes()), elements_(mesh.host().elements()),
	  linear_(linear), slope_(linear ? 1.f : 0.1f)
{
	if (layers < 1 || layers > kMaxLayers) Fail(-1, "learned preconditioner: layers must be in [1, 8]");
	const HostMesh& m = mesh.host();
	if (m.max_basis > 64) Fail(-7, "learned preconditioner: more than 64 basis functions per element");
	ConfigureKernels();
	const long long E = elements_;
	std::vector<int32_t> conn(64*E, -1);
	std::vector<int32_t> count(nodes_+1, 0);
	for (long long e = 0; e < E; ++e)
		for (int a = 0; a < m.element_offsets[e+1]-m.element_offsets[e]; ++a) {
			const int32_t node = m.connectivity[m.element_offsets[e]+a];
			conn[64*e+a] = node;
			++count[node+1];
		}
	for (int i = 0; i < nodes_; ++i) count[i+1] += count[i];
	std::vector<int32_t> entries(count[nodes_]);
	{
		std::vector<int32_t> fill(count.begin(), count.end()-1);
		for (long long e = 0; e < E; ++e)
			for (int a = 0; a < 64; ++a)
				if (conn[64*e+a] >= 0) entries[fill[conn[64*e+a]]++] = (int32_t)(64*e+a);
	}
	nb_host_ = FaceNeighbours(m);
	auto up = [&](DeviceArray<int32_t>& d, const std::vector<int32_t>& h) { d.Allocate(h.size()); d.Upload(h.data(), h.size(), stream_); };
	up(conn_, conn); up(nb_, nb_host_); up(node_offsets_, count); up(node_entries_, entries);

	params_ = OffBout(layers)+kIn;
	theta_.Allocate(params_); grad_.Allocate(params_); adam_m_.Allocate(params_); adam_v_.Allocate(params_);
	theta16_.Allocate(params_);
	adam_m_.Zero(stream_); adam_v_.Zero(stream_); grad_.Zero(stream_);
	const long long chunks = (E+kChunk-1)/kChunk;
	partial_.Allocate((size_t)chunks*kIn*(H+1) > (size_t)chunks*H*(kIn+1) ? (size_t)chunks*kIn*(H+1)
		: (size_t)chunks*H*(kIn+1));
	X_.Allocate((size_t)E*kIn); z0_.Allocate((size_t)E*H); y_.Allocate((size_t)E*kIn); dy_.Allocate((size_t)E*kIn);
	dh_.Allocate((size_t)E*H); dprev_.Allocate((size_t)E*H); dm_.Allocate((size_t)E*H); dz0_.Allocate((size_t)E*H);
	node_do_.Allocate(4*(size_t)nodes_);
	h_.resize(layers+1); m_.resize(layers); z_.resize(layers); dz_.resize(layers);
	for (auto& a : h_) a.Allocate((size_t)E*H);
	for (int l = 0; l < layers; ++l) { m_[l].Allocate((size_t)E*H); z_[l].Allocate((size_t)E*H); dz_[l].Allocate((size_t)E*H); }
	o_.Allocate(4*(size_t)nodes_);
	scales_.Allocate(12);
	loss_partial_.Allocate(2*148);
	loss_.Allocate(1);

	// Initial weights: normal, fan-in scaled; the decoder starts small so the stage starts near zero.
	std::mt19937_64 rng(seed);
	std::normal_distribution<float> normal(0.f, 1.f);
	std::vector<float> t(params_, 0.f);
	for (long long k = 0; k < (long long)H*kIn; ++k) t[OffWin()+k] = normal(rng)*std::sqrt(2.f/kIn);
	for (int l = 0; l < layers; ++l)
		for (long long k = 0; k < 2LL*H*H; ++k) t[OffLayer(l)+k] = normal(rng)*0.5f*std::sqrt(1.f/H);
	for (long long k = 0; k < (long long)kIn*H; ++k) t[OffWout(layers)+k] = normal(rng)*0.01f*std::sqrt(1.f/H);
	SetParameters(t.data());
	SetScales(scale_in_, scale_out_, weight_);
}

float* LearnedPreconditioner::param(const char* name, int layer)
{
	float* base = theta_.get();
	if (!std::strcmp(name, "Win")) return base+OffWin();
	if (!std::strcmp(name, "bin")) return base+OffBin();
	if (!std::strcmp(name, "Ws")) return base+OffLayer(layer);
	if (!std::strcmp(name, "Wn")) return base+OffLayer(layer)+H*H;
	if (!std::strcmp(name, "b")) return base+OffLayer(layer)+2*H*H;
	if (!std::strcmp(name, "Wout")) return base+OffWout(layers_);
	return base+OffBout(layers_);
}

void LearnedPreconditioner::SetParameters(const float* host)
{
	theta_.Upload(host, params_, stream_);
	bf16_dirty_ = true;
	CudaCheck(cudaStreamSynchronize(stream_), "learned parameters");
}

void LearnedPreconditioner::GetParameters(float* host) const
{
	theta_.Download(host, params_, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "learned parameters");
}

void LearnedPreconditioner::SetScales(const double in[4], const double out[4], const double weights[4])
{
	double s[12];
	for (int c = 0; c < 4; ++c) {
		if (!(in[c] > 0.0) || !(out[c] > 0.0) || !(weights[c] >= 0.0) || !std::isfinite(in[c]) || !std::isfinite(out[c]))
			Fail(-1, "learned preconditioner: scales must be positive and finite");
		scale_in_[c] = in[c]; scale_out_[c] = out[c]; weight_[c] = weights[c];
		s[c] = in[c]; s[4+c] = out[c]; s[8+c] = weights[c];
	}
	scales_.Upload(s, 12, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "learned scales");
}

void LearnedPreconditioner::GetScales(double in[4], double out[4], double weights[4]) const
{
	for (int c = 0; c < 4; ++c) { in[c] = scale_in_[c]; out[c] = scale_out_[c]; weights[c] = weight_[c]; }
}

void LearnedPreconditioner::SyncBf16()
{
	if (!bf16_dirty_) return;
	ToBf16Kernel<<<Grid(params_, 256), 256, 0, stream_>>>(params_, theta_.get(), theta16_.get());
	LaunchCheck("ToBf16Kernel");
	bf16_dirty_ = false;
}

void LearnedPreconditioner::Gather(const double* x)
{
	GatherKernel<<<Grid(elements_*64, 256), 256, 0, stream_>>>(elements_, conn_.get(), x, scales_.get(), X_.get(),
		nullptr);
	LaunchCheck("GatherKernel");
}

void LearnedPreconditioner::ForwardLayers(bool keep)
{
	const long long E = elements_;
	const unsigned grid = PersistentGrid(E);
	EncodeKernel<float><<<grid, kThreads, kEncodeSmem, stream_>>>(E, X_.get(), param("Win"), param("bin"),
		keep ? z0_.get() : nullptr, h_[0].get(), slope_, nullptr);
	LaunchCheck("EncodeKernel");
	for (int l = 0; l < layers_; ++l) {
		LayerKernel<float><<<grid, kThreads, kLayerSmem, stream_>>>(E, nb_.get(), h_[l].get(), param("Ws", l),
			param("Wn", l), param("b", l), keep ? m_[l].get() : nullptr, keep ? z_[l].get() : nullptr, h_[l+1].get(),
			slope_, nullptr);
		LaunchCheck("LayerKernel");
	}
	DecodeKernel<float><<<grid, kThreads, kDecodeSmem, stream_>>>(E, h_[layers_].get(), param("Wout"), param("bout"),
		y_.get(), nullptr);
	LaunchCheck("DecodeKernel");
}

void LearnedPreconditioner::Forward(const double* x, double* o)
{
	Gather(x);
	ForwardLayers(false);
	NodeOutKernel<<<Grid(4LL*nodes_, 256), 256, 0, stream_>>>(nodes_, node_offsets_.get(), node_entries_.get(),
		y_.get(), scales_.get(), o, 0, nullptr);
	LaunchCheck("NodeOutKernel");
}

void LearnedPreconditioner::Apply(const double* x, double* z, const int* stop)
{
	SyncBf16();
	const long long E = elements_;
	const unsigned grid = PersistentGrid(E);
	const __nv_bfloat16* t = theta16_.get();
	GatherKernel<<<Grid(E*64, 256), 256, 0, stream_>>>(E, conn_.get(), x, scales_.get(), X_.get(), stop);
	EncodeKernel<__nv_bfloat16><<<grid, kThreads, kEncodeSmem, stream_>>>(E, X_.get(), t+OffWin(), t+OffBin(), nullptr,
		h_[0].get(), slope_, stop);
	for (int l = 0; l < layers_; ++l)
		LayerKernel<__nv_bfloat16><<<grid, kThreads, kLayerSmem, stream_>>>(E, nb_.get(), h_[l & 1].get(),
			t+OffLayer(l), t+OffLayer(l)+H*H, t+OffLayer(l)+2*H*H, nullptr, nullptr, h_[(l+1) & 1].get(), slope_, stop);
	DecodeKernel<__nv_bfloat16><<<grid, kThreads, kDecodeSmem, stream_>>>(E, h_[layers_ & 1].get(), t+OffWout(layers_),
		t+OffBout(layers_), y_.get(), stop);
	NodeOutKernel<<<Grid(4LL*nodes_, 256), 256, 0, stream_>>>(nodes_, node_offsets_.get(), node_entries_.get(),
		y_.get(), scales_.get(), z, 1, stop);
	LaunchCheck("learned preconditioner");
}

void LearnedPreconditioner::SetOperator(const DevicePatternView& pattern, const float* values32,
	const double* values64)
{
	op_ = pattern;
	op32_ = values32;
	op64_ = values64;
	if (values32 != nullptr || values64 != nullptr) {
		if (ro_.size() == 0) { ro_.Allocate(4*(size_t)nodes_); g_.Allocate(4*(size_t)nodes_); atg_.Allocate(4*(size_t)nodes_); }
	}
}

void LearnedPreconditioner::ApplyOperator(const double* in, double* out)
{
	if (op32_ != nullptr) LaunchSpmv<float>(op_, op32_, in, out, stream_);
	else LaunchSpmv<double>(op_, op64_, in, out, stream_);
}

void LearnedPreconditioner::Backward()
{
	const long long E = elements_;
	const unsigned grid = PersistentGrid(E);
	DyGatherKernel<<<Grid(E*64, 256), 256, 0, stream_>>>(E, conn_.get(), node_do_.get(), dy_.get());
	LaunchCheck("DyGatherKernel");
	const int chunks = (int)((E+kChunk-1)/kChunk);
	auto weight_grad = [&](const float* A, int R, const float* B, int C, long long w_off, long long b_off) {
		WeightGradKernel<<<dim3(R/32, C/32, chunks), kThreads, 0, stream_>>>(E, A, R, B, C, partial_.get());
		WeightGradReduceKernel<<<Grid((long long)R*(C+1), 256), 256, 0, stream_>>>(chunks, R, C, partial_.get(),
			grad_.get(), w_off, b_off);
		LaunchCheck("WeightGradKernel");
	};
	weight_grad(dy_.get(), kIn, h_[layers_].get(), H, OffWout(layers_), OffBout(layers_));
	DecodeBackKernel<<<grid, kThreads, kDecodeBackSmem, stream_>>>(E, dy_.get(), param("Wout"), dh_.get());
	LaunchCheck("DecodeBackKernel");
	for (int l = layers_-1; l >= 0; --l) {
		LayerBackKernel<<<grid, kThreads, kLayerBackSmem, stream_>>>(E, nb_.get(), dh_.get(), z_[l].get(),
			param("Ws", l), param("Wn", l), dz_[l].get(), dprev_.get(), dm_.get(), slope_);
		LaunchCheck("LayerBackKernel");
		weight_grad(dz_[l].get(), H, h_[l].get(), H, OffLayer(l), OffLayer(l)+2*H*H);
		weight_grad(dz_[l].get(), H, m_[l].get(), H, OffLayer(l)+H*H, -1);
		NeighbourGatherKernel<<<Grid(E*H, 256), 256, 0, stream_>>>(E, nb_.get(), dprev_.get(), dm_.get(), dh_.get());
		LaunchCheck("NeighbourGatherKernel");
	}
	ActBackKernel<<<Grid(E*H, 256), 256, 0, stream_>>>(E*H, dh_.get(), z0_.get(), dz0_.get(), slope_);
	LaunchCheck("ActBackKernel");
	weight_grad(dz0_.get(), H, X_.get(), kIn, OffWin(), OffBin());
	if (linear_) {
		// a linear stage keeps its biases at zero
		CudaCheck(cudaMemsetAsync(grad_.get()+OffBin(), 0, sizeof(float)*H, stream_), "bias gradient");
		for (int l = 0; l < layers_; ++l)
			CudaCheck(cudaMemsetAsync(grad_.get()+OffLayer(l)+2*H*H, 0, sizeof(float)*H, stream_), "bias gradient");
		CudaCheck(cudaMemsetAsync(grad_.get()+OffBout(layers_), 0, sizeof(float)*kIn, stream_), "bias gradient");
	}
}

double LearnedPreconditioner::LossAndGradient(const double* x, const double* target)
{
	Gather(x);
	ForwardLayers(true);
	NodeOutKernel<<<Grid(4LL*nodes_, 256), 256, 0, stream_>>>(nodes_, node_offsets_.get(), node_entries_.get(),
		y_.get(), scales_.get(), o_.get(), 0, nullptr);
	LossKernel<<<2*148, kThreads, 0, stream_>>>(nodes_, node_offsets_.get(), o_.get(), target, scales_.get(),
		node_do_.get(), loss_partial_.get());
	LossFinalizeKernel<<<1, kThreads, 0, stream_>>>(2*148, loss_partial_.get(), 1.0/(4.0*nodes_), loss_.get());
	LaunchCheck("learned loss");
	Backward();
	double loss = 0.0;
	loss_.Download(&loss, 1, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "learned loss");
	return loss;
}

double LearnedPreconditioner::ResidualLossAndGradient(const double* x, const double* q)
{
	if (!has_operator()) Fail(-1, "learned preconditioner: no operator bound for the residual loss");
	const long long n4 = 4LL*nodes_;
	Gather(x);
	ForwardLayers(true);
	NodeOutKernel<<<Grid(n4, 256), 256, 0, stream_>>>(nodes_, node_offsets_.get(), node_entries_.get(), y_.get(),
		scales_.get(), o_.get(), 0, nullptr);
	ApplyOperator(o_.get(), ro_.get());
	ResidualLossKernel<<<2*148, kThreads, 0, stream_>>>(n4, ro_.get(), q, scales_.get(), g_.get(),
		loss_partial_.get());
	LossFinalizeKernel<<<1, kThreads, 0, stream_>>>(2*148, loss_partial_.get(), 1.0/(double)n4, loss_.get());
	atg_.Zero(stream_);
	if (op32_ != nullptr)
		TransposeSpmvKernel<float><<<Grid(32LL*op_.nodes, 256), 256, 0, stream_>>>(op_, op32_, g_.get(), atg_.get());
	else
		TransposeSpmvKernel<double><<<Grid(32LL*op_.nodes, 256), 256, 0, stream_>>>(op_, op64_, g_.get(), atg_.get());
	NodeDoKernel<<<Grid(n4, 256), 256, 0, stream_>>>(nodes_, node_offsets_.get(), atg_.get(), scales_.get(),
		node_do_.get());
	LaunchCheck("learned residual loss");
	Backward();
	double loss = 0.0;
	loss_.Download(&loss, 1, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "learned loss");
	return loss;
}

void LearnedPreconditioner::AddPair(const double* x, const double* target)
{
	AllocatePairs();
	const size_t n4 = 4*(size_t)nodes_;
	CudaCheck(cudaMemcpyAsync(pairs_x_.get()+(size_t)next_pair_*n4, x, n4*sizeof(double), cudaMemcpyDeviceToDevice,
		stream_), "training pair");
	CudaCheck(cudaMemcpyAsync(pairs_t_.get()+(size_t)next_pair_*n4, target, n4*sizeof(double),
		cudaMemcpyDeviceToDevice, stream_), "training pair");
	CudaCheck(cudaMemsetAsync(pairs_q_.get()+(size_t)next_pair_*n4, 0, n4*sizeof(double), stream_), "training pair");
	next_pair_ = (next_pair_+1)%capacity_;
	pair_count_ = std::min(pair_count_+1, capacity_);
}

void LearnedPreconditioner::SetCapacity(int capacity)
{
	if (capacity_ != 0) Fail(-1, "the learned stage's pair store is already allocated");
	if (capacity < 1) Fail(-1, "pair capacity must be positive");
	requested_capacity_ = capacity;
}

void LearnedPreconditioner::AllocatePairs()
{
	if (capacity_ != 0) return;
	capacity_ = requested_capacity_;
	for (auto* a : {&pairs_x_, &pairs_t_, &pairs_q_}) {
		a->Allocate((size_t)capacity_*4*nodes_);
		a->Zero(stream_);
	}
}

void LearnedPreconditioner::AddKrylovPair(const double* dinv_w, const double* z, const double* amg_w,
	const double* w, const double* a_amg_w, const int* stop)
{
	AllocatePairs();
	const size_t n4 = 4*(size_t)nodes_;
	KrylovPairKernel<<<Grid((long long)n4, 256), 256, 0, stream_>>>((long long)n4, dinv_w, z, amg_w, w, a_amg_w,
		pairs_x_.get()+(size_t)next_pair_*n4, pairs_t_.get()+(size_t)next_pair_*n4,
		pairs_q_.get()+(size_t)next_pair_*n4, stop);
	LaunchCheck("KrylovPairKernel");
	next_pair_ = (next_pair_+1)%capacity_;
	pair_count_ = std::min(pair_count_+1, capacity_);
}

void LearnedPreconditioner::AddSolvedPair(const double* dinv_b, const double* delta, const double* amg_b,
	const double* b, const double* a_amg_b, double b_norm)
{
	if (!(b_norm > 0.0) || !std::isfinite(b_norm)) return;
	AllocatePairs();
	const size_t n4 = 4*(size_t)nodes_;
	SolvedPairKernel<<<Grid((long long)n4, 256), 256, 0, stream_>>>((long long)n4, dinv_b, delta, amg_b, b, a_amg_b,
		1.0/b_norm, pairs_x_.get()+(size_t)next_pair_*n4, pairs_t_.get()+(size_t)next_pair_*n4,
		pairs_q_.get()+(size_t)next_pair_*n4);
	LaunchCheck("SolvedPairKernel");
	next_pair_ = (next_pair_+1)%capacity_;
	pair_count_ = std::min(pair_count_+1, capacity_);
}

void LearnedPreconditioner::FitScales()
{
	if (pair_count_ == 0) Fail(-1, "learned preconditioner: no training pairs");
	const size_t n4 = 4*(size_t)nodes_;
	std::vector<double> x(n4), t(n4), q(n4);
	double sx[4] = {0, 0, 0, 0}, st[4] = {0, 0, 0, 0}, sq[4] = {0, 0, 0, 0};
	for (int p = 0; p < pair_count_; ++p) {
		CudaCheck(cudaMemcpyAsync(x.data(), pairs_x_.get()+(size_t)p*n4, n4*sizeof(double), cudaMemcpyDeviceToHost,
			stream_), "training pairs");
		CudaCheck(cudaMemcpyAsync(t.data(), pairs_t_.get()+(size_t)p*n4, n4*sizeof(double), cudaMemcpyDeviceToHost,
			stream_), "training pairs");
		CudaCheck(cudaMemcpyAsync(q.data(), pairs_q_.get()+(size_t)p*n4, n4*sizeof(double), cudaMemcpyDeviceToHost,
			stream_), "training pairs");
		CudaCheck(cudaStreamSynchronize(stream_), "training pairs");
		for (size_t k = 0; k < n4; ++k) { sx[k & 3] += x[k]*x[k]; st[k & 3] += t[k]*t[k]; sq[k & 3] += q[k]*q[k]; }
	}
	double in[4], out[4], w[4];
	const double count = (double)pair_count_*nodes_;
	for (int c = 0; c < 4; ++c) {
		const double rx = std::sqrt(sx[c]/count), rt = std::sqrt(st[c]/count), rq = std::sqrt(sq[c]/count);
		const double rw = has_operator() ? rq : rt;      // the loss is on the residual when an operator is bound
		in[c] = rx > 0.0 ? 1.0/rx : 1.0;
		out[c] = rt > 0.0 ? rt : 1.0;
		w[c] = rw > 0.0 ? 1.0/(rw*rw) : 0.0;
	}
	SetScales(in, out, w);
}

double LearnedPreconditioner::PairLoss(int p, bool gradient)
{
	const size_t n4 = 4*(size_t)nodes_;
	const double* x = pairs_x_.get()+(size_t)p*n4;
	if (has_operator()) return ResidualLossAndGradient(x, pairs_q_.get()+(size_t)p*n4);
	(void)gradient;
	return LossAndGradient(x, pairs_t_.get()+(size_t)p*n4);
}

double LearnedPreconditioner::Train(int steps, double learning_rate)
{
	if (pair_count_ == 0) Fail(-1, "learned preconditioner: no training pairs");
	double last = 0.0;
	int in_pass = 0;
	for (int s = 0; s < steps; ++s) {
		const double l = PairLoss(s%pair_count_, true);
		if (!std::isfinite(l)) Fail(-6, "learned preconditioner: training loss is not finite");
		++adam_steps_;
		const float b1 = 0.9f, b2 = 0.999f;
		const float c1 = 1.f-std::pow(b1, (float)adam_steps_), c2 = 1.f-std::pow(b2, (float)adam_steps_);
		AdamKernel<<<Grid(params_, 256), 256, 0, stream_>>>(params_, theta_.get(), grad_.get(), adam_m_.get(),
			adam_v_.get(), (float)learning_rate, b1, b2, 1e-8f, c1, c2);
		LaunchCheck("AdamKernel");
		if (s >= steps-pair_count_) { last += l; ++in_pass; }
	}
	bf16_dirty_ = true;
	return in_pass ? last/in_pass : 0.0;
}

double LearnedPreconditioner::FitGain()
{
	if (pair_count_ == 0) Fail(-1, "learned preconditioner: no training pairs");
	const size_t n4 = 4*(size_t)nodes_;
	double ot = 0.0, oo = 0.0;
	std::vector<double> host(2*148);
	for (int p = 0; p < pair_count_; ++p) {
		Forward(pairs_x_.get()+(size_t)p*n4, o_.get());
		const double* pred = o_.get();
		const double* target = pairs_t_.get()+(size_t)p*n4;
		if (has_operator()) {
			ApplyOperator(o_.get(), ro_.get());
			pred = ro_.get();
			target = pairs_q_.get()+(size_t)p*n4;
		}
		GainKernel<<<148, kThreads, 0, stream_>>>((long long)n4, pred, target, scales_.get(), loss_partial_.get());
		LaunchCheck("GainKernel");
		loss_partial_.Download(host.data(), 2*148, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "learned gain");
		for (int b = 0; b < 148; ++b) { ot += host[2*b]; oo += host[2*b+1]; }
	}
	const double gain = oo > 0.0 ? std::max(0.0, ot/oo) : 0.0;
	double out[4];
	for (int c = 0; c < 4; ++c) out[c] = scale_out_[c]*(gain > 0.0 ? gain : 1e-30);
	SetScales(scale_in_, out, weight_);
	return gain;
}

double LearnedPreconditioner::EvaluatePairs()
{
	if (pair_count_ == 0) return 0.0;
	double total = 0.0;
	for (int p = 0; p < pair_count_; ++p) total += PairLoss(p, false);
	return total/pair_count_;
}

} // namespace tfiga
