// Tensor-core (tcgen05) element tangent for the mixed-precision Newton path:
// the exact VMS tangent contracted in BF16 with FP32 accumulation in tensor
// memory and added into an FP32 block-CSR Jacobian, plus the FP64 residual of
// the same element (the residual drives the Newton refinement and stays FP64).
//
// Formulation: identical to the FP64 assembly (vms_point.cuh, the reference's
// NavierStokesElement.hpp:149-317 with the exact tangent :244-312).  The
// tangent of element e, row field i, column field f is
//   K^{if}_{ab} = sum_k Psi(a, k) G^{if}(b, k),   k = (q, s): 64 points x 4 test features,
//   G^{if}(b, (q, s)) = sum_t M_q^{if}[s][t] Phi_t(b, q),
// i.e. D[m = (b, f)][n = a] = A[m][k] B[n][k]^T with A = G (K-major) and
// B = Psi (K-major), one GEMM of M = 512 x N = 64 x K = 256 per row field.
//
// Two kernels.
//   TangentPointKernel (FP64, CTA per element, 256 threads): nodal state, the
//     state at the 64 points (thread per point and quarter of the basis, the
//     quarters summed in shared memory), the coefficients M_q of all four row
//     fields (thread per row field and point, two column-field halves through
//     a shared-memory scratch) written to a coefficient array laid out
//     [element][row field][80 coefficients][64 points] (coalesced over the
//     points), and the FP64 residual (thread per basis function and quarter
//     of the points, one read of each basis value for the four row fields)
//     added into rhs.
//   TangentTcKernel (CTA per element and row-field pair h: i in {2h, 2h+1},
//     256 threads, 4 M = 128 accumulator tiles in 256 TMEM columns; tile T:
//     row field 2h + T/2, basis b in [32 (T&1), +32), tile row m = 4 (b mod
//     32) + f): K chunks of NP points; the FP32 basis and the two row fields'
//     coefficients of chunk c+2 are copied (cp.async) into the buffers chunk
//     c has just consumed, and the operand tiles are double-buffered, so chunk
//     c+1 is built while the MMAs of chunk c run.  Psi and G are written as
//     BF16 in the 64-byte-swizzled K-major layout with K ordered (s, point)
//     inside each point pair; the two points of a pair ride in one FP32
//     register pair (fma.rn.f32x2), and a pair's two coefficients are one
//     8-byte shared-memory load.  One thread issues the tile MMAs
//     (tcgen05.mma.cta_group::1.kind::f16, M = 128, N = 64, K = 16) and
//     commits them to the mbarrier of the operand buffer.  Epilogue:
//     tcgen05.ld rows (b, f) x 32 columns a of both row fields; shuffles inside
//     each lane quad give every lane the four f of one (a, b, row field), and
//     the two row fields of one (a, b) -- the two halves of a 32-byte sector --
//     go out from adjacent lanes of the same red.global.add.v4.f32.
// Split mode (TFIGA_PRECISION_MIXED_BF16X3): every operand x is carried as
// hi = bf16(x) and lo = bf16(x - hi), and the contraction takes the three
// products hi.hi + hi.lo + lo.hi (the dropped lo.lo term is 2^-16 relative),
// so the tangent is accurate to about 1e-5 instead of BF16's 2e-3.  Chunks
// hold 4 points (K = 16) and each 64-byte swizzled row carries the hi values
// in its first 32 bytes and the lo values in its last 32; the three MMAs of a
// tile start their A / B descriptors at byte 0 or 32 of the row.  Plain mode:
// chunks of 8 points, K = 32 per row, two K = 16 MMAs per tile.
// Every mbarrier wait is bounded (one second of globaltimer); on expiry the
// CTA records TFIGA status bit 1, waits once more (bounded) for its own MMAs,
// frees its tensor memory and returns without writing the tangent.
#include "common.hpp"
#include "kernels.cuh"
#include "l2_prefetch.cuh"
#include "vms_point.cuh"

#include <cuda_bf16.h>

namespace tfiga {
namespace {

constexpr int kTcThreads = 256;
constexpr int kMaxPts = 8;                       // points per K chunk (plain); split uses 4
constexpr int kTiles = 4;                        // M = 128 tiles per CTA
constexpr int kTileBytes = 128*64;               // 128 rows x 32 BF16 (64 B, one swizzle row)
constexpr int kTmemCols = 256;                   // 4 tiles x N = 64 FP32 columns
constexpr unsigned long long kWaitNs = 1000000000ull;
constexpr int kRcStride = 5;                     // doubles per (field, point) residual coefficient row
constexpr int kPartStride = 23;                  // odd double stride of the point-state partial sums
constexpr int kScratchStride = 41;               // odd float stride of the per-thread coefficient scratch

// TangentTcKernel shared memory (bytes from a 1024-aligned base).
constexpr int kOperandBytes = kTiles*kTileBytes+64*64;            // A tiles + B (Psi: 64 rows x 64 B)
constexpr int kOffOp0 = 0;                                        // operand buffer 0
constexpr int kOffOp1 = kOperandBytes;                            // operand buffer 1 (36 KiB, 1024-aligned)
constexpr int kPhiBytes = kFeatures*kMaxPts*64*4;                 // float [5][NP/2][64][2] per chunk
constexpr int kOffPhi0 = 2*kOperandBytes;
constexpr int kOffPhi1 = kOffPhi0+kPhiBytes;
// float [2 rows][80][NP] per chunk, each row field's 4 column-field groups of 20 rows followed by
// kCfPad floats, so that the four column fields' coefficients (read together) start in different banks
constexpr int kCfPad = 8;
constexpr int kCfBytes = (2*kCoef*kMaxPts+8*kCfPad)*4;
constexpr int kOffCf0 = kOffPhi1+kPhiBytes;
constexpr int kOffCf1 = kOffCf0+kCfBytes;
constexpr int kOffBar = kOffCf1+kCfBytes;                         // 2 mbarriers, TMEM slot
constexpr int kTcSmemBytes = kOffBar+32+1024;                     // + alignment slack
static_assert(kTcSmemBytes <= 113*1024, "two CTAs per SM");
static_assert(kOffOp1 % 1024 == 0, "operand buffers 1024-aligned");

// TangentPointKernel shared memory (bytes).
constexpr int kPtOffU = 0;                                        // double [4 fields][64]
constexpr int kPtOffUp = kPtOffU+64*4*8;                          // double [4 fields][64]
constexpr int kPtOffPart = kPtOffUp+64*4*8;                       // double [4][64][kPartStride]
constexpr int kPtPartBytes = 4*64*kPartStride*8;                  // (later: float [256][kScratchStride])
constexpr int kPtOffQS = kPtOffPart+kPtPartBytes;                 // double [64][kQS]
constexpr int kPtOffRC = kPtOffQS+kQuad*kQS*8;                    // double [4][64][kRcStride]
constexpr int kPtSmemBytes = kPtOffRC+4*kQuad*kRcStride*8;
static_assert(kTcThreads*kScratchStride*4 <= kPtPartBytes, "coefficient scratch fits in the partial sums");
constexpr int kStageBasis = 16;                  // basis functions per staged chunk of the point-state stage
constexpr int kPointStride = 22;                 // doubles per point of the stored point state (kU .. kLap+2)
constexpr int kStageStride = kStageBasis+1;      // odd double stride of a staged (feature, point) row
static_assert(kFeatures*kQuad*kStageStride*8 <= kPtPartBytes, "staged basis chunk fits in the partial sums");

// Instruction descriptor of tcgen05.mma kind::f16: D FP32, A and B BF16, both
// K-major, M = 128, N = 64.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
// kind::tf32: D FP32, A and B TF32 (format 2), both K-major, M = 128, N = 64.
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// Operand organisations of the tensor-core tangent (template parameter kMode):
constexpr int kModeBf16 = 0;      // BF16 operands, K = 32 (8 points) per chunk, two K = 16 MMAs per tile
constexpr int kModeSplit = 1;     // split BF16 (hi + lo), K = 16 (4 points), three products per tile
constexpr int kModeTf32 = 2;      // TF32 operands (FP32 in shared memory, rounded to TF32), K = 16 (4
                                  // points), two K = 8 MMAs per tile; no conversion into two terms

__device__ __forceinline__ uint32_t SmemAddress(const void* p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, 64-byte swizzle: 8-row atoms of
// 512 B (stride byte offset 512), leading byte offset unused (1), version 1.
__device__ __forceinline__ uint64_t DescSw64(uint32_t address)
{
	return (uint64_t)((address >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46)
		| (4ull << 61);
}

// Byte offset of 16-byte chunk j (0..3) of row r in a 64-byte-swizzled K-major tile.
__device__ __forceinline__ int Sw64(int r, int j)
{
	return r*64+((j ^ ((r >> 1) & 3)) << 4);
}

__device__ __forceinline__ unsigned long long GlobalTimer()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

__device__ __forceinline__ void MbarInit(uint64_t* bar)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(SmemAddress(bar)) : "memory");
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool MbarTryWait(uint64_t* bar, uint32_t parity)
{
	uint32_t done;
	asm volatile("{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(done) : "r"(SmemAddress(bar)), "r"(parity) : "memory");
	return done != 0;
}

// Waits for completion of the mbarrier phase with the given parity, for at most kWaitNs.
__device__ bool MbarWaitBounded(uint64_t* bar, uint32_t parity)
{
	const unsigned long long start = GlobalTimer();
	while (!MbarTryWait(bar, parity))
		if (GlobalTimer()-start > kWaitNs) return false;
	return true;
}

__device__ __forceinline__ void MmaBf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
	asm volatile("{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
		:: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0u) : "memory");
}

__device__ __forceinline__ void MmaTf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
	asm volatile("{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
		:: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kIdescTf32), "r"(accumulate), "r"(0u) : "memory");
}

__device__ __forceinline__ void MmaCommit(uint64_t* bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
		:: "r"(SmemAddress(bar)) : "memory");
}

__device__ __forceinline__ void FenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void FenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void FenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16-byte global -> shared copy, cached in L2 only.
__device__ __forceinline__ void CopyAsync16(uint32_t dst, const void* src)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void CopyAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void CopyAsyncWait()
{
	asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory");
}

// 32 lanes x 32 consecutive FP32 columns: thread l gets row (lane base + l), columns c..c+31.
__device__ __forceinline__ void TmemLoad32(uint32_t taddr, float v[32])
{
	uint32_t r[32];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
		"{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
		"%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
		  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
		  "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
		  "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
		: "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
	#pragma unroll
	for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ uint32_t PackBf16(float lo, float hi)
{
	const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
	return *reinterpret_cast<const uint32_t*>(&v);
}

// x rounded to TF32 (10 fraction bits, nearest with ties away), as the 32-bit pattern the MMA reads.
__device__ __forceinline__ uint32_t Tf32(float x)
{
	uint32_t r;
	asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
	return r;
}

// x - bf16(x): the part of x that its BF16 rounding drops (exact in FP32).
__device__ __forceinline__ float Bf16Residual(float x)
{
	return x-__bfloat162float(__float2bfloat16_rn(x));
}

// Two FP32 values in one 64-bit register pair (first value in the low half), for the packed
// FP32 pipe of sm_100 (fma / sub .f32x2: one instruction for both halves).
__device__ __forceinline__ unsigned long long Pack2(float lo, float hi)
{
	unsigned long long d;
	asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
	return d;
}
__device__ __forceinline__ float Low(unsigned long long v) { return __uint_as_float((uint32_t)v); }
__device__ __forceinline__ float High(unsigned long long v) { return __uint_as_float((uint32_t)(v >> 32)); }
__device__ __forceinline__ unsigned long long Fma2(unsigned long long a, unsigned long long b, unsigned long long c)
{
	unsigned long long d;
	asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
	return d;
}
__device__ __forceinline__ unsigned long long Mul2(unsigned long long a, unsigned long long b)
{
	unsigned long long d;
	asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
	return d;
}
__device__ __forceinline__ unsigned long long Sub2(unsigned long long a, unsigned long long b)
{
	unsigned long long d;
	asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
	return d;
}

// BF16 pair of a packed FP32 pair (low half -> low 16 bits).
__device__ __forceinline__ uint32_t Bf16Pair(unsigned long long v)
{
	return PackBf16(Low(v), High(v));
}

// The FP32 pair a BF16 pair stands for (exact).
__device__ __forceinline__ unsigned long long WidenBf16Pair(uint32_t h)
{
	return Pack2(__uint_as_float(h << 16), __uint_as_float(h & 0xffff0000u));
}

__device__ __forceinline__ void StoreShared16(uint32_t address, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
	asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" :: "r"(address), "r"(a), "r"(b), "r"(c), "r"(d)
		: "memory");
}

__device__ __forceinline__ void RedAdd4(float* p, float a, float b, float c, float d)
{
	asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" :: "l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
		: "memory");
}


// Basis chunk c (points NP c .. NP c + NP - 1, five features, 64 functions) of
// one element, FP32 with the points of each pair interleaved (the layout of
// Mesh::phi32), into a [5][NP/2][64][2] buffer; the coefficients of kRows row
// fields (from CF on) at those points into a [kRows][80][NP] buffer (padded per
// group of 20 rows).  One commit group.
template <int NP, int kRows = 2>
__device__ __forceinline__ void PrefetchChunk(const float* P32, const float* CF, int c, uint32_t phi_dst,
	uint32_t cf_dst, int tid)
{
	for (int idx = tid; idx < kFeatures*NP*16; idx += kTcThreads) {
		const int t = idx/(NP*16), rem = idx%(NP*16);
		CopyAsync16(phi_dst+16*idx, P32+(size_t)(t*kQuad+c*NP)*kMaxBasis+4*rem);
	}
	for (int idx = tid; idx < kRows*kCoef*NP/4; idx += kTcThreads) {
		const int rk = idx/(NP/4), part = idx%(NP/4);           // rk = row field * 80 + k
		CopyAsync16(cf_dst+16*idx+(rk/20)*kCfPad*4, CF+(size_t)rk*kQuad+c*NP+4*part);
	}
	CopyAsyncCommit();
}

// Coefficients of row field kRow at one point: both column-field halves through the thread's
// scratch, stored at out[k * 64] (coalesced over the points of a warp).
template <int kRow>
__device__ __forceinline__ void PointCoefficients(const PointState& S, const double* qd, const AssemblyParams& prm,
	float* scratch, double* rc, float* out)
{
	RowCoefficients<float>(kRow, S, qd, prm, scratch, rc, 0, 2);
	#pragma unroll 8
	for (int k = 0; k < 40; ++k) out[(size_t)k*kQuad] = scratch[k];
	RowCoefficients<float>(kRow, S, qd, prm, scratch, nullptr, 2, 4);
	#pragma unroll 8
	for (int k = 0; k < 40; ++k) out[(size_t)(40+k)*kQuad] = scratch[k];
}

// kMode: what the kernel stores besides adding the FP64 residual into rhs -- kPointResidual nothing
// (the residual-first Newton check of the FP64 solver), kPointCoefficients the tangent coefficients of
// the four row fields (TangentTcKernel), kPointState the FP64 state at the 64 points
// (TangentTcFusedKernel).
enum : int { kPointResidual = 0, kPointCoefficients = 1, kPointState = 2 };

template <int kMode>
__global__ void __launch_bounds__(kTcThreads, 2) TangentPointKernel(DeviceMeshView mesh,
	const double* __restrict__ phi, const double* __restrict__ qdata, const double* __restrict__ state,
	const double* __restrict__ previous, AssemblyParams prm, float* __restrict__ coef,
	double* __restrict__ point_state, double* __restrict__ rhs)
{
	extern __shared__ uint8_t smem_raw[];
	uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw)+15) & ~uintptr_t(15));
	double* U = reinterpret_cast<double*>(sm+kPtOffU);
	double* Up = reinterpret_cast<double*>(sm+kPtOffUp);
	double* Part = reinterpret_cast<double*>(sm+kPtOffPart);
	float* Scratch = reinterpret_cast<float*>(sm+kPtOffPart);
	double* QS = reinterpret_cast<double*>(sm+kPtOffQS);
	double* RC = reinterpret_cast<double*>(sm+kPtOffRC);

	const int e = blockIdx.x;
	const int tid = threadIdx.x;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	const double* P = phi+(size_t)e*kFeatures*kQuad*kMaxBasis;

	// 1. Nodal state.
	if (tid < kMaxBasis) {
		const int a = tid;
		double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, p0 = 0.0, p1 = 0.0, p2 = 0.0;
		if (a < nen) {
			const size_t node = (size_t)mesh.connectivity[begin+a];
			s0 = state[4*node]; s1 = state[4*node+1]; s2 = state[4*node+2]; s3 = state[4*node+3];
			if (prm.dt > 0.0) { p0 = previous[4*node]; p1 = previous[4*node+1]; p2 = previous[4*node+2]; }
		}
		U[a] = s0; U[64+a] = s1; U[128+a] = s2; U[192+a] = s3;
		Up[a] = p0; Up[64+a] = p1; Up[128+a] = p2; Up[192+a] = 0.0;
	}
	__syncthreads();

	// 2. State at every point (FP64): the basis tables are staged 16 functions at a time in shared
	//    memory with coalesced 16-byte loads (rows of 17 doubles, so that 8-byte reads across the
	//    points of a warp are conflict-free); thread (point q, quarter aq) takes 4 functions of each
	//    chunk; the four quarters meet in shared memory.  The staging buffer overlays the partial
	//    sums, which are written only after the last chunk has been read.
	{
		double* Stage = Part;
		const int q = tid & 63, aq = tid >> 6;
		double v[22];
		#pragma unroll
		for (int k = 0; k < 22; ++k) v[k] = 0.0;
		for (int a0 = 0; a0 < kMaxBasis; a0 += kStageBasis) {
			if (a0) __syncthreads();                 // the previous chunk has been read
			for (int idx = tid; idx < kFeatures*kQuad*(kStageBasis/2); idx += kTcThreads) {
				const int row = idx/(kStageBasis/2), k = idx%(kStageBasis/2);     // row = t*64 + point
				const double2 w = *reinterpret_cast<const double2*>(P+(size_t)row*kMaxBasis+a0+2*k);
				Stage[row*kStageStride+2*k] = w.x;
				Stage[row*kStageStride+2*k+1] = w.y;
			}
			__syncthreads();
			#pragma unroll
			for (int jj = 0; jj < kStageBasis/4; ++jj) {
				const int j = aq*(kStageBasis/4)+jj, b = a0+j;
				const double n = Stage[(0*kQuad+q)*kStageStride+j], g0 = Stage[(1*kQuad+q)*kStageStride+j];
				const double g1 = Stage[(2*kQuad+q)*kStageStride+j], g2 = Stage[(3*kQuad+q)*kStageStride+j];
				const double l = Stage[(4*kQuad+q)*kStageStride+j];
				const double uf[4] = {U[b], U[64+b], U[128+b], U[192+b]};
				v[0] += n*uf[0]; v[1] += n*uf[1]; v[2] += n*uf[2]; v[3] += n*uf[3];
				v[4] += n*Up[b]; v[5] += n*Up[64+b]; v[6] += n*Up[128+b];
				#pragma unroll
				for (int f = 0; f < 4; ++f) { v[7+3*f] += g0*uf[f]; v[8+3*f] += g1*uf[f]; v[9+3*f] += g2*uf[f]; }
				v[19] += l*uf[0]; v[20] += l*uf[1]; v[21] += l*uf[2];
			}
		}
		__syncthreads();                             // the last chunk has been read
		double* part = Part+(aq*kQuad+q)*kPartStride;
		#pragma unroll
		for (int k = 0; k < 22; ++k) part[k] = v[k];
	}
	__syncthreads();
	for (int idx = tid; idx < kQuad*22; idx += kTcThreads) {
		const int q = idx/22, k = idx%22;
		const double* part = Part+q*kPartStride+k;
		const double v = ((part[0]+part[kQuad*kPartStride])+part[2*kQuad*kPartStride])+part[3*kQuad*kPartStride];
		QS[q*kQS+k] = v;
		if constexpr (kMode == kPointState) point_state[(size_t)e*kQuad*kPointStride+idx] = v;
	}
	__syncthreads();

	// 3. Coefficients: thread (row field il, point q), two column-field halves through the
	//    scratch (the partial sums are dead), stored coalesced over the points.  The row field is
	//    uniform over a warp and a compile-time constant of each branch, so the point state and the
	//    coefficient temporaries stay in registers.
	{
		const int q = tid & 63, il = tid >> 6;
		PointState S;
		const double* s = QS+q*kQS;
		#pragma unroll
		for (int c = 0; c < 3; ++c) {
			S.u[c] = s[kU+c]; S.up[c] = s[kUp+c]; S.lap[c] = s[kLap+c]; S.gp[c] = s[kGrad+9+c];
			#pragma unroll
			for (int d = 0; d < 3; ++d) S.gv[c][d] = s[kGrad+3*c+d];
		}
		S.p = s[kP];
		const double* qd = qdata+((size_t)e*kQuad+q)*kQData;
		double* rc = RC+(il*kQuad+q)*kRcStride;
		if constexpr (kMode == kPointCoefficients) {
			float* scratch = Scratch+tid*kScratchStride;
			float* out = coef+((size_t)e*4+il)*kCoef*kQuad+q;
			switch (il) {
			case 0: PointCoefficients<0>(S, qd, prm, scratch, rc, out); break;
			case 1: PointCoefficients<1>(S, qd, prm, scratch, rc, out); break;
			case 2: PointCoefficients<2>(S, qd, prm, scratch, rc, out); break;
			default: PointCoefficients<3>(S, qd, prm, scratch, rc, out); break;
			}
		} else {
			switch (il) {
			case 0: RowCoefficients<float, 1, false>(0, S, qd, prm, nullptr, rc); break;
			case 1: RowCoefficients<float, 1, false>(1, S, qd, prm, nullptr, rc); break;
			case 2: RowCoefficients<float, 1, false>(2, S, qd, prm, nullptr, rc); break;
			default: RowCoefficients<float, 1, false>(3, S, qd, prm, nullptr, rc); break;
			}
		}
	}
	__syncthreads();

	// 4. FP64 residual of the four row fields (rhs holds -r): thread (basis function a, quarter
	//    qq of the points) reads each basis value once for all four row fields; the quarters meet
	//    in shared memory (the coefficient scratch is dead).
	{
		const int a = tid & 63, qq = tid >> 6;
		double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
		for (int q = qq*16; q < qq*16+16; ++q) {
			#pragma unroll
			for (int s = 0; s < 4; ++s) {
				const double v = P[(s*kQuad+q)*kMaxBasis+a];
				r0 += v*RC[(0*kQuad+q)*kRcStride+s];
				r1 += v*RC[(1*kQuad+q)*kRcStride+s];
				r2 += v*RC[(2*kQuad+q)*kRcStride+s];
				r3 += v*RC[(3*kQuad+q)*kRcStride+s];
			}
		}
		double* red = Part;                     // [4 quarters][4 row fields][64]
		red[(qq*4+0)*64+a] = r0; red[(qq*4+1)*64+a] = r1; red[(qq*4+2)*64+a] = r2; red[(qq*4+3)*64+a] = r3;
		__syncthreads();
		const int il = tid >> 6;
		const double r = ((red[(0*4+il)*64+a]+red[(1*4+il)*64+a])+red[(2*4+il)*64+a])+red[(3*4+il)*64+a];
		if (a < nen) atomicAdd(rhs+4*(size_t)mesh.connectivity[begin+a]+il, r);
	}
}

// lookahead: the number of CTAs resident at once (two per SM); CTA k also prefetches the tables of
// CTA k + lookahead, which starts about when CTA k finishes.
template <int kMode>
__global__ void __launch_bounds__(kTcThreads, 2) TangentTcKernel(DeviceMeshView mesh,
	const float* __restrict__ phi32, const float* __restrict__ coef, const int32_t* __restrict__ element_blocks,
	float* __restrict__ values, int* __restrict__ status, int lookahead)
{
	constexpr bool kSplit = kMode == kModeSplit, kTf32 = kMode == kModeTf32;
	constexpr bool kFour = kMode != kModeBf16;   // four points (K = 16) per chunk
	constexpr int NP = kFour ? 4 : kMaxPts;      // points per K chunk
	constexpr int kChunks = kQuad/NP;
	extern __shared__ uint8_t smem_raw[];
	uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw)+1023) & ~uintptr_t(1023));
	const uint32_t sOp[2] = {SmemAddress(sm+kOffOp0), SmemAddress(sm+kOffOp1)};
	const uint32_t sPhi[2] = {SmemAddress(sm+kOffPhi0), SmemAddress(sm+kOffPhi1)};
	const uint32_t sCf[2] = {SmemAddress(sm+kOffCf0), SmemAddress(sm+kOffCf1)};
	uint64_t* bars = reinterpret_cast<uint64_t*>(sm+kOffBar);
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm+kOffBar+16);

	const int e = blockIdx.x >> 1;
	const int h = blockIdx.x & 1;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	const float* P32 = phi32+(size_t)e*kFeatures*kQuad*kMaxBasis;
	const float* CF = coef+((size_t)e*4+2*h)*kCoef*kQuad;

	// the element's basis table and this row-field pair's coefficients into L2 at once, so that the
	// chunk copies below (one chunk ahead) wait for L2 rather than for DRAM; and those of the CTA one
	// resident wave later
	if (tid == 0) {
		PrefetchL2(P32, kFeatures*kQuad*kMaxBasis*4);
		PrefetchL2(CF, 2*kCoef*kQuad*4);
		const long long ahead = (long long)blockIdx.x+lookahead;
		if (ahead < 2LL*mesh.elements) {
			const long long ea = ahead >> 1;
			if ((ahead & 1) == 0) PrefetchL2(phi32+(size_t)ea*kFeatures*kQuad*kMaxBasis, kFeatures*kQuad*kMaxBasis*4);
			PrefetchL2(coef+((size_t)ea*4+2*(ahead & 1))*kCoef*kQuad, 2*kCoef*kQuad*4);
		}
	}
	PrefetchChunk<NP>(P32, CF, 0, sPhi[0], sCf[0], tid);
	PrefetchChunk<NP>(P32, CF, 1, sPhi[1], sCf[1], tid);
	// Tensor memory for the four accumulator tiles; one mbarrier per operand buffer.
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
			:: "r"(SmemAddress(tmem_slot)), "r"(kTmemCols) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	if (tid == 32) { MbarInit(bars); MbarInit(bars+1); }
	FenceBeforeSync();
	__syncthreads();
	FenceAfterSync();
	const uint32_t tmem = *tmem_slot;

	// Chunks, one barrier each.  On entry to chunk c its basis and coefficients are in staging buffer
	// c & 1 and visible to every thread, and operand buffer c & 1 is free.  The chunk builds its operands,
	// each thread waits for its own copies of chunk c + 1 (issued one chunk earlier), and thread 0 waits
	// for the MMAs of chunk c - 1, the last users of operand buffer (c + 1) & 1; the barrier then makes
	// all of that hold for chunk c + 1, thread 0 issues chunk c's MMAs, and chunk c + 2's data is fetched
	// into the staging buffer chunk c has just consumed.  Only thread 0 polls an mbarrier.
	const int gil = warp >> 2, gqp = warp & 3;     // G builder: row field, point pair / b quarter
	const int gf = lane & 3, gbs = lane >> 2;       //            column field, basis sub-index
	bool failed = false;
	int issued = 0;                                  // chunks whose MMAs were committed
	CopyAsyncWait<1>();                              // chunk 0 (this thread's copies)
	__syncthreads();                                 // ... and every thread's
	for (int c = 0; c < kChunks; ++c) {
		const int buf = c & 1;
		const float* PhiS = reinterpret_cast<const float*>(sm+(buf ? kOffPhi1 : kOffPhi0));
		const float* CfS = reinterpret_cast<const float*>(sm+(buf ? kOffCf1 : kOffCf0));
		const uint32_t sA = sOp[buf], sB = sOp[buf]+kTiles*kTileBytes;

		// B = Psi: row a, K = (s, point) inside each 16-byte unit (k = 2 s + point of the pair);
		// thread (a, 16-byte unit u of the row).  Plain: unit u is point pair u.  Split: units 0, 1
		// hold hi of point pairs 0, 1 and units 2, 3 their lo.
		{
			// thread (unit u, row a): a warp reads 32 consecutive functions of one point pair
			const int u = tid >> 6, a = tid & 63;
			const float2* pairs = reinterpret_cast<const float2*>(PhiS);     // [5][NP/2][64] point pairs
			if constexpr (kTf32) {
				// unit u: point pair u >> 1, test features 2 (u & 1) and 2 (u & 1) + 1, both points each
				const int qp = u >> 1, s0 = 2*(u & 1);
				const float2 x0 = pairs[(s0*(NP/2)+qp)*64+a], x1 = pairs[((s0+1)*(NP/2)+qp)*64+a];
				StoreShared16(sB+Sw64(a, u), Tf32(x0.x), Tf32(x0.y), Tf32(x1.x), Tf32(x1.y));
			} else {
				const int qp = kSplit ? (u & 1) : u;
				float x[8];
				#pragma unroll
				for (int s = 0; s < 4; ++s) {
					const float2 v = pairs[(s*(NP/2)+qp)*64+a];
					x[2*s] = v.x;
					x[2*s+1] = v.y;
				}
				if (kSplit && u >= 2) {
					#pragma unroll
					for (int k = 0; k < 8; ++k) x[k] = Bf16Residual(x[k]);
				}
				StoreShared16(sB+Sw64(a, u), PackBf16(x[0], x[1]), PackBf16(x[2], x[3]), PackBf16(x[4], x[5]),
					PackBf16(x[6], x[7]));
			}
		}
		// A = G: row (b, f) of tile (il, b / 32).  Plain: warp (il, point pair) over all b.  Split:
		// warp (il, point pair, half of the b groups), writing hi and lo units.  Both points of
		// the pair ride in one register pair: coefficients mm[k] = (M_q0, M_q1)[k] (one 8-byte
		// load from the [2][80][NP] chunk), basis pb[t] = (Phi_t(q0, b), Phi_t(q1, b)).
		{
			const int qpair = kFour ? (gqp & 1) : gqp;
			const int ql0 = 2*qpair;
			constexpr int kGroups = kFour ? 4 : 8;
			const int g0 = kFour ? (gqp >> 1)*4 : 0;
			unsigned long long mm[20];
			const float* c0 = CfS+(gil*kCoef+gf*20)*NP+(gil*4+gf)*kCfPad+ql0;
			#pragma unroll
			for (int k = 0; k < 20; ++k) mm[k] = *reinterpret_cast<const unsigned long long*>(c0+k*NP);
			#pragma unroll 2
			for (int j = 0; j < kGroups; ++j) {
				const int b = (g0+j)*8+gbs;
				unsigned long long pb[5];
				#pragma unroll
				for (int t = 0; t < 5; ++t)
					pb[t] = *reinterpret_cast<const unsigned long long*>(PhiS+((t*(NP/2)+qpair)*64+b)*2);
				unsigned long long gg[4];
				#pragma unroll
				for (int s = 0; s < 4; ++s) {
					gg[s] = Mul2(mm[s*5], pb[0]);
					#pragma unroll
					for (int t = 1; t < 5; ++t) gg[s] = Fma2(mm[s*5+t], pb[t], gg[s]);
				}
				const int tile = gil*2+(b >> 5), row = (b & 31)*4+gf;
				const uint32_t dst = sA+tile*kTileBytes;
				if constexpr (kTf32) {
					// units 2 qpair (features 0, 1) and 2 qpair + 1 (features 2, 3), both points each
					StoreShared16(dst+Sw64(row, 2*qpair), Tf32(Low(gg[0])), Tf32(High(gg[0])), Tf32(Low(gg[1])),
						Tf32(High(gg[1])));
					StoreShared16(dst+Sw64(row, 2*qpair+1), Tf32(Low(gg[2])), Tf32(High(gg[2])), Tf32(Low(gg[3])),
						Tf32(High(gg[3])));
				} else {
					uint32_t hi[4];
					#pragma unroll
					for (int s = 0; s < 4; ++s) hi[s] = Bf16Pair(gg[s]);
					StoreShared16(dst+Sw64(row, qpair), hi[0], hi[1], hi[2], hi[3]);
					if (kSplit) {
						uint32_t lo[4];
						#pragma unroll
						for (int s = 0; s < 4; ++s) lo[s] = Bf16Pair(Sub2(gg[s], WidenBf16Pair(hi[s])));
						StoreShared16(dst+Sw64(row, 2+qpair), lo[0], lo[1], lo[2], lo[3]);
					}
				}
			}
		}
		FenceProxyAsync();
		CopyAsyncWait<0>();                      // chunk c + 1 (the only group in flight)
		bool ok = true;
		if (tid == 0 && c >= 1) ok = MbarWaitBounded(bars+((c-1) & 1), (uint32_t)(((c-1) >> 1) & 1));
		if (__syncthreads_or(!ok)) { failed = true; break; }
		if (tid == 0) {
			FenceAfterSync();
			#pragma unroll
			for (int tile = 0; tile < kTiles; ++tile) {
				const uint32_t a = sA+tile*kTileBytes;
				if constexpr (kTf32) {
					#pragma unroll
					for (int ks = 0; ks < 2; ++ks)
						MmaTf32(tmem+tile*64, DescSw64(a+ks*32), DescSw64(sB+ks*32), (c > 0 || ks > 0) ? 1u : 0u);
				} else if (kSplit) {
					MmaBf16(tmem+tile*64, DescSw64(a), DescSw64(sB), c > 0 ? 1u : 0u);       // hi hi
					MmaBf16(tmem+tile*64, DescSw64(a), DescSw64(sB+32), 1u);                 // hi lo
					MmaBf16(tmem+tile*64, DescSw64(a+32), DescSw64(sB), 1u);                 // lo hi
				} else {
					#pragma unroll
					for (int ks = 0; ks < 2; ++ks)
						MmaBf16(tmem+tile*64, DescSw64(a+ks*32), DescSw64(sB+ks*32), (c > 0 || ks > 0) ? 1u : 0u);
				}
			}
			MmaCommit(bars+buf);
		}
		issued = c+1;
		// the staging buffers of chunk c are free: fetch chunk c + 2 into them (an empty group at the end)
		if (c+2 < kChunks) PrefetchChunk<NP>(P32, CF, c+2, sPhi[buf], sCf[buf], tid);
		else CopyAsyncCommit();
	}
	// every thread observes the last commit itself before it reads the accumulators
	if (!failed)
		failed = __syncthreads_or(!MbarWaitBounded(bars+((kChunks-1) & 1), (uint32_t)(((kChunks-1) >> 1) & 1))) != 0;

	if (!failed) {
		// Epilogue: warp -> (basis half bh = warp/4 of b, TMEM lane quarter warp%4); both row fields.
		// Lane f of a quad holds column field f of node b for every a.  In pass p the quad's lanes
		// write (a = 4g + (f & 2) + p, row field 2h + (f & 1), all four column fields), so lanes
		// f, f^1 fill the two 16-byte halves of one 32-byte sector in the same instruction.  Each
		// round r of a pass sends to lane f^r the value it needs from this lane's column field.
		FenceAfterSync();
		const int bh = warp >> 2, quarter = warp & 3;
		const int32_t* EB = element_blocks+(size_t)e*kMaxBasis*kMaxBasis;
		const int f = lane & 3;
		const int b = bh*32+quarter*8+(lane >> 2);
		float* row_base = values+(size_t)(2*h+(f & 1))*4;
		for (int ah = 0; ah < 2; ++ah) {
			int blocks[2][8];                 // fetched before the TMEM loads
			#pragma unroll
			for (int g = 0; g < 8; ++g)
				#pragma unroll
				for (int p = 0; p < 2; ++p) {
					const int a = ah*32+4*g+(f & 2)+p;
					blocks[p][g] = (a < nen && b < nen) ? EB[a*kMaxBasis+b] : -1;
				}
			float v0[32], v1[32];
			const uint32_t lanes = (uint32_t)(quarter*32) << 16;
			TmemLoad32(tmem+lanes+bh*64+ah*32, v0);          // row field 2h
			TmemLoad32(tmem+lanes+(2+bh)*64+ah*32, v1);      // row field 2h+1
			#pragma unroll
			for (int g = 0; g < 8; ++g)
				#pragma unroll
				for (int p = 0; p < 2; ++p) {
					const float c00 = v0[4*g+p], c02 = v0[4*g+2+p], c10 = v1[4*g+p], c12 = v1[4*g+2+p];
					float o0 = 0.f, o1 = 0.f, o2 = 0.f, o3 = 0.f;
					#pragma unroll
					for (int r = 0; r < 4; ++r) {
						const int d = f ^ r;          // the lane served this round (and the source heard from)
						const float send = (d & 1) ? ((d & 2) ? c12 : c10) : ((d & 2) ? c02 : c00);
						const float got = r ? __shfl_xor_sync(0xffffffffu, send, r) : send;
						o0 = d == 0 ? got : o0; o1 = d == 1 ? got : o1;
						o2 = d == 2 ? got : o2; o3 = d == 3 ? got : o3;
					}
					if (blocks[p][g] >= 0) RedAdd4(row_base+(size_t)blocks[p][g]*16, o0, o1, o2, o3);
				}
		}
	} else {
		if (tid == 0) atomicOr(status, 1);
		CopyAsyncWait<0>();                     // this thread's copies in flight
		// let this CTA's own MMAs drain before freeing TMEM: the newest commit covers all earlier ones
		if (issued > 0) MbarWaitBounded(bars+((issued-1) & 1), (uint32_t)(((issued-1) >> 1) & 1));
	}
	FenceBeforeSync();
	__syncthreads();
	if (warp == 0) {
		FenceAfterSync();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTmemCols)
			: "memory");
	}
}

// ---- element variant: one persistent CTA per SM, all four row fields ---------------------------------
// TangentTcQuadKernel: the contraction of TangentTcKernel for all four row fields of an element in one
// CTA, so that the basis chunk is staged and Psi built once per element instead of once per row-field
// pair, and each G-building thread keeps the coefficients of two row fields in registers and reuses
// every basis value it loads for both (half the basis loads per G entry).  Eight M = 128 accumulator
// tiles (row field il, basis half) fill the 512 TMEM columns, so one CTA runs per SM; it is persistent
// (elements blockIdx.x, + gridDim.x, ...), keeps its tensor memory and mbarriers across elements, and
// fetches the next element's first two chunks before the epilogue of the current one.
constexpr int kQTiles = 8;
constexpr int kQTmemCols = 512;
constexpr int kQOperandBytes = kQTiles*kTileBytes+64*64;          // A tiles + B, 68 KiB
constexpr int kQOffOp0 = 0;
constexpr int kQOffOp1 = kQOperandBytes;
constexpr int kQOffPhi0 = 2*kQOperandBytes;
constexpr int kQOffPhi1 = kQOffPhi0+kPhiBytes;
constexpr int kQCfBytes = (4*kCoef*kMaxPts+16*kCfPad)*4;           // float [4 rows][80][NP], padded
constexpr int kQOffCf0 = kQOffPhi1+kPhiBytes;
constexpr int kQOffCf1 = kQOffCf0+kQCfBytes;
constexpr int kQOffBar = kQOffCf1+kQCfBytes;                       // 2 mbarriers, TMEM slot
constexpr int kQSmemBytes = kQOffBar+32+1024;
static_assert(kQSmemBytes <= 227*1024, "element tangent shared memory");
static_assert(kQOffOp1 % 1024 == 0, "operand buffers 1024-aligned");

template <int kMode>
__global__ void __launch_bounds__(kTcThreads, 1) TangentTcQuadKernel(DeviceMeshView mesh,
	const float* __restrict__ phi32, const float* __restrict__ coef, const int32_t* __restrict__ element_blocks,
	float* __restrict__ values, int* __restrict__ status)
{
	constexpr bool kSplit = kMode == kModeSplit, kTf32 = kMode == kModeTf32;
	constexpr bool kFour = kMode != kModeBf16;   // four points (K = 16) per chunk
	constexpr int NP = kFour ? 4 : kMaxPts;      // points per K chunk
	constexpr int kChunks = kQuad/NP;            // even: chunk c of every element uses buffer c & 1
	static_assert(kChunks % 2 == 0, "chunks per element");
	extern __shared__ uint8_t smem_raw[];
	uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw)+1023) & ~uintptr_t(1023));
	const uint32_t sOp[2] = {SmemAddress(sm+kQOffOp0), SmemAddress(sm+kQOffOp1)};
	const uint32_t sPhi[2] = {SmemAddress(sm+kQOffPhi0), SmemAddress(sm+kQOffPhi1)};
	const uint32_t sCf[2] = {SmemAddress(sm+kQOffCf0), SmemAddress(sm+kQOffCf1)};
	uint64_t* bars = reinterpret_cast<uint64_t*>(sm+kQOffBar);
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm+kQOffBar+16);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const size_t kPhiPer = (size_t)kFeatures*kQuad*kMaxBasis, kCfPer = (size_t)4*kCoef*kQuad;

	int e = blockIdx.x;
	if (e >= mesh.elements) return;
	PrefetchChunk<NP, 4>(phi32+e*kPhiPer, coef+e*kCfPer, 0, sPhi[0], sCf[0], tid);
	PrefetchChunk<NP, 4>(phi32+e*kPhiPer, coef+e*kCfPer, 1, sPhi[1], sCf[1], tid);
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
			:: "r"(SmemAddress(tmem_slot)), "r"(kQTmemCols) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	if (tid == 32) { MbarInit(bars); MbarInit(bars+1); }
	FenceBeforeSync();
	__syncthreads();
	FenceAfterSync();
	const uint32_t tmem = *tmem_slot;

	// G builder: warp -> (row-field pair ip: rows 2 ip, 2 ip + 1; point pair / basis quarter gqp);
	// lane -> (column field gf, basis sub-index gbs).
	const int ip = warp >> 2, gqp = warp & 3;
	const int gf = lane & 3, gbs = lane >> 2;
	bool failed = false;
	long long done = 0;                              // chunks of the elements before this one
	long long committed = 0;                         // chunks whose MMAs were committed
	for (; e < mesh.elements; e += gridDim.x) {
		const int begin = mesh.element_offsets[e];
		const int nen = mesh.element_offsets[e+1]-begin;
		const float* P32 = phi32+e*kPhiPer;
		const float* CF = coef+e*kCfPer;
		const int en = e+(int)gridDim.x;
		// the next element's tables into L2 while this one is contracted
		if (tid == 0 && en < mesh.elements) {
			PrefetchL2(phi32+en*kPhiPer, (int)(kPhiPer*4));
			PrefetchL2(coef+en*kCfPer, (int)(kCfPer*4));
		}
		CopyAsyncWait<1>();                          // chunk 0 (this thread's copies)
		__syncthreads();                             // ... and every thread's
		for (int c = 0; c < kChunks; ++c) {
			const long long gc = done+c;             // chunk index over the CTA's lifetime
			const int buf = c & 1;
			const float* PhiS = reinterpret_cast<const float*>(sm+(buf ? kQOffPhi1 : kQOffPhi0));
			const float* CfS = reinterpret_cast<const float*>(sm+(buf ? kQOffCf1 : kQOffCf0));
			const uint32_t sA = sOp[buf], sB = sOp[buf]+kQTiles*kTileBytes;
			// B = Psi (as in TangentTcKernel), built once for all four row fields.
			{
				const int u = tid >> 6, a = tid & 63;
				const float2* pairs = reinterpret_cast<const float2*>(PhiS);
				if constexpr (kTf32) {
					const int qp = u >> 1, s0 = 2*(u & 1);
					const float2 x0 = pairs[(s0*(NP/2)+qp)*64+a], x1 = pairs[((s0+1)*(NP/2)+qp)*64+a];
					StoreShared16(sB+Sw64(a, u), Tf32(x0.x), Tf32(x0.y), Tf32(x1.x), Tf32(x1.y));
				} else {
					const int qp = kSplit ? (u & 1) : u;
					float x[8];
					#pragma unroll
					for (int s = 0; s < 4; ++s) {
						const float2 v = pairs[(s*(NP/2)+qp)*64+a];
						x[2*s] = v.x;
						x[2*s+1] = v.y;
					}
					if (kSplit && u >= 2) {
						#pragma unroll
						for (int k = 0; k < 8; ++k) x[k] = Bf16Residual(x[k]);
					}
					StoreShared16(sB+Sw64(a, u), PackBf16(x[0], x[1]), PackBf16(x[2], x[3]), PackBf16(x[4], x[5]),
						PackBf16(x[6], x[7]));
				}
			}
			// A = G for row fields 2 ip and 2 ip + 1: each basis pair pb feeds both rows' products.
			{
				const int qpair = kFour ? (gqp & 1) : gqp;
				const int ql0 = 2*qpair;
				constexpr int kGroups = kFour ? 4 : 8;
				const int g0 = kFour ? (gqp >> 1)*4 : 0;
				unsigned long long mm[2][20];
				#pragma unroll
				for (int r = 0; r < 2; ++r) {
					const int il = 2*ip+r;
					const float* c0 = CfS+(il*kCoef+gf*20)*NP+(il*4+gf)*kCfPad+ql0;
					#pragma unroll
					for (int k = 0; k < 20; ++k) mm[r][k] = *reinterpret_cast<const unsigned long long*>(c0+k*NP);
				}
				// two basis groups per iteration: twice the independent FMA chains between the basis loads
				#pragma unroll 2
				for (int j = 0; j < kGroups; ++j) {
					const int b = (g0+j)*8+gbs;
					unsigned long long pb[5];
					#pragma unroll
					for (int t = 0; t < 5; ++t)
						pb[t] = *reinterpret_cast<const unsigned long long*>(PhiS+((t*(NP/2)+qpair)*64+b)*2);
					#pragma unroll
					for (int r = 0; r < 2; ++r) {
						unsigned long long gg[4];
						#pragma unroll
						for (int s = 0; s < 4; ++s) {
							gg[s] = Mul2(mm[r][s*5], pb[0]);
							#pragma unroll
							for (int t = 1; t < 5; ++t) gg[s] = Fma2(mm[r][s*5+t], pb[t], gg[s]);
						}
						const int tile = (2*ip+r)*2+(b >> 5), row = (b & 31)*4+gf;
						const uint32_t dst = sA+tile*kTileBytes;
						if constexpr (kTf32) {
							StoreShared16(dst+Sw64(row, 2*qpair), Tf32(Low(gg[0])), Tf32(High(gg[0])), Tf32(Low(gg[1])),
								Tf32(High(gg[1])));
							StoreShared16(dst+Sw64(row, 2*qpair+1), Tf32(Low(gg[2])), Tf32(High(gg[2])), Tf32(Low(gg[3])),
								Tf32(High(gg[3])));
						} else {
							uint32_t hi[4];
							#pragma unroll
							for (int s = 0; s < 4; ++s) hi[s] = Bf16Pair(gg[s]);
							StoreShared16(dst+Sw64(row, qpair), hi[0], hi[1], hi[2], hi[3]);
							if (kSplit) {
								uint32_t lo[4];
								#pragma unroll
								for (int s = 0; s < 4; ++s) lo[s] = Bf16Pair(Sub2(gg[s], WidenBf16Pair(hi[s])));
								StoreShared16(dst+Sw64(row, 2+qpair), lo[0], lo[1], lo[2], lo[3]);
							}
						}
					}
				}
			}
			FenceProxyAsync();
			CopyAsyncWait<0>();                      // chunk c + 1 (the only group in flight)
			bool ok = true;
			// the MMAs of chunk gc - 1 (this element's previous chunk, or the previous element's last)
			// were the last users of operand buffer (c + 1) & 1
			if (tid == 0 && gc >= 1) ok = MbarWaitBounded(bars+((gc-1) & 1), (uint32_t)(((gc-1) >> 1) & 1));
			if (__syncthreads_or(!ok)) { failed = true; break; }
			if (tid == 0) {
				FenceAfterSync();
				#pragma unroll
				for (int tile = 0; tile < kQTiles; ++tile) {
					const uint32_t a = sA+tile*kTileBytes;
					if constexpr (kTf32) {
						#pragma unroll
						for (int ks = 0; ks < 2; ++ks)
							MmaTf32(tmem+tile*64, DescSw64(a+ks*32), DescSw64(sB+ks*32), (c > 0 || ks > 0) ? 1u : 0u);
					} else if (kSplit) {
						MmaBf16(tmem+tile*64, DescSw64(a), DescSw64(sB), c > 0 ? 1u : 0u);
						MmaBf16(tmem+tile*64, DescSw64(a), DescSw64(sB+32), 1u);
						MmaBf16(tmem+tile*64, DescSw64(a+32), DescSw64(sB), 1u);
					} else {
						#pragma unroll
						for (int ks = 0; ks < 2; ++ks)
							MmaBf16(tmem+tile*64, DescSw64(a+ks*32), DescSw64(sB+ks*32), (c > 0 || ks > 0) ? 1u : 0u);
					}
				}
				MmaCommit(bars+buf);
			}
			committed = gc+1;
			// the staging buffers of chunk c are free: fetch chunk c + 2, or the next element's chunk
			// c + 2 - kChunks (an empty group after the last element)
			if (c+2 < kChunks) PrefetchChunk<NP, 4>(P32, CF, c+2, sPhi[buf], sCf[buf], tid);
			else if (en < mesh.elements)
				PrefetchChunk<NP, 4>(phi32+en*kPhiPer, coef+en*kCfPer, c+2-kChunks, sPhi[buf], sCf[buf], tid);
			else CopyAsyncCommit();
		}
		if (failed) break;
		done += kChunks;
		// every thread observes the element's last commit itself before it reads the accumulators
		if (__syncthreads_or(!MbarWaitBounded(bars+((done-1) & 1), (uint32_t)(((done-1) >> 1) & 1)))) {
			failed = true;
			break;
		}
		// Epilogue (as in TangentTcKernel) for row-field pairs p = 0, 1: warp -> (basis half bh, TMEM lane
		// quarter); tile (row field il, half bh) sits in columns (2 il + bh) 64.
		FenceAfterSync();
		{
			const int bh = warp >> 2, quarter = warp & 3;
			const int32_t* EB = element_blocks+(size_t)e*kMaxBasis*kMaxBasis;
			const int f = lane & 3;
			const int b = bh*32+quarter*8+(lane >> 2);
			for (int p = 0; p < 2; ++p) {
				float* row_base = values+(size_t)(2*p+(f & 1))*4;
				for (int ah = 0; ah < 2; ++ah) {
					int blocks[2][8];
					#pragma unroll
					for (int g = 0; g < 8; ++g)
						#pragma unroll
						for (int q = 0; q < 2; ++q) {
							const int a = ah*32+4*g+(f & 2)+q;
							blocks[q][g] = (a < nen && b < nen) ? EB[a*kMaxBasis+b] : -1;
						}
					float v0[32], v1[32];
					const uint32_t lanes = (uint32_t)(quarter*32) << 16;
					TmemLoad32(tmem+lanes+(4*p+bh)*64+ah*32, v0);          // row field 2p
					TmemLoad32(tmem+lanes+(4*p+2+bh)*64+ah*32, v1);        // row field 2p + 1
					#pragma unroll
					for (int g = 0; g < 8; ++g)
						#pragma unroll
						for (int q = 0; q < 2; ++q) {
							const float c00 = v0[4*g+q], c02 = v0[4*g+2+q], c10 = v1[4*g+q], c12 = v1[4*g+2+q];
							float o0 = 0.f, o1 = 0.f, o2 = 0.f, o3 = 0.f;
							#pragma unroll
							for (int r = 0; r < 4; ++r) {
								const int d = f ^ r;
								const float send = (d & 1) ? ((d & 2) ? c12 : c10) : ((d & 2) ? c02 : c00);
								const float got = r ? __shfl_xor_sync(0xffffffffu, send, r) : send;
								o0 = d == 0 ? got : o0; o1 = d == 1 ? got : o1;
								o2 = d == 2 ? got : o2; o3 = d == 3 ? got : o3;
							}
							if (blocks[q][g] >= 0) RedAdd4(row_base+(size_t)blocks[q][g]*16, o0, o1, o2, o3);
						}
				}
			}
		}
		// the accumulators have been read before the next element's first MMAs overwrite them
		FenceBeforeSync();
		__syncthreads();
		FenceAfterSync();
	}
	if (failed) {
		if (tid == 0) atomicOr(status, 1);
		CopyAsyncWait<0>();
		// let this CTA's own MMAs drain before freeing TMEM: the newest commit covers all earlier ones
		if (tid == 0 && committed > 0)
			MbarWaitBounded(bars+((committed-1) & 1), (uint32_t)(((committed-1) >> 1) & 1));
	}
	FenceBeforeSync();
	__syncthreads();
	if (warp == 0) {
		FenceAfterSync();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kQTmemCols)
			: "memory");
	}
}

// ---- fused variant: coefficients made in the tensor-core kernel ------------------------------------
// TangentTcFusedKernel: the same contraction as TangentTcKernel, but its operands come from tables
// that cost far less memory.  The point kernel stores the FP64 state at the 64 points (11 KiB per
// element instead of 80 KiB of coefficients); this kernel computes its two row fields' coefficients
// M_q from it in its prologue (FP64 arithmetic, FP32 storage, bitwise the coefficients the point
// kernel would have written) into shared memory, and stages the basis chunks from the FP64 tables:
// the next-but-one chunk is loaded into registers while the current chunk is built and converted to
// FP32 in shared memory after it, so no FP32 copy of the tables is kept.  One CTA per (element,
// row-field pair) and SM: 512 threads (16 warps), 256 TMEM columns, 135 KiB of shared memory.
constexpr int kFusedThreads = 512;
constexpr int kFOffOp0 = 0;
constexpr int kFOffOp1 = kOperandBytes;
constexpr int kFOffPhi0 = 2*kOperandBytes;
constexpr int kFOffPhi1 = kFOffPhi0+kPhiBytes;
// Staged coefficients: float [2 rows][80][kCoefStride] with the 64 points of a coefficient row padded to
// 66 floats, so that the four column fields' rows (20 coefficients apart) start in different banks.
constexpr int kCoefStride = 66;
constexpr int kFCoefBytes = 2*kCoef*kCoefStride*4;
constexpr int kFOffCoef = kFOffPhi1+kPhiBytes;
constexpr int kFOffBar = kFOffCoef+kFCoefBytes;
constexpr int kFusedSmemBytes = kFOffBar+32+1024;
static_assert(kFusedSmemBytes <= 227*1024, "fused tangent shared memory");
static_assert(kQuad*kPointStride*8 <= kOperandBytes, "point-state staging fits in operand buffer 0");

// One basis chunk (points NP c .. NP c + NP - 1, five features, 64 functions) of one element:
// FP64 loads into registers, then FP32 stores into a [5][NP][64] buffer.
// One (feature, point pair, function) per slot: the two points' FP64 values (64 apart in the table)
// into registers, then one float2 into the [5][NP/2][64][2] staging layout of the coefficient kernel.
template <int NP>
struct PhiChunk {
	static constexpr int kPairs = kFeatures*(NP/2)*64;                 // point pairs per chunk
	static constexpr int kSlots = (kPairs+kFusedThreads-1)/kFusedThreads;
	double2 v[kSlots];
	__device__ __forceinline__ void Load(const double* P, int c, int tid)
	{
		#pragma unroll
		for (int s = 0; s < kSlots; ++s) {
			const int idx = tid+s*kFusedThreads;
			if (idx < kPairs) {
				const int t = idx/((NP/2)*64), rem = idx%((NP/2)*64), qp = rem/64, b = rem%64;
				const double* row = P+(size_t)(t*kQuad+c*NP+2*qp)*kMaxBasis+b;
				v[s] = make_double2(__ldg(row), __ldg(row+kMaxBasis));
			}
		}
	}
	__device__ __forceinline__ void Store(float* dst, int tid) const
	{
		#pragma unroll
		for (int s = 0; s < kSlots; ++s) {
			const int idx = tid+s*kFusedThreads;
			if (idx < kPairs) reinterpret_cast<float2*>(dst)[idx] = make_float2((float)v[s].x, (float)v[s].y);
		}
	}
};

template <int kMode>
__global__ void __launch_bounds__(kFusedThreads, 1) TangentTcFusedKernel(DeviceMeshView mesh,
	const double* __restrict__ phi, const double* __restrict__ qdata, const double* __restrict__ point_state,
	AssemblyParams prm, const int32_t* __restrict__ element_blocks, float* __restrict__ values,
	int* __restrict__ status, int lookahead)
{
	constexpr bool kSplit = kMode == kModeSplit, kTf32 = kMode == kModeTf32;
	constexpr bool kFour = kMode != kModeBf16;   // four points (K = 16) per chunk
	constexpr int NP = kFour ? 4 : kMaxPts;      // points per K chunk
	constexpr int kChunks = kQuad/NP;
	extern __shared__ uint8_t smem_raw[];
	uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw)+1023) & ~uintptr_t(1023));
	const uint32_t sOp[2] = {SmemAddress(sm+kFOffOp0), SmemAddress(sm+kFOffOp1)};
	float* PhiF[2] = {reinterpret_cast<float*>(sm+kFOffPhi0), reinterpret_cast<float*>(sm+kFOffPhi1)};
	float* CoefS = reinterpret_cast<float*>(sm+kFOffCoef);
	uint64_t* bars = reinterpret_cast<uint64_t*>(sm+kFOffBar);
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm+kFOffBar+16);

	const int e = blockIdx.x >> 1;
	const int h = blockIdx.x & 1;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	const double* P = phi+(size_t)e*kFeatures*kQuad*kMaxBasis;
	if (tid == 0) {
		PrefetchL2(P, kFeatures*kQuad*kMaxBasis*8);
		PrefetchL2(point_state+(size_t)e*kQuad*kPointStride, kQuad*kPointStride*8);
		// the element of the CTA one resident wave later (the pair of CTAs of an element shares it)
		const long long ahead = (long long)blockIdx.x+lookahead;
		if (ahead < 2LL*mesh.elements && (ahead & 1) == 0) {
			const long long ea = ahead >> 1;
			PrefetchL2(phi+(size_t)ea*kFeatures*kQuad*kMaxBasis, kFeatures*kQuad*kMaxBasis*8);
			PrefetchL2(point_state+(size_t)ea*kQuad*kPointStride, kQuad*kPointStride*8);
		}
	}

	PhiChunk<NP> stage;
	stage.Load(P, 0, tid);
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
			:: "r"(SmemAddress(tmem_slot)), "r"(kTmemCols) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	if (tid == 32) { MbarInit(bars); MbarInit(bars+1); }
	// the element's point state, staged in operand buffer 0 (free until the first chunk is built)
	double* QSs = reinterpret_cast<double*>(sm+kFOffOp0);
	const double* PS = point_state+(size_t)e*kQuad*kPointStride;
	for (int idx = tid; idx < kQuad*kPointStride; idx += kFusedThreads) QSs[idx] = PS[idx];
	stage.Store(PhiF[0], tid);
	stage.Load(P, 1, tid);
	FenceBeforeSync();
	__syncthreads();
	FenceAfterSync();
	const uint32_t tmem = *tmem_slot;
	// coefficients of row fields 2h, 2h + 1 at every point: thread (row rl, point q, column field f)
	{
		const int rl = tid >> 8, q = (tid >> 2) & 63, f = tid & 3;
		const double* s = QSs+q*kPointStride;
		PointState S;
		#pragma unroll
		for (int c = 0; c < 3; ++c) {
			S.u[c] = s[kU+c]; S.up[c] = s[kUp+c]; S.lap[c] = s[kLap+c]; S.gp[c] = s[kGrad+9+c];
			#pragma unroll
			for (int d = 0; d < 3; ++d) S.gv[c][d] = s[kGrad+3*c+d];
		}
		S.p = s[kP];
		RowCoefficients<float, kCoefStride>(2*h+rl, S, qdata+((size_t)e*kQuad+q)*kQData, prm,
			CoefS+(rl*kCoef+f*20)*kCoefStride+q, nullptr, f, f+1);
	}
	stage.Store(PhiF[1], tid);
	__syncthreads();                             // coefficients and chunks 0, 1 in place; QSs free

	// Chunks: as TangentTcKernel, with 16 warps: warp & 7 picks the row field and point pair (and in
	// split mode the basis half) as there, warp >> 3 half of that warp's basis groups.
	const int gil = (warp >> 2) & 1, gqp = warp & 3, ghalf = warp >> 3;
	const int gf = lane & 3, gbs = lane >> 2;
	bool failed = false;
	int issued = 0;
	// One barrier per chunk, as TangentTcKernel: after building chunk c, thread 0 waits for the MMAs of
	// chunk c - 1 (the last users of operand buffer (c + 1) & 1) before the barrier.
	for (int c = 0; c < kChunks; ++c) {
		const int buf = c & 1;
		const float* PhiS = PhiF[buf];
		if (c+2 < kChunks) stage.Load(P, c+2, tid);
		const uint32_t sA = sOp[buf], sB = sOp[buf]+kTiles*kTileBytes;
		if (tid < kTcThreads) {
			// thread (unit u, row a): a warp reads 32 consecutive functions of one point pair
			const int u = tid >> 6, a = tid & 63;
			const float2* pairs = reinterpret_cast<const float2*>(PhiS);     // [5][NP/2][64] point pairs
			if constexpr (kTf32) {
				// unit u: point pair u >> 1, test features 2 (u & 1) and 2 (u & 1) + 1, both points each
				const int qp = u >> 1, s0 = 2*(u & 1);
				const float2 x0 = pairs[(s0*(NP/2)+qp)*64+a], x1 = pairs[((s0+1)*(NP/2)+qp)*64+a];
				StoreShared16(sB+Sw64(a, u), Tf32(x0.x), Tf32(x0.y), Tf32(x1.x), Tf32(x1.y));
			} else {
				const int qp = kSplit ? (u & 1) : u;
				float x[8];
				#pragma unroll
				for (int s = 0; s < 4; ++s) {
					const float2 v = pairs[(s*(NP/2)+qp)*64+a];
					x[2*s] = v.x;
					x[2*s+1] = v.y;
				}
				if (kSplit && u >= 2) {
					#pragma unroll
					for (int k = 0; k < 8; ++k) x[k] = Bf16Residual(x[k]);
				}
				StoreShared16(sB+Sw64(a, u), PackBf16(x[0], x[1]), PackBf16(x[2], x[3]), PackBf16(x[4], x[5]),
					PackBf16(x[6], x[7]));
			}
		}
		{
			const int qpair = kFour ? (gqp & 1) : gqp;
			const int ql0 = 2*qpair;
			constexpr int kGroups = kFour ? 2 : 4;
			const int g0 = kFour ? (gqp >> 1)*4+ghalf*2 : ghalf*4;
			unsigned long long mm[20];
			const float* c0 = CoefS+(gil*kCoef+gf*20)*kCoefStride+c*NP+ql0;
			#pragma unroll
			for (int k = 0; k < 20; ++k) mm[k] = *reinterpret_cast<const unsigned long long*>(c0+k*kCoefStride);
			#pragma unroll
			for (int j = 0; j < kGroups; ++j) {
				const int b = (g0+j)*8+gbs;
				unsigned long long pb[5];
				#pragma unroll
				for (int t = 0; t < 5; ++t)
					pb[t] = *reinterpret_cast<const unsigned long long*>(PhiS+((t*(NP/2)+qpair)*64+b)*2);
				unsigned long long gg[4];
				#pragma unroll
				for (int s = 0; s < 4; ++s) {
					gg[s] = Mul2(mm[s*5], pb[0]);
					#pragma unroll
					for (int t = 1; t < 5; ++t) gg[s] = Fma2(mm[s*5+t], pb[t], gg[s]);
				}
				const int tile = gil*2+(b >> 5), row = (b & 31)*4+gf;
				const uint32_t dst = sA+tile*kTileBytes;
				if constexpr (kTf32) {
					// units 2 qpair (features 0, 1) and 2 qpair + 1 (features 2, 3), both points each
					StoreShared16(dst+Sw64(row, 2*qpair), Tf32(Low(gg[0])), Tf32(High(gg[0])), Tf32(Low(gg[1])),
						Tf32(High(gg[1])));
					StoreShared16(dst+Sw64(row, 2*qpair+1), Tf32(Low(gg[2])), Tf32(High(gg[2])), Tf32(Low(gg[3])),
						Tf32(High(gg[3])));
				} else {
					uint32_t hi[4];
					#pragma unroll
					for (int s = 0; s < 4; ++s) hi[s] = Bf16Pair(gg[s]);
					StoreShared16(dst+Sw64(row, qpair), hi[0], hi[1], hi[2], hi[3]);
					if (kSplit) {
						uint32_t lo[4];
						#pragma unroll
						for (int s = 0; s < 4; ++s) lo[s] = Bf16Pair(Sub2(gg[s], WidenBf16Pair(hi[s])));
						StoreShared16(dst+Sw64(row, 2+qpair), lo[0], lo[1], lo[2], lo[3]);
					}
				}
			}
		}
		FenceProxyAsync();
		bool ok = true;
		if (tid == 0 && c >= 1) ok = MbarWaitBounded(bars+((c-1) & 1), (uint32_t)(((c-1) >> 1) & 1));
		if (__syncthreads_or(!ok)) { failed = true; break; }
		if (tid == 0) {
			FenceAfterSync();
			#pragma unroll
			for (int tile = 0; tile < kTiles; ++tile) {
				const uint32_t a = sA+tile*kTileBytes;
				if constexpr (kTf32) {
					#pragma unroll
					for (int ks = 0; ks < 2; ++ks)
						MmaTf32(tmem+tile*64, DescSw64(a+ks*32), DescSw64(sB+ks*32), (c > 0 || ks > 0) ? 1u : 0u);
				} else if (kSplit) {
					MmaBf16(tmem+tile*64, DescSw64(a), DescSw64(sB), c > 0 ? 1u : 0u);
					MmaBf16(tmem+tile*64, DescSw64(a), DescSw64(sB+32), 1u);
					MmaBf16(tmem+tile*64, DescSw64(a+32), DescSw64(sB), 1u);
				} else {
					#pragma unroll
					for (int ks = 0; ks < 2; ++ks)
						MmaBf16(tmem+tile*64, DescSw64(a+ks*32), DescSw64(sB+ks*32), (c > 0 || ks > 0) ? 1u : 0u);
				}
			}
			MmaCommit(bars+buf);
		}
		issued = c+1;
		// every thread has passed this chunk's barrier, so the chunk's basis buffer is free for chunk c + 2
		if (c+2 < kChunks) stage.Store(PhiF[buf], tid);
	}
	if (!failed)
		failed = __syncthreads_or(!MbarWaitBounded(bars+((kChunks-1) & 1), (uint32_t)(((kChunks-1) >> 1) & 1))) != 0;

	if (!failed) {
		// Epilogue as TangentTcKernel's, each warp taking one of the two a halves: warp -> (a half
		// warp >> 3, basis half (warp >> 2) & 1, TMEM lane quarter warp & 3).
		FenceAfterSync();
		const int bh = (warp >> 2) & 1, quarter = warp & 3, ah = warp >> 3;
		const int32_t* EB = element_blocks+(size_t)e*kMaxBasis*kMaxBasis;
		const int f = lane & 3;
		const int b = bh*32+quarter*8+(lane >> 2);
		float* row_base = values+(size_t)(2*h+(f & 1))*4;
		int blocks[2][8];
		#pragma unroll
		for (int g = 0; g < 8; ++g)
			#pragma unroll
			for (int p = 0; p < 2; ++p) {
				const int a = ah*32+4*g+(f & 2)+p;
				blocks[p][g] = (a < nen && b < nen) ? EB[a*kMaxBasis+b] : -1;
			}
		float v0[32], v1[32];
		const uint32_t lanes = (uint32_t)(quarter*32) << 16;
		TmemLoad32(tmem+lanes+bh*64+ah*32, v0);
		TmemLoad32(tmem+lanes+(2+bh)*64+ah*32, v1);
		#pragma unroll
		for (int g = 0; g < 8; ++g)
			#pragma unroll
			for (int p = 0; p < 2; ++p) {
				const float c00 = v0[4*g+p], c02 = v0[4*g+2+p], c10 = v1[4*g+p], c12 = v1[4*g+2+p];
				float o0 = 0.f, o1 = 0.f, o2 = 0.f, o3 = 0.f;
				#pragma unroll
				for (int r = 0; r < 4; ++r) {
					const int d = f ^ r;
					const float send = (d & 1) ? ((d & 2) ? c12 : c10) : ((d & 2) ? c02 : c00);
					const float got = r ? __shfl_xor_sync(0xffffffffu, send, r) : send;
					o0 = d == 0 ? got : o0; o1 = d == 1 ? got : o1;
					o2 = d == 2 ? got : o2; o3 = d == 3 ? got : o3;
				}
				if (blocks[p][g] >= 0) RedAdd4(row_base+(size_t)blocks[p][g]*16, o0, o1, o2, o3);
			}
	} else {
		if (tid == 0) atomicOr(status, 1);
		if (issued > 0) MbarWaitBounded(bars+((issued-1) & 1), (uint32_t)(((issued-1) >> 1) & 1));
	}
	FenceBeforeSync();
	__syncthreads();
	if (warp == 0) {
		FenceAfterSync();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTmemCols)
			: "memory");
	}
}

} // namespace

namespace {

// SMs of the current device (queried once per process).
int MultiprocessorCount()
{
	static int sms = 0;
	if (sms == 0) {
		int device = 0;
		CudaCheck(cudaGetDevice(&device), "device");
		CudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
	}
	return sms;
}

} // namespace

void LaunchTangentPoint(const DeviceMeshView& mesh, const double* phi, const double* qdata, const double* state,
	const double* previous, AssemblyParams params, float* coef, double* point_state, double* rhs, cudaStream_t stream)
{
	if (mesh.elements == 0) return;
	if (rhs == nullptr) Fail(-1, "tangent point kernel: the residual output is required");
	if (coef && point_state) Fail(-1, "tangent point kernel: coefficients or point state, not both");
	static bool configured = false;
	if (!configured) {
		CudaCheck(cudaFuncSetAttribute(TangentPointKernel<kPointResidual>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			kPtSmemBytes+16), "tangent point-kernel shared-memory attribute");
		CudaCheck(cudaFuncSetAttribute(TangentPointKernel<kPointCoefficients>,
			cudaFuncAttributeMaxDynamicSharedMemorySize, kPtSmemBytes+16), "tangent point-kernel shared-memory attribute");
		CudaCheck(cudaFuncSetAttribute(TangentPointKernel<kPointState>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			kPtSmemBytes+16), "tangent point-kernel shared-memory attribute");
		configured = true;
	}
	const unsigned grid = (unsigned)mesh.elements;
	const size_t bytes = kPtSmemBytes+16;
	if (coef)
		TangentPointKernel<kPointCoefficients><<<grid, kTcThreads, bytes, stream>>>(mesh, phi, qdata, state, previous,
			params, coef, nullptr, rhs);
	else if (point_state)
		TangentPointKernel<kPointState><<<grid, kTcThreads, bytes, stream>>>(mesh, phi, qdata, state, previous,
			params, nullptr, point_state, rhs);
	else
		TangentPointKernel<kPointResidual><<<grid, kTcThreads, bytes, stream>>>(mesh, phi, qdata, state, previous,
			params, nullptr, nullptr, rhs);
	LaunchCheck("TangentPointKernel");
}

namespace {

template <int kMode>
void StartTangentTc(unsigned ctas, const DeviceMeshView& mesh, const float* phi32, const float* coef,
	const int32_t* element_blocks, float* values, int* status, int lookahead, cudaStream_t stream)
{
	static bool configured = false;
	if (!configured) {
		CudaCheck(cudaFuncSetAttribute(TangentTcKernel<kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			kTcSmemBytes), "tensor-core tangent shared-memory attribute");
		configured = true;
	}
	TangentTcKernel<kMode><<<ctas, kTcThreads, kTcSmemBytes, stream>>>(mesh, phi32, coef, element_blocks, values,
		status, lookahead);
}

template <int kMode>
void StartTangentTcQuad(unsigned ctas, const DeviceMeshView& mesh, const float* phi32, const float* coef,
	const int32_t* element_blocks, float* values, int* status, cudaStream_t stream)
{
	static bool configured = false;
	if (!configured) {
		CudaCheck(cudaFuncSetAttribute(TangentTcQuadKernel<kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			kQSmemBytes), "element tensor-core tangent shared-memory attribute");
		configured = true;
	}
	TangentTcQuadKernel<kMode><<<ctas, kTcThreads, kQSmemBytes, stream>>>(mesh, phi32, coef, element_blocks, values,
		status);
}

template <int kMode>
void StartTangentTcFused(unsigned ctas, const DeviceMeshView& mesh, const double* phi, const double* qdata,
	const double* point_state, AssemblyParams params, const int32_t* element_blocks, float* values, int* status,
	int lookahead, cudaStream_t stream)
{
	static bool configured = false;
	if (!configured) {
		CudaCheck(cudaFuncSetAttribute(TangentTcFusedKernel<kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			kFusedSmemBytes), "fused tensor-core tangent shared-memory attribute");
		configured = true;
	}
	TangentTcFusedKernel<kMode><<<ctas, kFusedThreads, kFusedSmemBytes, stream>>>(mesh, phi, qdata, point_state,
		params, element_blocks, values, status, lookahead);
}

} // namespace

void LaunchTangentTcElement(const DeviceMeshView& mesh, const float* phi32, const float* coef,
	const int32_t* element_blocks, float* values, int* status, int operands, cudaStream_t stream)
{
	if (mesh.elements == 0) return;
	const unsigned ctas = (unsigned)std::min<long long>(mesh.elements, MultiprocessorCount());
	if (operands == TC_OPERANDS_SPLIT)
		StartTangentTcQuad<kModeSplit>(ctas, mesh, phi32, coef, element_blocks, values, status, stream);
	else if (operands == TC_OPERANDS_TF32)
		StartTangentTcQuad<kModeTf32>(ctas, mesh, phi32, coef, element_blocks, values, status, stream);
	else if (operands == TC_OPERANDS_BF16)
		StartTangentTcQuad<kModeBf16>(ctas, mesh, phi32, coef, element_blocks, values, status, stream);
	else
		Fail(-1, "tensor-core tangent: unknown operand organisation");
	LaunchCheck("TangentTcQuadKernel");
}

void LaunchTangentTc(const DeviceMeshView& mesh, const float* phi32, const float* coef,
	const int32_t* element_blocks, float* values, int* status, int operands, cudaStream_t stream)
{
	if (mesh.elements == 0) return;
	const long long ctas = 2LL*mesh.elements;
	if (ctas > 0x7fffffffLL) Fail(-7, "too many elements for one tangent launch");
	const int lookahead = 2*MultiprocessorCount();            // two CTAs per SM
	if (operands == TC_OPERANDS_SPLIT)
		StartTangentTc<kModeSplit>((unsigned)ctas, mesh, phi32, coef, element_blocks, values, status, lookahead, stream);
	else if (operands == TC_OPERANDS_TF32)
		StartTangentTc<kModeTf32>((unsigned)ctas, mesh, phi32, coef, element_blocks, values, status, lookahead, stream);
	else if (operands == TC_OPERANDS_BF16)
		StartTangentTc<kModeBf16>((unsigned)ctas, mesh, phi32, coef, element_blocks, values, status, lookahead, stream);
	else
		Fail(-1, "tensor-core tangent: unknown operand organisation");
	LaunchCheck("TangentTcKernel");
}

void LaunchTangentTcFused(const DeviceMeshView& mesh, const double* phi, const double* qdata,
	const double* point_state, AssemblyParams params, const int32_t* element_blocks, float* values, int* status,
	int operands, cudaStream_t stream)
{
	if (mesh.elements == 0) return;
	const long long ctas = 2LL*mesh.elements;
	if (ctas > 0x7fffffffLL) Fail(-7, "too many elements for one tangent launch");
	const int lookahead = MultiprocessorCount();              // one CTA per SM
	if (operands == TC_OPERANDS_SPLIT)
		StartTangentTcFused<kModeSplit>((unsigned)ctas, mesh, phi, qdata, point_state, params, element_blocks, values,
			status, lookahead, stream);
	else if (operands == TC_OPERANDS_TF32)
		StartTangentTcFused<kModeTf32>((unsigned)ctas, mesh, phi, qdata, point_state, params, element_blocks, values,
			status, lookahead, stream);
	else if (operands == TC_OPERANDS_BF16)
		StartTangentTcFused<kModeBf16>((unsigned)ctas, mesh, phi, qdata, point_state, params, element_blocks, values,
			status, lookahead, stream);
	else
		Fail(-1, "fused tensor-core tangent: unknown operand organisation");
	LaunchCheck("TangentTcFusedKernel");
}

} // namespace tfiga
