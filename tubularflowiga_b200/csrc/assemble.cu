// FP64 VMS Navier-Stokes element assembly with the exact Newton tangent.
//
// Formulation: the reference's BuildNavierStokesElementFromPreparedPoints
// (solvers/cpu/include/NavierStokesElement.hpp:149-317, LegacyBodyFitted
// weak form, zero body force).  Its residual is the one the reference GPU
// kernel assembles (solvers/cuda/include/IgaCudaKernels.cuh:360-379); its
// tangent is the exact derivative (NavierStokesElement.hpp:244-312), not the
// frozen-tau tangent of the reference GPU kernel (IgaCudaKernels.cuh:380-396).
//
// Organisation.  At each quadrature point q every term of the tangent is a
// product (test feature s of N_a) x (trial feature t of N_b) with
// s in {N, dN/dx, dN/dy, dN/dz} and t in {N, dN/dx, dN/dy, dN/dz, Lap N}, so
//   K^{if}_{ab} = sum_q sum_s Psi_s(a,q) * G^{if}_s(b,q),
//   G^{if}_s(b,q) = measure_q * sum_t M_q^{if}[s][t] Phi_t(b,q),
// a GEMM of K = 64 points x 4 test features.  One CTA owns one element and one
// row field i; it builds the 4x5 coefficient matrices M_q^{i f} once per point,
// forms G in shared memory chunk by chunk and accumulates the 64 x 256 block
// (a, (b, f)) in registers with an 8x8 FP64 tile per thread, then adds the
// result into block CSR through the precomputed element -> block map.
#include "common.hpp"
#include "kernels.cuh"
#include "l2_prefetch.cuh"
#include "vms_point.cuh"

namespace tfiga {
namespace {

constexpr int kThreads = 256;
constexpr int kChunkPoints = 8;                 // quadrature points per GEMM chunk
constexpr int kChunkK = kChunkPoints*4;         // GEMM depth per chunk
template <int NP>
__global__ void __launch_bounds__(kThreads, 1) AssembleKernel(DeviceMeshView mesh, const double* __restrict__ phi,
	const double* __restrict__ qdata, const int32_t* __restrict__ element_blocks, const double* __restrict__ state,
	const double* __restrict__ previous, AssemblyParams prm, double* __restrict__ values, double* __restrict__ rhs)
{
	static_assert(NP == 64, "the register tiling assumes 64 padded basis functions");
	extern __shared__ __align__(16) double sm[];
	double* U = sm;                          // [NP][4] current state
	double* Up = U+NP*4;                     // [NP][4] previous velocity
	double* QS = Up+NP*4;                    // [64][kQS]
	double* Msm = QS+kQuad*kQS;              // [64][kCoef]
	double* RC = Msm+kQuad*kCoef;            // [64][4]
	double* Psi = RC+kQuad*4;                // [kChunkK][NP]
	double* Gs = Psi+kChunkK*NP;             // [kChunkK][4*NP]

	const int e = blockIdx.x >> 2;
	const int row = blockIdx.x & 3;
	const int tid = threadIdx.x;
	const int warp = tid >> 5, lane = tid & 31;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	const double* P = phi+(size_t)e*kFeatures*kQuad*NP;
	if (tid == 0) PrefetchL2(P, kFeatures*kQuad*NP*8);

	// 1. Gather nodal state.
	for (int a = tid; a < NP; a += kThreads) {
		double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, p0 = 0.0, p1 = 0.0, p2 = 0.0;
		if (a < nen) {
			const size_t node = (size_t)mesh.connectivity[begin+a];
			const double2 x01 = *reinterpret_cast<const double2*>(state+4*node);
			const double2 x23 = *reinterpret_cast<const double2*>(state+4*node+2);
			s0 = x01.x; s1 = x01.y; s2 = x23.x; s3 = x23.y;
			if (prm.dt > 0.0) {
				const double2 y01 = *reinterpret_cast<const double2*>(previous+4*node);
				p0 = y01.x; p1 = y01.y; p2 = previous[4*node+2];
			}
		}
		U[a*4] = s0; U[a*4+1] = s1; U[a*4+2] = s2; U[a*4+3] = s3;
		Up[a*4] = p0; Up[a*4+1] = p1; Up[a*4+2] = p2; Up[a*4+3] = 0.0;
	}
	__syncthreads();

	// 2. State at every point: a warp per point, lanes over basis functions.
	for (int q = warp; q < kQuad; q += kThreads/32) {
		double v[22];
		#pragma unroll
		for (int k = 0; k < 22; ++k) v[k] = 0.0;
		for (int a = lane; a < NP; a += 32) {
			const double n = P[(0*kQuad+q)*NP+a];
			const double g0 = P[(1*kQuad+q)*NP+a], g1 = P[(2*kQuad+q)*NP+a], g2 = P[(3*kQuad+q)*NP+a];
			const double l = P[(4*kQuad+q)*NP+a];
			const double u0 = U[a*4], u1 = U[a*4+1], u2 = U[a*4+2], u3 = U[a*4+3];
			v[0] += n*u0; v[1] += n*u1; v[2] += n*u2; v[3] += n*u3;
			v[4] += n*Up[a*4]; v[5] += n*Up[a*4+1]; v[6] += n*Up[a*4+2];
			const double uf[4] = {u0, u1, u2, u3};
			#pragma unroll
			for (int f = 0; f < 4; ++f) { v[7+3*f] += g0*uf[f]; v[8+3*f] += g1*uf[f]; v[9+3*f] += g2*uf[f]; }
			v[19] += l*u0; v[20] += l*u1; v[21] += l*u2;
		}
		#pragma unroll
		for (int k = 0; k < 22; ++k)
			#pragma unroll
			for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
		if (lane == 0)
			#pragma unroll
			for (int k = 0; k < 22; ++k) QS[q*kQS+k] = v[k];
	}
	__syncthreads();

	// 3. Coefficients of this CTA's row field at every point.
	if (tid < kQuad) {
		PointState S;
		const double* s = QS+tid*kQS;
		for (int c = 0; c < 3; ++c) {
			S.u[c] = s[kU+c]; S.up[c] = s[kUp+c]; S.lap[c] = s[kLap+c]; S.gp[c] = s[kGrad+9+c];
			for (int d = 0; d < 3; ++d) S.gv[c][d] = s[kGrad+3*c+d];
		}
		S.p = s[kP];
		RowCoefficients(row, S, qdata+((size_t)e*kQuad+tid)*kQData, prm, Msm+tid*kCoef, RC+tid*4);
	}
	__syncthreads();

	// 4. Residual of row field `row` (rhs holds -r).
	if (rhs != nullptr && tid < nen) {
		double r = 0.0;
		for (int q = 0; q < kQuad; ++q)
			#pragma unroll
			for (int s = 0; s < 4; ++s) r += P[(s*kQuad+q)*NP+tid]*RC[q*4+s];
		atomicAdd(rhs+4*(size_t)mesh.connectivity[begin+tid]+row, r);
	}
	if (values == nullptr) return;

	// 5. Tangent: acc[a-tile][col-tile] over K = 64 points x 4 test features.
	double acc[8][8];
	#pragma unroll
	for (int i = 0; i < 8; ++i)
		#pragma unroll
		for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
	const int ta = warp, tb = lane;
	for (int qc = 0; qc < kQuad; qc += kChunkPoints) {
		for (int idx = tid; idx < kChunkK*NP; idx += kThreads) {
			const int k = idx/NP, a = idx%NP;
			Psi[idx] = P[((k&3)*kQuad+qc+(k>>2))*NP+a];
		}
		{
			const int c = tid, b = c >> 2, f = c & 3;   // column (b, f) of G
			#pragma unroll 2
			for (int qq = 0; qq < kChunkPoints; ++qq) {
				const int q = qc+qq;
				double ph[5];
				#pragma unroll
				for (int t = 0; t < 5; ++t) ph[t] = P[(t*kQuad+q)*NP+b];
				const double* Mq = Msm+q*kCoef+f*20;
				#pragma unroll
				for (int s = 0; s < 4; ++s)
					Gs[(qq*4+s)*(4*NP)+c] = Mq[s*5]*ph[0]+Mq[s*5+1]*ph[1]+Mq[s*5+2]*ph[2]+Mq[s*5+3]*ph[3]
						+Mq[s*5+4]*ph[4];
			}
		}
		__syncthreads();
		#pragma unroll 2
		for (int k = 0; k < kChunkK; ++k) {
			const double2* pr = reinterpret_cast<const double2*>(Psi+k*NP+ta*8);
			const double2 p0 = pr[0], p1 = pr[1], p2 = pr[2], p3 = pr[3];
			const double* gr = Gs+k*(4*NP)+2*tb;
			const double2 g0 = *reinterpret_cast<const double2*>(gr);
			const double2 g1 = *reinterpret_cast<const double2*>(gr+64);
			const double2 g2 = *reinterpret_cast<const double2*>(gr+128);
			const double2 g3 = *reinterpret_cast<const double2*>(gr+192);
			const double pa[8] = {p0.x, p0.y, p1.x, p1.y, p2.x, p2.y, p3.x, p3.y};
			const double gb[8] = {g0.x, g0.y, g1.x, g1.y, g2.x, g2.y, g3.x, g3.y};
			#pragma unroll
			for (int i = 0; i < 8; ++i)
				#pragma unroll
				for (int j = 0; j < 8; ++j) acc[i][j] = fma(pa[i], gb[j], acc[i][j]);
		}
		__syncthreads();
	}

	// 6. Scatter-add into block CSR: column 2*tb + 64*j + s is (b = 16j + tb/2, f = 2(tb&1) + s).
	const int32_t* EB = element_blocks+(size_t)e*NP*NP;
	const int f0 = 2*(tb & 1);
	#pragma unroll
	for (int i = 0; i < 8; ++i) {
		const int a = ta*8+i;
		if (a >= nen) continue;
		#pragma unroll
		for (int j = 0; j < 4; ++j) {
			const int b = 16*j+(tb >> 1);
			const int block = b < nen ? EB[a*NP+b] : -1;
			if (block < 0) continue;
			double* dst = values+(size_t)block*16+row*4+f0;
			atomicAdd(dst, acc[i][2*j]);
			atomicAdd(dst+1, acc[i][2*j+1]);
		}
	}
}

constexpr size_t SharedBytes(int np)
{
	return sizeof(double)*(size_t)(np*4+np*4+kQuad*kQS+kQuad*kCoef+kQuad*4+kChunkK*np+kChunkK*4*np);
}

// Elements with 65..80 basis functions (rare: the spline extraction's extraordinary vertices), from
// their 80-wide tables.  CTA per (element, row field), 256 threads: nodal state, point state (warp per
// point), the row field's coefficients M_q and residual coefficients (thread per point), the residual
// (thread per basis function), then the tangent K^{if}_{ab} = sum_q sum_s Psi_s(a, q) sum_t
// M_q^{if}[s][t] Phi_t(b, q) with one task per (a, eight consecutive b): per point the task folds its
// test function into w[f][t] = sum_s Psi_s(a, q) M_q[f][s][t] and adds w[f][.] Phi_.(b, q) for its b.
// FP64 throughout; the sums are added into FP64 or FP32 block storage.
constexpr int kLargeThreads = 256;
constexpr int kLargeBGroup = 8;

constexpr size_t LargeSharedBytes()
{
	return sizeof(double)*(size_t)(kMaxBasisLarge*4*2+kQuad*kQS+kQuad*kCoef+kQuad*4);
}

template <class T>
__global__ void __launch_bounds__(kLargeThreads) AssembleLargeKernel(DeviceMeshView mesh, int first,
	const double* __restrict__ phi, const double* __restrict__ qdata, const int32_t* __restrict__ element_blocks,
	const double* __restrict__ state, const double* __restrict__ previous, AssemblyParams prm,
	T* __restrict__ values, double* __restrict__ rhs)
{
	constexpr int NP = kMaxBasisLarge;
	extern __shared__ __align__(16) double lsm[];
	double* U = lsm;                          // [NP][4]
	double* Up = U+NP*4;                      // [NP][4]
	double* QS = Up+NP*4;                     // [64][kQS]
	double* Msm = QS+kQuad*kQS;               // [64][kCoef]
	double* RC = Msm+kQuad*kCoef;             // [64][4]
	const int e = first+(blockIdx.x >> 2);
	const int row = blockIdx.x & 3;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	const double* P = phi+(size_t)(e-first)*kFeatures*kQuad*NP;

	for (int a = tid; a < NP; a += kLargeThreads) {
		double s[4] = {0.0, 0.0, 0.0, 0.0}, p[3] = {0.0, 0.0, 0.0};
		if (a < nen) {
			const size_t node = (size_t)mesh.connectivity[begin+a];
			for (int f = 0; f < 4; ++f) s[f] = state[4*node+f];
			if (prm.dt > 0.0) for (int f = 0; f < 3; ++f) p[f] = previous[4*node+f];
		}
		for (int f = 0; f < 4; ++f) U[a*4+f] = s[f];
		for (int f = 0; f < 3; ++f) Up[a*4+f] = p[f];
		Up[a*4+3] = 0.0;
	}
	__syncthreads();
	for (int q = warp; q < kQuad; q += kLargeThreads/32) {
		double v[22];
		#pragma unroll
		for (int k = 0; k < 22; ++k) v[k] = 0.0;
		for (int a = lane; a < NP; a += 32) {
			const double n = P[(0*kQuad+q)*NP+a];
			const double g0 = P[(1*kQuad+q)*NP+a], g1 = P[(2*kQuad+q)*NP+a], g2 = P[(3*kQuad+q)*NP+a];
			const double l = P[(4*kQuad+q)*NP+a];
			const double uf[4] = {U[a*4], U[a*4+1], U[a*4+2], U[a*4+3]};
			v[0] += n*uf[0]; v[1] += n*uf[1]; v[2] += n*uf[2]; v[3] += n*uf[3];
			v[4] += n*Up[a*4]; v[5] += n*Up[a*4+1]; v[6] += n*Up[a*4+2];
			#pragma unroll
			for (int f = 0; f < 4; ++f) { v[7+3*f] += g0*uf[f]; v[8+3*f] += g1*uf[f]; v[9+3*f] += g2*uf[f]; }
			v[19] += l*uf[0]; v[20] += l*uf[1]; v[21] += l*uf[2];
		}
		#pragma unroll
		for (int k = 0; k < 22; ++k)
			#pragma unroll
			for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
		if (lane == 0)
			#pragma unroll
			for (int k = 0; k < 22; ++k) QS[q*kQS+k] = v[k];
	}
	__syncthreads();
	if (tid < kQuad) {
		PointState S;
		const double* s = QS+tid*kQS;
		for (int c = 0; c < 3; ++c) {
			S.u[c] = s[kU+c]; S.up[c] = s[kUp+c]; S.lap[c] = s[kLap+c]; S.gp[c] = s[kGrad+9+c];
			for (int d = 0; d < 3; ++d) S.gv[c][d] = s[kGrad+3*c+d];
		}
		S.p = s[kP];
		RowCoefficients(row, S, qdata+((size_t)e*kQuad+tid)*kQData, prm, Msm+tid*kCoef, RC+tid*4);
	}
	__syncthreads();
	if (rhs != nullptr)
		for (int a = tid; a < nen; a += kLargeThreads) {
			double r = 0.0;
			for (int q = 0; q < kQuad; ++q)
				#pragma unroll
				for (int s = 0; s < 4; ++s) r += P[(s*kQuad+q)*NP+a]*RC[q*4+s];
			atomicAdd(rhs+4*(size_t)mesh.connectivity[begin+a]+row, r);
		}
	if (values == nullptr) return;
	const int32_t* EB = element_blocks+(size_t)(e-first)*NP*NP;
	constexpr int kGroups = NP/kLargeBGroup;
	for (int task = tid; task < NP*kGroups; task += kLargeThreads) {
		const int a = task/kGroups, b0 = (task%kGroups)*kLargeBGroup;
		if (a >= nen || b0 >= nen) continue;
		double acc[kLargeBGroup][4];
		#pragma unroll
		for (int j = 0; j < kLargeBGroup; ++j)
			#pragma unroll
			for (int f = 0; f < 4; ++f) acc[j][f] = 0.0;
		for (int q = 0; q < kQuad; ++q) {
			double psi[4];
			#pragma unroll
			for (int s = 0; s < 4; ++s) psi[s] = P[(s*kQuad+q)*NP+a];
			const double* Mq = Msm+q*kCoef;
			double w[4][5];
			#pragma unroll
			for (int f = 0; f < 4; ++f)
				#pragma unroll
				for (int t = 0; t < 5; ++t)
					w[f][t] = psi[0]*Mq[f*20+t]+psi[1]*Mq[f*20+5+t]+psi[2]*Mq[f*20+10+t]+psi[3]*Mq[f*20+15+t];
			#pragma unroll
			for (int j = 0; j < kLargeBGroup; ++j) {
				double ph[5];
				#pragma unroll
				for (int t = 0; t < 5; ++t) ph[t] = P[(t*kQuad+q)*NP+b0+j];
				#pragma unroll
				for (int f = 0; f < 4; ++f)
					acc[j][f] += w[f][0]*ph[0]+w[f][1]*ph[1]+w[f][2]*ph[2]+w[f][3]*ph[3]+w[f][4]*ph[4];
			}
		}
		#pragma unroll
		for (int j = 0; j < kLargeBGroup; ++j) {
			const int b = b0+j;
			if (b >= nen) break;
			const int block = EB[a*NP+b];
			if (block < 0) continue;
			T* dst = values+(size_t)block*16+row*4;
			#pragma unroll
			for (int f = 0; f < 4; ++f) atomicAdd(dst+f, (T)acc[j][f]);
		}
	}
}

} // namespace

void LaunchAssemble(const DeviceMeshView& mesh, const double* phi, const double* qdata,
	const int32_t* element_blocks, const double* state, const double* previous, AssemblyParams params,
	double* values, double* rhs, cudaStream_t stream)
{
	if (mesh.elements == 0) return;
	constexpr size_t bytes = SharedBytes(kMaxBasis);
	static bool configured = false;
	if (!configured) {
		CudaCheck(cudaFuncSetAttribute(AssembleKernel<kMaxBasis>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)bytes), "assembly shared-memory attribute");
		configured = true;
	}
	const long long ctas = 4LL*mesh.elements;
	if (ctas > 0x7fffffffLL) Fail(-7, "too many elements for one assembly launch");
	AssembleKernel<kMaxBasis><<<(unsigned)ctas, kThreads, bytes, stream>>>(mesh, phi, qdata, element_blocks,
		state, previous, params, values, rhs);
	LaunchCheck("AssembleKernel");
}

template <class T>
void LaunchAssembleLarge(const DeviceMeshView& mesh, int first, int count, const double* phi, const double* qdata,
	const int32_t* element_blocks, const double* state, const double* previous, AssemblyParams params, T* values,
	double* rhs, cudaStream_t stream)
{
	if (count == 0 || (values == nullptr && rhs == nullptr)) return;
	constexpr size_t bytes = LargeSharedBytes();
	static bool configured = false;
	if (!configured) {
		CudaCheck(cudaFuncSetAttribute(AssembleLargeKernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)bytes), "large-element assembly shared-memory attribute");
		configured = true;
	}
	AssembleLargeKernel<T><<<4u*(unsigned)count, kLargeThreads, bytes, stream>>>(mesh, first, phi, qdata,
		element_blocks, state, previous, params, values, rhs);
	LaunchCheck("AssembleLargeKernel");
}

template void LaunchAssembleLarge<double>(const DeviceMeshView&, int, int, const double*, const double*,
	const int32_t*, const double*, const double*, AssemblyParams, double*, double*, cudaStream_t);
template void LaunchAssembleLarge<float>(const DeviceMeshView&, int, int, const double*, const double*,
	const int32_t*, const double*, const double*, AssemblyParams, float*, double*, cudaStream_t);

} // namespace tfiga
