// Per-mesh precomputation on the device: Bernstein/extraction basis tables
// at the 4x4x4 Gauss points, the element -> block-CSR scatter map, and the
// boundary-face flow/traction coefficients.
//
// The arithmetic follows the reference's EvaluateBasis
// (solvers/cpu/include/TransportElement.hpp:118-206) and BuildGeometryKernel
// (solvers/cuda/include/IgaCudaKernels.cuh:61-111), but is organised for the
// GPU: one CTA per element with a thread per quadrature point, the Bernstein
// tensor product formed from 1D factors in registers, and only the trace of
// the physical Hessian kept (the VMS formulation uses the Laplacian alone:
// NavierStokesElement.hpp:206 and :251).  For a basis function with
// parametric derivatives g_a and h_ab,
//   Lap N = sum_ab h_ab (J^-1 J^-T)_ab + sum_c g_c m_c,
//   m_c   = -sum_{x,a,b} (d2x_x/dxi_a dxi_b) J^-1_{c x} (J^-1 J^-T)_ab,
// which is the trace of the reference's Hessian expression (:181-202).
#include "common.hpp"
#include "kernels.cuh"

namespace tfiga {
namespace {

__constant__ double kGaussPoint[4] = {0.06943184420297371, 0.33000947820757187,
	0.6699905217924281, 0.9305681557970262};
__constant__ double kGaussWeight[4] = {0.3478548451374539, 0.6521451548625461,
	0.6521451548625461, 0.3478548451374539};

__device__ __forceinline__ void Bernstein(double t, double b[4], double db[4], double d2b[4])
{
	const double s = 1.0-t;
	b[0] = s*s*s; b[1] = 3.0*s*s*t; b[2] = 3.0*s*t*t; b[3] = t*t*t;
	db[0] = -3.0*s*s; db[1] = 3.0-12.0*t+9.0*t*t; db[2] = 3.0*(2.0-3.0*t)*t; db[3] = 3.0*t*t;
	d2b[0] = 6.0*s; d2b[1] = -12.0+18.0*t; d2b[2] = 6.0-18.0*t; d2b[3] = 6.0*t;
}

// Determinant and cofactor inverse in the reference's term order
// (TransportElement.hpp:33-53).  Returns false for a singular Jacobian.
__device__ __forceinline__ bool Invert(const double a[3][3], double inv[3][3], double& det)
{
	det = a[0][0]*a[1][1]*a[2][2]+a[0][1]*a[1][2]*a[2][0]+a[0][2]*a[1][0]*a[2][1]
		-a[0][2]*a[1][1]*a[2][0]-a[0][0]*a[1][2]*a[2][1]-a[0][1]*a[1][0]*a[2][2];
	if (!isfinite(det) || fabs(det) < 1e-14) return false;
	inv[0][0] = (a[1][1]*a[2][2]-a[1][2]*a[2][1])/det;
	inv[0][1] = (a[2][1]*a[0][2]-a[0][1]*a[2][2])/det;
	inv[0][2] = (a[0][1]*a[1][2]-a[1][1]*a[0][2])/det;
	inv[1][0] = (a[2][0]*a[1][2]-a[1][0]*a[2][2])/det;
	inv[1][1] = (a[0][0]*a[2][2]-a[0][2]*a[2][0])/det;
	inv[1][2] = (a[1][0]*a[0][2]-a[0][0]*a[1][2])/det;
	inv[2][0] = (a[1][0]*a[2][1]-a[1][1]*a[2][0])/det;
	inv[2][1] = (a[0][1]*a[2][0]-a[0][0]*a[2][1])/det;
	inv[2][2] = (a[0][0]*a[1][1]-a[0][1]*a[1][0])/det;
	return true;
}

constexpr int kChunk = 16;   // basis functions staged per shared-memory pass

// Elements first + blockIdx.x; phi is indexed from `first` (table of NP padded functions per
// element), qdata by the global element id.
template <int NP>
__global__ void __launch_bounds__(64) BuildBasisKernel(DeviceMeshView mesh, int first, double* __restrict__ phi,
	double* __restrict__ qdata)
{
	const int e = first+blockIdx.x;
	const int q = threadIdx.x;
	__shared__ double X[192];
	__shared__ double tile[kFeatures][kQuad][kChunk+1];
	for (int i = q; i < 192; i += 64) X[i] = mesh.bezier_points[(size_t)e*192+i];
	__syncthreads();
	double bu[4], du[4], hu[4], bv[4], dv[4], hv[4], bw[4], dw[4], hw[4];
	Bernstein(kGaussPoint[q&3], bu, du, hu);
	Bernstein(kGaussPoint[(q>>2)&3], bv, dv, hv);
	Bernstein(kGaussPoint[q>>4], bw, dw, hw);
	double J[3][3] = {{0.0}}, S[3][6] = {{0.0}};
	for (int k = 0; k < 4; ++k)
		for (int j = 0; j < 4; ++j)
			for (int i = 0; i < 4; ++i) {
				const int p = i+4*j+16*k;
				const double g0 = du[i]*bv[j]*bw[k], g1 = bu[i]*dv[j]*bw[k], g2 = bu[i]*bv[j]*dw[k];
				const double s00 = hu[i]*bv[j]*bw[k], s01 = du[i]*dv[j]*bw[k], s02 = du[i]*bv[j]*dw[k];
				const double s11 = bu[i]*hv[j]*bw[k], s12 = bu[i]*dv[j]*dw[k], s22 = bu[i]*bv[j]*hw[k];
				for (int x = 0; x < 3; ++x) {
					const double c = X[p*3+x];
					J[x][0] += c*g0; J[x][1] += c*g1; J[x][2] += c*g2;
					S[x][0] += c*s00; S[x][1] += c*s01; S[x][2] += c*s02;
					S[x][3] += c*s11; S[x][4] += c*s12; S[x][5] += c*s22;
				}
			}
	double inv[3][3], det = 0.0;
	const bool ok = Invert(J, inv, det);
	const double weight = kGaussWeight[q&3]*kGaussWeight[(q>>2)&3]*kGaussWeight[q>>4]/8.0;
	double M2[3][3], m1[3] = {0.0, 0.0, 0.0};
	double* qd = qdata+((size_t)e*kQuad+q)*kQData;
	if (ok) {
		for (int a = 0; a < 3; ++a)
			for (int b = 0; b < 3; ++b) M2[a][b] = inv[a][0]*inv[b][0]+inv[a][1]*inv[b][1]+inv[a][2]*inv[b][2];
		const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
		for (int c = 0; c < 3; ++c) {
			double value = 0.0;
			for (int x = 0; x < 3; ++x)
				for (int s = 0; s < 6; ++s) {
					const double mult = ia[s] == ib[s] ? 1.0 : 2.0;
					value -= mult*S[x][s]*inv[c][x]*M2[ia[s]][ib[s]];
				}
			m1[c] = value;
		}
		// Stabilization metric (NavierStokesElement.hpp:121-139).
		double G[3][3], direction[3];
		for (int i = 0; i < 3; ++i) {
			direction[i] = inv[0][i]+inv[1][i]+inv[2][i];
			for (int j = 0; j < 3; ++j) G[i][j] = inv[0][i]*inv[0][j]+inv[1][i]*inv[1][j]+inv[2][i]*inv[2][j];
		}
		double gnorm = 0.0;
		for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) gnorm += G[i][j]*G[i][j];
		qd[0] = weight*det;
		qd[1] = G[0][0]; qd[2] = G[0][1]; qd[3] = G[0][2]; qd[4] = G[1][1]; qd[5] = G[1][2]; qd[6] = G[2][2];
		qd[7] = direction[0]*direction[0]+direction[1]*direction[1]+direction[2]*direction[2];
		qd[8] = gnorm;
	} else {
		for (int k = 0; k < 9; ++k) qd[k] = 0.0;
		for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) { M2[a][b] = 0.0; inv[a][b] = 0.0; }
	}
	qd[9] = 0.125*det;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	for (int chunk = 0; chunk < NP; chunk += kChunk) {
		for (int l = 0; l < kChunk; ++l) {
			const int a = chunk+l;
			double N = 0.0, g[3] = {0.0, 0.0, 0.0}, h[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
			if (a < nen && ok) {
				const int lo = mesh.extraction_offsets[begin+a], hi = mesh.extraction_offsets[begin+a+1];
				for (int k = lo; k < hi; ++k) {
					const int p = mesh.extraction_columns[k];
					const double c = mesh.extraction_values[k];
					const int i = p&3, j = (p>>2)&3, kk = p>>4;
					N += c*bu[i]*bv[j]*bw[kk];
					g[0] += c*du[i]*bv[j]*bw[kk]; g[1] += c*bu[i]*dv[j]*bw[kk]; g[2] += c*bu[i]*bv[j]*dw[kk];
					h[0] += c*hu[i]*bv[j]*bw[kk]; h[1] += c*du[i]*dv[j]*bw[kk]; h[2] += c*du[i]*bv[j]*dw[kk];
					h[3] += c*bu[i]*hv[j]*bw[kk]; h[4] += c*bu[i]*dv[j]*dw[kk]; h[5] += c*bu[i]*bv[j]*hw[kk];
				}
			}
			tile[0][q][l] = N;
			for (int d = 0; d < 3; ++d) tile[1+d][q][l] = g[0]*inv[0][d]+g[1]*inv[1][d]+g[2]*inv[2][d];
			tile[4][q][l] = h[0]*M2[0][0]+2.0*h[1]*M2[0][1]+2.0*h[2]*M2[0][2]+h[3]*M2[1][1]
				+2.0*h[4]*M2[1][2]+h[5]*M2[2][2]+g[0]*m1[0]+g[1]*m1[1]+g[2]*m1[2];
		}
		__syncthreads();
		// Coalesced write-out: kChunk consecutive basis entries per (feature, point).
		for (int idx = q; idx < kFeatures*kQuad*kChunk; idx += 64) {
			const int l = idx%kChunk, qq = (idx/kChunk)%kQuad, t = idx/(kChunk*kQuad);
			phi[(((size_t)(e-first)*kFeatures+t)*kQuad+qq)*NP+chunk+l] = tile[t][qq][l];
		}
		__syncthreads();
	}
}

// Block index of every (a, b) basis pair of every element, by binary search
// of the sorted block row (FindBlock, SparseKernels.cuh:13-23), done once.
template <int NP>
__global__ void ElementBlocksKernel(DeviceMeshView mesh, DevicePatternView pattern, int first,
	int32_t* __restrict__ out)
{
	const int e = first+blockIdx.x;
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	for (int pair = threadIdx.x; pair < NP*NP; pair += blockDim.x) {
		const int a = pair/NP, b = pair%NP;
		int block = -1;
		if (a < nen && b < nen) {
			const int row = mesh.connectivity[begin+a], column = mesh.connectivity[begin+b];
			const int end = pattern.row_offsets[row+1];
			int first = pattern.row_offsets[row], last = end;
			while (first < last) {
				const int middle = first+(last-first)/2;
				if (pattern.columns[middle] < column) first = middle+1;
				else last = middle;
			}
			block = first < end && pattern.columns[first] == column ? first : -1;
		}
		out[(size_t)(e-first)*NP*NP+pair] = block;
	}
}

// Face tables of the 4x4 surface rule (BoundaryFlow.hpp:175-180).
__constant__ int kFixedAxis[6] = {2, 1, 0, 1, 0, 2};
__constant__ int kVaryingAxes[6][2] = {{0, 1}, {0, 2}, {1, 2}, {0, 2}, {1, 2}, {0, 1}};
__constant__ double kFixedValue[6] = {0.0, 0.0, 1.0, 1.0, 0.0, 1.0};
__constant__ double kOutwardSign[6] = {-1.0, -1.0, 1.0, 1.0, -1.0, 1.0};

// F[a][c] with flow = sum_a F[a].u_a and traction(p) = -p F (BoundaryFlow.hpp:165-200, 445-475).
template <int NP>
__global__ void __launch_bounds__(64) FaceCoefficientsKernel(DeviceMeshView mesh, const int32_t* face_element,
	const int32_t* face_index, double* __restrict__ face_coef)
{
	const int face_id = blockIdx.x;
	const int e = face_element[face_id];
	const int face = face_index[face_id];
	__shared__ double X[192];
	__shared__ double B[16][3][4];
	__shared__ double scale[16][3];
	for (int i = threadIdx.x; i < 192; i += 64) X[i] = mesh.bezier_points[(size_t)e*192+i];
	__syncthreads();
	if (threadIdx.x < 16) {
		const int s = threadIdx.x, qi = s/4, qj = s%4;
		double coordinate[3] = {0.0, 0.0, 0.0};
		coordinate[kFixedAxis[face]] = kFixedValue[face];
		coordinate[kVaryingAxes[face][0]] = kGaussPoint[qi];
		coordinate[kVaryingAxes[face][1]] = kGaussPoint[qj];
		double b[3][4], db[3][4], h[4];
		for (int d = 0; d < 3; ++d) Bernstein(coordinate[d], b[d], db[d], h);
		double J[3][3] = {{0.0}};
		for (int k = 0; k < 4; ++k)
			for (int j = 0; j < 4; ++j)
				for (int i = 0; i < 4; ++i) {
					const int p = i+4*j+16*k;
					const double g0 = db[0][i]*b[1][j]*b[2][k], g1 = b[0][i]*db[1][j]*b[2][k], g2 = b[0][i]*b[1][j]*db[2][k];
					for (int x = 0; x < 3; ++x) {
						J[x][0] += X[p*3+x]*g0; J[x][1] += X[p*3+x]*g1; J[x][2] += X[p*3+x]*g2;
					}
				}
		double inv[3][3], det = 0.0;
		const bool ok = Invert(J, inv, det);
		const double w = kOutwardSign[face]*kGaussWeight[qi]*kGaussWeight[qj]*2.0*(0.125*det);
		for (int c = 0; c < 3; ++c) scale[s][c] = ok ? w*inv[kFixedAxis[face]][c] : 0.0;
		for (int d = 0; d < 3; ++d) for (int i = 0; i < 4; ++i) B[s][d][i] = b[d][i];
	}
	__syncthreads();
	const int begin = mesh.element_offsets[e];
	const int nen = mesh.element_offsets[e+1]-begin;
	for (int a = threadIdx.x; a < NP; a += blockDim.x) {
		double F[3] = {0.0, 0.0, 0.0};
		if (a < nen) {
			const int lo = mesh.extraction_offsets[begin+a], hi = mesh.extraction_offsets[begin+a+1];
			for (int s = 0; s < 16; ++s) {
				double N = 0.0;
				for (int k = lo; k < hi; ++k) {
					const int p = mesh.extraction_columns[k];
					N += mesh.extraction_values[k]*B[s][0][p&3]*B[s][1][(p>>2)&3]*B[s][2][p>>4];
				}
				for (int c = 0; c < 3; ++c) F[c] += scale[s][c]*N;
			}
		}
		for (int c = 0; c < 3; ++c) face_coef[((size_t)face_id*NP+a)*3+c] = F[c];
	}
}

} // namespace

void LaunchBuildBasis(const DeviceMeshView& mesh, double* phi, double* qdata, cudaStream_t stream)
{
	if (mesh.elements == 0) return;
	BuildBasisKernel<kMaxBasis><<<mesh.elements, 64, 0, stream>>>(mesh, 0, phi, qdata);
	LaunchCheck("BuildBasisKernel");
}

void LaunchBuildBasisLarge(const DeviceMeshView& mesh, int first, int count, double* phi, double* qdata,
	cudaStream_t stream)
{
	if (count == 0) return;
	BuildBasisKernel<kMaxBasisLarge><<<count, 64, 0, stream>>>(mesh, first, phi, qdata);
	LaunchCheck("BuildBasisKernel<80>");
}

void LaunchElementBlocks(const DeviceMeshView& mesh, const DevicePatternView& pattern, int32_t* element_blocks,
	cudaStream_t stream)
{
	if (mesh.elements == 0) return;
	ElementBlocksKernel<kMaxBasis><<<mesh.elements, 256, 0, stream>>>(mesh, pattern, 0, element_blocks);
	LaunchCheck("ElementBlocksKernel");
}

void LaunchElementBlocksLarge(const DeviceMeshView& mesh, const DevicePatternView& pattern, int first, int count,
	int32_t* element_blocks, cudaStream_t stream)
{
	if (count == 0) return;
	ElementBlocksKernel<kMaxBasisLarge><<<count, 256, 0, stream>>>(mesh, pattern, first, element_blocks);
	LaunchCheck("ElementBlocksKernel<80>");
}

void LaunchFaceCoefficients(const DeviceMeshView& mesh, int faces, const int32_t* face_element,
	const int32_t* face_index, double* face_coef, int stride, cudaStream_t stream)
{
	if (faces == 0) return;
	if (stride == kMaxBasis)
		FaceCoefficientsKernel<kMaxBasis><<<faces, 64, 0, stream>>>(mesh, face_element, face_index, face_coef);
	else if (stride == kMaxBasisLarge)
		FaceCoefficientsKernel<kMaxBasisLarge><<<faces, 64, 0, stream>>>(mesh, face_element, face_index, face_coef);
	else
		Fail(-1, "face coefficient stride must be 64 or 80");
	LaunchCheck("FaceCoefficientsKernel");
}

} // namespace tfiga
