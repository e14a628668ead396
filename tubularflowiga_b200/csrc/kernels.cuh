// Device data layout and kernel entry points of the B200 Navier-Stokes path.
//
// Per-element basis tables (built once per mesh, FP64):
//   phi[((e*5 + t)*64 + q)*NP + a]   t = 0: N, 1..3: dN/dx_t, 4: Laplacian of N
//   qdata[(e*64 + q)*QD + k]          k = 0 measure (w_q/8 * det), 1..6 metric G =
//                                     J^-T J^-1 (00,01,02,11,12,22), 7 |sum_j J^-1_j.|^2,
//                                     8 |G|_F^2, 9 det/8
// Block-CSR matrix: values[block*16 + 4*i + f] (row field i, column field f),
// node-major vectors value[4*node + field].
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tfiga {

constexpr int kQuad = 64;       // 4x4x4 Gauss points
constexpr int kFeatures = 5;    // N, dN/dx, dN/dy, dN/dz, Laplacian
constexpr int kQData = 10;
constexpr int kMaxBasis = 64;   // padded basis count NP of the device tables
// Elements with 65..80 basis functions (the reference's limit, solvers/cuda/include/DeviceMesh.hpp:55-56)
// keep their own tables padded to 80 and go through the large-element kernels.
constexpr int kMaxBasisLarge = 80;

struct DeviceMeshView {
	int nodes = 0;
	int elements = 0;
	const int32_t* element_offsets = nullptr;
	const int32_t* connectivity = nullptr;
	const int32_t* extraction_offsets = nullptr;
	const uint8_t* extraction_columns = nullptr;
	const double* extraction_values = nullptr;
	const double* bezier_points = nullptr;
};

struct DevicePatternView {
	int nodes = 0;
	long long blocks = 0;
	const int32_t* row_offsets = nullptr;
	const int32_t* columns = nullptr;
	const int32_t* diagonal = nullptr;
};

struct AssemblyParams {
	double density;
	double viscosity;
	double dt;
};

// ---- basis.cu -----------------------------------------------------------
// Tables of the first mesh.elements elements (64 padded functions each).
void LaunchBuildBasis(const DeviceMeshView& mesh, double* phi, double* qdata, cudaStream_t stream);
void LaunchElementBlocks(const DeviceMeshView& mesh, const DevicePatternView& pattern, int32_t* element_blocks,
	cudaStream_t stream);
// Tables of the elements [first, first + count) with 80 padded functions: phi and element_blocks
// indexed from `first`, qdata by the global element id.
void LaunchBuildBasisLarge(const DeviceMeshView& mesh, int first, int count, double* phi, double* qdata,
	cudaStream_t stream);
void LaunchElementBlocksLarge(const DeviceMeshView& mesh, const DevicePatternView& pattern, int first, int count,
	int32_t* element_blocks, cudaStream_t stream);
// face_coef[face][stride][3] with stride 64 or 80 (the widest element of the mesh).
void LaunchFaceCoefficients(const DeviceMeshView& mesh, int faces, const int32_t* face_element,
	const int32_t* face_index, double* face_coef, int stride, cudaStream_t stream);

// ---- assemble.cu --------------------------------------------------------
// Exact-tangent VMS assembly: jacobian values (may be null: residual only) and
// rhs (= -r) are ADDED to.
void LaunchAssemble(const DeviceMeshView& mesh, const double* phi, const double* qdata,
	const int32_t* element_blocks, const double* state, const double* previous, AssemblyParams params,
	double* values, double* rhs, cudaStream_t stream);
// The same element (FP64 point state, coefficients, residual and exact tangent) for the elements
// [first, first + count) with up to 80 basis functions, from their 80-wide tables; values (FP64 or
// FP32 storage, may be null: residual only) and rhs (may be null: tangent only) are ADDED to.
template <class T>
void LaunchAssembleLarge(const DeviceMeshView& mesh, int first, int count, const double* phi, const double* qdata,
	const int32_t* element_blocks, const double* state, const double* previous, AssemblyParams params, T* values,
	double* rhs, cudaStream_t stream);

// ---- tangent_tc.cu -----------------------------------------------------
// Tensor-core tangent in two launches.  LaunchTangentPoint: FP64 point state,
// the coefficients of all four row fields into coef (workspace of elements x 4
// x 80 x 64 floats; null: residual only) and the FP64 residual ADDED into rhs
// (= -r).
// LaunchTangentTc: the tangent contracted on the tcgen05 tensor cores from
// coef and phi32 (the FP32 copy of phi, Mesh::phi32), FP32 accumulation, ADDED
// into the FP32 values; status bit 1 set if an MMA completion wait expired.
// operands: TC_OPERANDS_BF16, TC_OPERANDS_SPLIT (hi + lo BF16) or TC_OPERANDS_TF32.
// point_state (elements x 64 x 22 doubles, may be null): the point state for LaunchTangentTcFused
// instead of the coefficients (coef and point_state are not both given).
void LaunchTangentPoint(const DeviceMeshView& mesh, const double* phi, const double* qdata, const double* state,
	const double* previous, AssemblyParams params, float* coef, double* point_state, double* rhs,
	cudaStream_t stream);
enum : int { TC_OPERANDS_BF16 = 0, TC_OPERANDS_SPLIT = 1, TC_OPERANDS_TF32 = 2 };
void LaunchTangentTc(const DeviceMeshView& mesh, const float* phi32, const float* coef,
	const int32_t* element_blocks, float* values, int* status, int operands, cudaStream_t stream);
// The same contraction with one persistent CTA per SM taking whole elements (all four row fields, the
// basis chunk staged once per element; 512 TMEM columns, so one CTA per SM).
void LaunchTangentTcElement(const DeviceMeshView& mesh, const float* phi32, const float* coef,
	const int32_t* element_blocks, float* values, int* status, int operands, cudaStream_t stream);
// The same contraction with the coefficients made in the kernel from the stored point state and the
// basis staged from the FP64 tables (no coefficient array, no FP32 copy of the tables).
void LaunchTangentTcFused(const DeviceMeshView& mesh, const double* phi, const double* qdata,
	const double* point_state, AssemblyParams params, const int32_t* element_blocks, float* values, int* status,
	int operands, cudaStream_t stream);

// ---- sparse.cu ----------------------------------------------------------
// Matrix values are FP64 or FP32 (T = double / float); vectors are FP64.
template <class T>
void LaunchSpmv(const DevicePatternView& pattern, const T* values, const double* x, double* y, cudaStream_t stream);
// y = D^{-1} (A (scale * x)) with D^{-1} stored per node as 4x4 (scale read from device, may be null);
// inverse == null gives y = scale * A x.  Returns early when *stop is set (stop may be null).
template <class T>
void LaunchSpmvBlockJacobi(const DevicePatternView& pattern, const T* values, const double* inverse,
	const double* x, const double* scale, double* y, const int* stop, cudaStream_t stream);
// y = A x on the block rows whose segment is still open (node_seg[row] its segment, seg_stop[s] set once
// segment s has stopped; the rows of stopped segments are skipped and keep their old y).  Returns
// early when *stop is set.
template <class T>
void LaunchSpmvMasked(const DevicePatternView& pattern, const T* values, const double* x, double* y,
	const int* stop, const int32_t* node_seg, const int* seg_stop, cudaStream_t stream);
template <class T>
void LaunchBlockInverse(const DevicePatternView& pattern, const T* values, double* inverse,
	unsigned int* singular, cudaStream_t stream);
void LaunchToFloat(long long n, const double* in, float* out, cudaStream_t stream);
// FP32 copy of basis tables [table][64 points][64 functions] (FP64) with the points of each pair
// interleaved: out[table][point pair][function][2] (the tensor-core tangent's staging layout).
void LaunchToFloatPointPairs(long long tables, const double* in, float* out, cudaStream_t stream);
void LaunchApplyBlockInverse(int nodes, const double* inverse, const double* x, double* y, cudaStream_t stream);
// state = prescribed value on the constrained entries (the Dirichlet values lifted into the state).
// ---- transport.cu (2x2 block CSR: values[block*4 + 2i + j], vectors value[2*node + field]) ----
void LaunchSpmv2(const DevicePatternView& pattern, const double* values, const double* x, double* y,
	cudaStream_t stream);
// y = D^{-1} (A x) * (*scale) with D^{-1} the 2x2 block-Jacobi inverse (scale may be null; stop: the
// GMRES early-out flag, may be null).  Values FP64 or FP32.
template <class T>
void LaunchSpmvBlockJacobi2(const DevicePatternView& pattern, const T* values, const double* inverse,
	const double* x, const double* scale, double* y, const int* stop, cudaStream_t stream);
void LaunchBlockInverse2(const DevicePatternView& pattern, const double* values, double* inverse,
	unsigned int* singular, cudaStream_t stream);
void LaunchApplyBlockInverse2(int nodes, const double* inverse, const double* x, double* y, cudaStream_t stream);
// Device view of the flow-line factors (flow_lines.hpp): y = M^{-1} x by a forward and a backward
// substitution along every line, one thread per line (x and y must not overlap; stop: the GMRES
// early-out flag, may be null).
struct LinePreconditionerView {
	int lines = 0;
	const int32_t* line_offsets = nullptr;
	const int32_t* line_nodes = nullptr;
	const int32_t* band_width = nullptr;
	const int64_t* band_offsets = nullptr;
	const double* factors = nullptr;
};
void LaunchLineApply(const LinePreconditionerView& view, const double* x, double* y, const int* stop,
	cudaStream_t stream);

void LaunchLiftDirichlet(int count, const int32_t* nodes, const int32_t* vmask, const int32_t* pmask,
	const double* velocity, const double* pressure, double* state, cudaStream_t stream);
template <class T>
void LaunchDirichletRows(const DevicePatternView& pattern, int count, const int32_t* constrained_nodes,
	const int32_t* velocity_mask, const int32_t* pressure_mask, const double* velocity, const double* pressure,
	const double* state, T* values, double* rhs, cudaStream_t stream);
void LaunchFaceFlows(int faces, const int32_t* face_element, const double* face_coef, int stride,
	const int32_t* element_offsets, const int32_t* connectivity, const double* state, double* face_flow,
	cudaStream_t stream);
void LaunchFaceTraction(int faces, const int32_t* face_element, const double* face_coef, int stride,
	const int32_t* element_offsets, const int32_t* connectivity, const double* face_pressure,
	double* traction, cudaStream_t stream);
// Deterministic sums: out[0] = sum x[i*stride+offset]^2, out[1] = sum x[i*stride+offset] over count items.
void LaunchStridedSums(long long count, int stride, int offset, const double* x, double* partial, double* out,
	cudaStream_t stream);
// out = sqrt(sum x^2) (deterministic two-stage).
void LaunchNorm(long long n, const double* x, double* partial, double* out, cudaStream_t stream);
void LaunchAxpy(long long n, double alpha, const double* x, double* y, cudaStream_t stream);
void LaunchSegmentSums(int segments, const int32_t* segment_of, int items, const double* values, double* out,
	cudaStream_t stream);

// Independent segments of a vector (the tubes of a batched mesh, in entries): out[k] = sum of x^2 over
// [offsets[k], offsets[k+1]).
void LaunchSegmentSquares(int segments, const int64_t* offsets, const double* x, double* out, cudaStream_t stream);
// x *= scale[k] over each segment k (0 clears it).
void LaunchScaleSegments(int segments, const int64_t* offsets, const double* scale, double* x, cudaStream_t stream);

int PartialSlots();

// ---- outlets.cu ---------------------------------------------------------
// One 0D outlet coupled on the device (kind: TFIGA_OUTLET_*; slot: the label slot of its faces, -1 if
// none).  capacitor_pressure is the value at the start of the step; pressure the one in use; flow,
// evaluated and evaluated_capacitor the last evaluation.
struct DeviceOutlet {
	int32_t kind;
	int32_t slot;
	double resistance, proximal, distal, capacitance, reference_pressure, capacitor_pressure;
	double pressure, flow, evaluated, evaluated_capacitor;
};
// Evaluates every outlet at label_flow; when `update` and the largest change exceeds
// 1e-8 + 1e-6 max(1, max |P_eval|), relaxes all pressures (and adds one to *updates); *accepted = 1
// when the pressures in use match their evaluation within that tolerance, else 0.
void LaunchOutletUpdate(int count, DeviceOutlet* outlets, const double* label_flow, double dt, double relaxation,
	bool update, double* accepted, int* updates, cudaStream_t stream);
// face_pressure[f] = outlets[slot_outlet[face_slot[f]]].pressure, or base[f] when that is -1.
void LaunchFacePressures(int faces, const int32_t* face_slot, const int32_t* slot_outlet, const double* base,
	const DeviceOutlet* outlets, double* face_pressure, cudaStream_t stream);

} // namespace tfiga
