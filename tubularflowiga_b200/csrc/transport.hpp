// Two-species transport solver: the reference's `iga_cuda transport`
// (solvers/cuda/src/iga_cuda.cu:621-732) on the Navier-Stokes path's mesh,
// basis tables, block pattern and GMRES.
//
// Unknowns per node: N0 (attached species, diffusion and exchange) and N+
// (advected by a prescribed nodal velocity, SUPG-stabilised), stored as
// vector[2 node + field] with 2x2 blocks values[block*4 + 2 i + j] on the
// mesh's node-graph pattern.  Backward Euler with a constant left matrix:
// each step is rhs = P c, the boundary values set in rhs, then
// L c' = rhs by block-Jacobi GMRES(restart) to rtol (warm-started from c
// after the first step; the block inverse is built once).
#pragma once

#include "common.hpp"
#include "gmres.hpp"
#include "kernels.cuh"
#include "mesh.hpp"

#include <cstdint>
#include <vector>

namespace tfiga {

// The element coefficients of iga::TransportParameters (solvers/cpu/include/CaseInput.hpp:19-33).
struct TransportCoefficients {
	double diffusion;
	double vplus;
	double kplus;
	double kminus;
	double detach_plus;
	double dt;
	double artificial_diffusion;
};

// Left and previous matrices of every element added into the 2x2 block values (once per run).
void LaunchTransportAssembly(const DeviceMeshView& mesh, const double* phi, const double* qdata,
	const int32_t* element_blocks, const double* velocity, const TransportCoefficients& coefficients, double* left,
	double* previous, cudaStream_t stream);
// The same for the elements [first, first + count) with up to 80 basis functions (80-wide tables).
void LaunchTransportAssemblyLarge(const DeviceMeshView& mesh, int first, int count, const double* phi,
	const double* qdata, const int32_t* element_blocks, const double* velocity,
	const TransportCoefficients& coefficients, double* left, double* previous, cudaStream_t stream);
void LaunchTransportBoundaryRows(const DevicePatternView& pattern, int count, const int32_t* nodes, double* left,
	double* previous, cudaStream_t stream);
void LaunchTransportBoundaryValues(int count, const int32_t* nodes, const double* n0, const double* nplus,
	double* vector, cudaStream_t stream);

struct TransportStepResult {
	int iterations = 0;          // GMRES iterations of the step
	double residual = 0.0;       // final preconditioned residual norm
	unsigned singular_blocks = 0;
};

class TransportSolver {
public:
	// velocity [3 nodes], constrained [nodes] (nonzero: Dirichlet node), n0 / nplus [nodes]:
	// host or device pointers.  Assembles both matrices, applies the boundary rows and sets the
	// boundary values into the zero initial state.  fp32_krylov: an FP32 copy of L serves the SpMV
	// of the Arnoldi process (the true residual of every restart stays FP64).  flow_lines: the
	// GMRES is preconditioned with the flow-line factors of L (flow_lines.hpp) instead of
	// block-Jacobi.
	TransportSolver(Mesh& mesh, const TransportCoefficients& coefficients, const double* velocity,
		const int32_t* constrained, const double* n0, const double* nplus, int restart, bool fp32_krylov = false,
		bool flow_lines = false);
	TransportSolver(const TransportSolver&) = delete;
	TransportSolver& operator=(const TransportSolver&) = delete;

	// One backward-Euler step (iga_cuda.cu:683-707).  Fails with TFIGA_E_NOT_CONVERGED when GMRES
	// stops above its tolerance.
	TransportStepResult Step(double rtol, int max_iterations);
	void SetState(const double* state);   // [2 nodes], host or device
	void GetState(double* state);         // [2 nodes], host or device
	void Matrices(double* left, double* previous);   // [4 blocks] each, host or device
	// y = M^{-1} x with the flow-line factors (flow_lines mode only), x and y [2 nodes], host or device.
	void ApplyLinePreconditioner(const double* x, double* y);
	double StateNorm();
	int steps() const { return steps_; }
	long long launches() const { return launches_; }
	cudaStream_t stream() const { return mesh_.stream(); }
	const double* device_state() const { return current_.get(); }
	double* device_left() { return left_.get(); }
	double* device_previous() { return previous_.get(); }
	double assembly_ms() const { return assembly_ms_; }
	Profiler& profiler() { return profiler_; }

private:
	Mesh& mesh_;
	int nodes_;
	int steps_ = 0;
	long long launches_ = 0;
	double assembly_ms_ = 0.0;
	DeviceArray<double> left_, previous_, current_, next_, rhs_, n0_, nplus_, scratch_;
	DeviceArray<float> left32_;        // FP32 copy of L (fp32_krylov)
	DeviceArray<int32_t> line_offsets_, line_nodes_, band_width_;   // flow-line factors (flow_lines)
	DeviceArray<int64_t> band_offsets_;
	DeviceArray<double> line_factors_;
	LinePreconditionerView line_view_;
	bool flow_lines_ = false;
	DeviceArray<int32_t> constrained_;
	int constrained_count_ = 0;
	Gmres gmres_;
	Profiler profiler_;
};

} // namespace tfiga
