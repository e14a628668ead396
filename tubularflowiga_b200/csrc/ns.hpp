// Device-resident Navier-Stokes solver: one Newton iteration and one physical
// step of the reference loop (solvers/cuda/src/iga_cuda.cu:952-1054).
#pragma once

#include "amg.hpp"
#include "gmres.hpp"
#include "case_input.hpp"
#include "mesh.hpp"

#include "../../include/tfiga.h"

#include <map>
#include <memory>
#include <vector>

namespace tfiga {

class NsSolver {
public:
	NsSolver(Mesh& mesh, const tfiga_ns_params& params);
	~NsSolver();
	NsSolver(const NsSolver&) = delete;
	NsSolver& operator=(const NsSolver&) = delete;

	void SetDirichlet(const int32_t* vmask, const int32_t* pmask, const double* velocity, const double* pressure);
	void SetDirichletValues(const double* velocity, const double* pressure);
	void SetTractions(const int32_t* labels, const double* pressures, int count);
	void SetState(const double* state, const double* previous);
	void GetState(double* state);
	void CommitStep();

	// values/rhs on the device: rhs = -r + traction.
	void Assemble();
	void ApplyDirichlet();
	void ApplyDirichletRhs();       // rhs rows only (g - u on constrained entries)
	// Inexact-Newton mode: the prescribed values into the state before a step's first Newton
	// iteration, so that its residual (and the forcing tolerances) measure the PDE rows only.
	void LiftDirichletForForcing();
	void ApplyDirichletMatrix();    // Jacobian rows only (zero rows, unit diagonal)
	GmresResult SolveLinear(double rtol, int max_iterations);
	tfiga_newton_report NewtonIteration(double initial_residual);
	tfiga_step_report Step();
	// Step coupled to outlet models (relaxed fixed point of iga_cuda.cu:927-1086); *iterations = Newton loops.
	tfiga_step_report StepOutlets(tfiga_outlet* outlets, int count, double relaxation, int max_iterations,
		int* iterations);
	// Step with the outlet pressures updated after every Newton update (one Newton loop); *updates =
	// pressure updates.  Same acceptance tests as StepOutlets.
	tfiga_step_report StepOutletsCoupled(tfiga_outlet* outlets, int count, double relaxation, int max_newton,
		int* updates);
	void BoundaryFlows(const int32_t* labels, int count, double* flows);
	// Independent segments of the node range (the tubes of a batched mesh): node_offsets[count + 1],
	// increasing from 0 to nodes; count 0 removes them.  With segments the Newton test is taken per
	// segment -- ||r_k|| <= max(atol sqrt(4 n_k), rtol ||r_k,0||) with r_k,0 the segment's residual at
	// the step's first iteration -- and a segment that passes is frozen: its rhs rows are zeroed before
	// each later linear solve, so its update is zero (the system is block diagonal over the segments),
	// and each open segment's rhs is scaled to unit norm for the solve (its update scaled back after).
	// The step converges when every segment passes (and the mass test holds).
	void SetSegments(const int64_t* node_offsets, int count);
	// After a Newton iteration: per segment 1 if it has passed its test in this step, and its residual.
	void SegmentStatus(int32_t* done, double* residuals) const;
	void Synchronize();

	int64_t nodes() const { return mesh_.nodes(); }
	long long blocks() const { return (long long)mesh_.pattern().columns.size(); }
	double* values() { return values_.get(); }       // null in TFIGA_PRECISION_MIXED
	float* values32() { return values32_.get(); }    // null in TFIGA_PRECISION_FP64
	// FP32 Jacobian storage (both reduced-precision modes).
	bool mixed() const { return params_.precision != TFIGA_PRECISION_FP64; }
	// Tangent contracted on the tensor cores (FP32 accumulation); no FP64 Jacobian is kept.
	bool tensor_tangent() const
	{
		return params_.precision == TFIGA_PRECISION_MIXED || params_.precision == TFIGA_PRECISION_MIXED_BF16X3
			|| params_.precision == TFIGA_PRECISION_MIXED_TF32;
	}
	// The tensor-core operand organisation of the precision mode (TC_OPERANDS_*).
	int tc_operands() const
	{
		return params_.precision == TFIGA_PRECISION_MIXED_BF16X3 ? TC_OPERANDS_SPLIT
			: params_.precision == TFIGA_PRECISION_MIXED_TF32 ? TC_OPERANDS_TF32 : TC_OPERANDS_BF16;
	}
	// Active Jacobian values as FP64 on the host (FP32 storage is widened).
	void DownloadValues(double* out);
	double* state() { return state_.get(); }
	double* rhs() { return rhs_.get(); }
	double* update() { return update_.get(); }
	const DevicePatternView pattern() const { return mesh_.pattern_view(); }
	cudaStream_t stream() const { return stream_; }
	long long launches() const { return launches_; }
	void AddLaunches(long long n) { launches_ += n; }
	const tfiga_ns_params& params() const { return params_; }
	Profiler& profiler() { return profiler_; }
	const Amg* amg() const { return amg_.get(); }
	// Learned preconditioner stage (not owned): used in the AMG-FGMRES solves when `use`, and a
	// training pair stored after every Newton solve when `collect`.
	void SetLearned(LearnedPreconditioner* learned, bool use, bool collect);
	long long learned_fallbacks() const { return learned_fallbacks_; }
	long long tangent_contractions() const { return tangent_contractions_; }
	// Tensor-core modes: the tangent organisation in use (TFIGA_TANGENT_*; TFIGA_TANGENT_AUTO until the
	// first tangent has been assembled) and the autotuner's timings of both (ms, 0 if not run).
	int tangent_kernel() const { return tangent_kernel_; }
	double tune_ms(int kernel) const
	{
		return kernel == TFIGA_TANGENT_FUSED ? tune_ms_[1] : kernel == TFIGA_TANGENT_ELEMENT ? tune_ms_[2] : tune_ms_[0];
	}
	// Binds the current (Dirichlet-row) Jacobian as the operator of the learned stage's residual loss.
	void BindLearnedOperator(LearnedPreconditioner& learned);

private:
	struct Diagnostics {
		double continuity_l2, continuity_sum, net_flow, absolute_flow, imbalance;
	};
	void ApplyTractions(const std::map<int32_t, double>& traction);
	// Tensor-core modes: the FP64 residual and point coefficients (rhs = -r + traction), then the
	// tangent from those coefficients into the FP32 Jacobian (builds the AMG on first use).
	void AssembleResidualTc();
	void ApplyDirichletParts(bool matrix, bool rhs);
	void AssembleTangentTc();
	// TFIGA_TANGENT_AUTO: times both tangent organisations on the current state (the separate one only
	// when its arrays fit in free memory), keeps the faster and releases the other's arrays; values32_
	// then holds the tangent.
	void AutotuneTangent();
	// Every mode, for the residual-first Newton iteration: the FP64 residual alone (rhs = -r +
	// traction; in the tensor-core modes with the point coefficients), then -- only for an
	// iteration that solves with a new tangent -- the Jacobian alone (FP64 assembly, or the
	// tensor-core contraction; builds the AMG on first use).
	void AssembleResidual();
	void AssembleTangent();
	// The elements with 65..80 basis functions (FP64 large-element kernel): tangent added into values
	// and residual into rhs, either may be null.  No launch when the mesh has none.
	template <class T> void LargeElements(T* values, double* rhs);
	std::vector<OutletModel> OutletModels(const tfiga_outlet* outlets, int count) const;
	void LaunchDiagnostics(bool flows);   // continuity sums of rhs (+ per-label flows of state when `flows`)
	// Device outlet coupling of StepOutletsCoupled, before an iteration's residual: per-label flows of
	// the state, the outlet update, the per-face pressures and the traction rhs.
	void CoupleOutletsOnDevice();
	Diagnostics ReadDiagnostics();

	Mesh& mesh_;
	tfiga_ns_params params_;
	cudaStream_t stream_ = nullptr;
	cudaEvent_t events_[6] = {};
	long long launches_ = 0;
	long long solves_ = 0;                   // linear solves so far (coarse refresh period)
	double forcing_norm_ = 0.0, forcing_eta_ = 0.0;   // previous residual and forcing term (inexact Newton)
	bool tangent_valid_ = false;             // the Jacobian holds the tangent of this step's last iteration
	double reuse_norm_ = 0.0, reuse_eta_ = 0.0;   // previous Newton residual and linear tolerance (tangent reuse)
	long long tangent_contractions_ = 0;     // tangent assemblies (FP64 or tensor-core) by NewtonIteration
	bool amg_current_ = false;               // the AMG data were refreshed from the current Jacobian
	long long refreshes_ = 0;                // AMG refreshes so far (coarse refresh period)
	std::map<int32_t, double> tractions_;    // label -> pressure set by SetTractions
	int64_t n4_;
	DeviceArray<double> values_, rhs_, state_, previous_, update_, traction_, velocity_bc_, pressure_bc_;
	DeviceArray<float> values32_;
	DeviceArray<float> coef32_;              // tensor-core tangent: point coefficients [e][4][80][64]
	DeviceArray<double> point_state_;        // fused tensor-core tangent: FP64 point state [e][64][22]
	int tangent_kernel_ = 0;                 // TFIGA_TANGENT_* in use
	double tune_ms_[3] = {0.0, 0.0, 0.0};    // autotuner: coefficient-array (pair), fused, element times
	bool coefficient_arrays() const
	{
		return tangent_kernel_ == TFIGA_TANGENT_COEFFICIENTS || tangent_kernel_ == TFIGA_TANGENT_ELEMENT;
	}
	DeviceArray<double> face_flow_, face_pressure_, label_flow_, partial_, scalars_;
	DeviceArray<int32_t> vmask_, pmask_, constrained_, face_slot_, status_;
	std::vector<int32_t> labels_;            // distinct face labels (slot order)
	std::map<int32_t, int> slot_of_label_;
	std::vector<int32_t> face_slot_host_;
	int constrained_count_ = 0;
	bool dirichlet_set_ = false;
	Gmres gmres_;
	Profiler profiler_;
	std::unique_ptr<Amg> amg_;
	double* pinned_ = nullptr;               // host mirror of scalars + label flows
	LearnedPreconditioner* learned_ = nullptr;
	bool collect_pairs_ = false;
	long long learned_fallbacks_ = 0;        // solves redone without the learned stage
	DeviceArray<double> pair_dinv_, pair_amg_, pair_aamg_;
	DeviceArray<int> zero_flag_;
	int32_t* pinned_status_ = nullptr;       // host mirror of the tensor-core kernel status
	// outlets coupled on the device (StepOutletsCoupled): active while outlet_count_ >= 0
	DeviceArray<DeviceOutlet> outlets_dev_;
	DeviceArray<int32_t> slot_outlet_, outlet_updates_;
	DeviceArray<double> face_base_;
	int outlet_count_ = -1;
	// outward-flow vectors of the coupled outlets (sparse, on the free velocity unknowns) and their
	// Jacobian coefficients dP/dQ, for the flexible GMRES's low-rank term
	DeviceArray<int32_t> lr_ptr_, lr_idx_;
	DeviceArray<double> lr_val_, lr_coef_;
	std::vector<int32_t> lr_labels_;
	bool lr_dirty_ = true;
	void BuildOutletFlowVectors(const std::vector<int32_t>& labels);
	int outlet_iteration_ = 0;
	double outlet_relaxation_ = 1.0;
	bool last_outlet_ok_ = false;
	// segments (SetSegments)
	int segments_ = 0;
	std::vector<int64_t> segment_nodes_;
	std::vector<double> segment_initial_, segment_norm_, segment_forcing_;
	std::vector<int32_t> segment_done_host_;
	DeviceArray<int64_t> segment_entries_;
	DeviceArray<double> segment_sq_;
	DeviceArray<double> segment_scale_;      // [rhs scale of each segment][update scale of each segment]
	std::vector<double> segment_scale_host_;
	double* pinned_segments_ = nullptr;
};

} // namespace tfiga
