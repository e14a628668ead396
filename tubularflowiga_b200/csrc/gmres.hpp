// Restarted left-preconditioned GMRES(m) with block-Jacobi preconditioning,
// the solver of the reference's Newton loop (SolveGmres,
// solvers/cuda/include/Gmres.hpp:192-336): same preconditioner, restart,
// tolerance definition (rtol * ||D^{-1} r0||) and true-residual restart check.
//
// B200 organisation: the Hessenberg matrix, Givens rotations and residual
// estimate live on the device; orthogonalisation is classical Gram-Schmidt
// applied twice (two multi-dot + multi-axpy passes over the basis instead of
// one dot/axpy pair per basis vector); Krylov vectors are normalised lazily
// through a per-vector scale; kernels of an iteration batch return early once
// the device has flagged convergence, so the host waits only once per batch.
#pragma once

#include "amg.hpp"
#include "common.hpp"
#include "kernels.cuh"
#include "learned.hpp"

namespace tfiga {

struct GmresResult {
	int iterations = 0;
	double residual = 0.0;
	unsigned singular_blocks = 0;
	bool converged = false;
};

class Gmres {
public:
	// fields: unknowns per node, the block size of the matrix (4: Navier-Stokes, 2: transport).
	Gmres(int nodes, int restart, cudaStream_t stream, int fields = 4);
	~Gmres();
	Gmres(const Gmres&) = delete;
	Gmres& operator=(const Gmres&) = delete;
	// Solves A x = rhs (x holds the initial guess).  Builds the block inverse first unless
	// rebuild_preconditioner is false (the matrix is the one of the previous Solve).  With
	// krylov_values (an FP32 copy of A) the Arnoldi SpMV reads it; the block inverse and each
	// restart's true residual use the FP64 values.
	GmresResult Solve(const DevicePatternView& pattern, const double* values, const double* rhs, double* x,
		double rtol, int max_iterations, long long* launches, bool rebuild_preconditioner = true,
		const float* krylov_values = nullptr);
	// Right-preconditioned flexible GMRES (FGMRES): z_j = M^{-1} v_j stored, tolerance
	// rtol * ||b - A x0|| on the true residual.
	// The matrix may be stored in FP64 or FP32 (T); with FP32 the Krylov basis is stored in FP32
	// too unless fp64_basis (dots, updates and the work vector in FP64 arithmetic); preconditioned
	// vectors, Hessenberg, Givens and the solution stay FP64, and each restart's true residual is the
	// FP64 refinement.  Needs fields == 4.
	template <class T>
	GmresResult SolveFlexible(const DevicePatternView& pattern, const T* values, const double* rhs, double* x,
		double rtol, int max_iterations, Amg& preconditioner, long long* launches, bool fp64_basis = false);
	int restart() const { return restart_; }
	int fields() const { return fields_; }
	// 2x2 blocks: precondition Solve with the flow-line factors instead of block-Jacobi (null: off).
	void set_line_preconditioner(const LinePreconditionerView* view)
	{
		line_on_ = view != nullptr;
		if (view) line_ = *view;
	}
	// Learned stage added to the AMG application in SolveFlexible (null: AMG only).
	void set_learned(LearnedPreconditioner* learned) { learned_ = learned; }
	LearnedPreconditioner* learned() const { return learned_; }
	// Stores a training pair (w_j = A z_j) into `collector` on every eighth iteration (null: off).
	void set_collector(LearnedPreconditioner* collector) { collector_ = collector; }
	void set_profiler(Profiler* profiler) { profiler_ = profiler; }
	// Low-rank term of the flexible solve's operator, A + sum_k c_k g_k g_k^T with each g_k a sparse
	// vector (entries ptr[k] .. ptr[k+1] of idx / val, distinct indices per k): the outlet coupling's
	// share of the Newton Jacobian.  Null: off.
	struct LowRank { int count; const int* ptr; const int* idx; const double* val; const double* coef; };
	void set_low_rank(const LowRank* term)
	{
		low_on_ = term != nullptr && term->count > 0;
		if (low_on_) low_ = *term;
	}
	// Independent segments of the unknowns (entry offsets, count + 1 values increasing from 0 to the
	// system size; fewer than 2 values: none) for SolveFlexibleSegments; blocks[k] the matrix blocks of
	// segment k's rows (for the profiler's byte counts of the masked SpMV).
	void SetSegments(const std::vector<int64_t>& entry_offsets, const std::vector<int64_t>& blocks = {});
	int segments() const { return segments_; }
	// SolveFlexible with one Arnoldi process per segment sharing the SpMV and preconditioner launches:
	// each segment its own Hessenberg matrix, rotations and tolerance rtol * ||b_k - A x0_k|| (the matrix
	// and the preconditioner must not couple segments).  Converged when every segment meets its own;
	// iterations count the union's steps.  No learned stage.
	template <class T>
	GmresResult SolveFlexibleSegments(const DevicePatternView& pattern, const T* values, const double* rhs, double* x,
		double rtol, int max_iterations, Amg& preconditioner, long long* launches, bool fp64_basis = false);
	std::size_t bytes() const;

private:
	template <class T>
	void Step(const DevicePatternView& pattern, const T* values, int j);
	// Both classical Gram-Schmidt passes of Arnoldi step j, then its Givens finalisation against
	// tolerance_ (one profiling interval of family kOrtho).
	template <class B> void Orthogonalize(int j, B* basis);
	// Krylov basis storage: FP64 (V_) or FP32 (V32_, allocated on first use).
	template <class B> B* Basis();
	template <class T, class B>
	GmresResult SolveFlexibleImpl(const DevicePatternView& pattern, const T* values, const double* rhs, double* x,
		double rtol, int max_iterations, Amg& preconditioner, long long* launches);
	template <class T, class B>
	void FlexibleStep(const DevicePatternView& pattern, const T* values, int j, Amg& preconditioner);
	template <class T, class B>
	double TrueResidualPlain(const DevicePatternView& pattern, const T* values, const double* rhs, const double* x);
	double TrueResidual(const DevicePatternView& pattern, const double* values, const double* rhs, const double* x);
	template <class T, class B>
	GmresResult SolveFlexibleSegmentsImpl(const DevicePatternView& pattern, const T* values, const double* rhs,
		double* x, double rtol, int max_iterations, Amg& preconditioner, long long* launches);
	template <class T, class B>
	void SegFlexibleStep(const DevicePatternView& pattern, const T* values, int j, Amg& preconditioner);
	// SegFlexibleStep through a CUDA graph captured on the step's first use (one graph per Arnoldi
	// index j, replayed while the operator, preconditioner and vectors stay where they are); direct
	// launches while profiling, with the outlet term or the learned stage, or if capture fails.
	template <class T, class B>
	void SegStep(const DevicePatternView& pattern, const T* values, int j, Amg& preconditioner);
	void ReleaseSegmentGraphs();
	// r = b - A x, segment norms into seg_host_beta_ / seg_beta_, r stored as basis vector 0
	template <class T, class B>
	void SegTrueResidual(const DevicePatternView& pattern, const T* values, const double* rhs, const double* x);
	int segments_ = 0, seg_dot_cx_ = 0, seg_vec_cx_ = 0;
	DeviceArray<int64_t> seg_off_;
	DeviceArray<int32_t> seg_node_;      // segment of every node (block row)
	DeviceArray<double> seg_H_, seg_cs_, seg_sn_, seg_g_, seg_y_, seg_scale_, seg_hpass_, seg_partial_,
		seg_norm_partial_, seg_tol_, seg_beta_, seg_sq_, seg_residual_;
	DeviceArray<int> seg_stop_, seg_used_, seg_all_;
	std::vector<double> seg_host_beta_, seg_host_tol_;
	std::vector<int> seg_host_flags_, seg_host_stop_;
	std::vector<int64_t> seg_blocks_;    // matrix blocks per segment (byte accounting)
	std::vector<int64_t> seg_len_;       // entries per segment
	std::vector<cudaGraphExec_t> seg_graphs_;            // per Arnoldi index j
	std::vector<long long> seg_graph_launches_, seg_graph_amg_launches_;
	const void* seg_graph_values_ = nullptr;             // operator the graphs were captured with
	const void* seg_graph_amg_ = nullptr;
	bool seg_graphs_ok_ = true;

	int nodes_, fields_, n_, restart_, blocks_;
	unsigned singular_count_ = 0;     // singular diagonal blocks of the last block-inverse build
	bool line_on_ = false;            // flow-line preconditioner (2x2 blocks)
	LinePreconditionerView line_;
	int update_blocks_ = 0;           // CTAs of the basis update (one per 32 entry pairs)
	int chunk_;
	// Fused first-pass update and second-pass dots of the Gram-Schmidt sweep: entries per CTA for an
	// FP32 / FP64 basis (0: that basis takes the unfused passes), CTAs, shared-memory bytes.
	int fused_chunk_[2] = {0, 0}, fused_blocks_[2] = {0, 0};
	size_t fused_smem_[2] = {0, 0};
	DeviceArray<double> fused_partial_;
	size_t finalize_smem_ = 0;
	cudaStream_t stream_;
	long long launches_ = 0;
	DeviceArray<double> Z_;
	DeviceArray<float> V32_;
	DeviceArray<double> V_, w_, r_, tmp_, inverse_, partial_, hpass_, H_, cs_, sn_, g_, y_, scale_, norm_partial_,
		scalar_;
	DeviceArray<int> state_;          // [0] stop, [1] used, [2] error
	DeviceArray<double> residual_;    // [0] residual estimate
	DeviceArray<unsigned> singular_;
	struct HostStatus { int stop, used, error, pad; double residual; double beta[2]; unsigned singular; };
	HostStatus* host_ = nullptr;
	Profiler* profiler_ = nullptr;
	double tolerance_ = 0.0;                 // absolute residual target of the current solve
	bool low_on_ = false;
	LowRank low_{};
	// y += sum_k c_k (g_k . x) g_k (skipped when *stop; stop may be null).
	void AddLowRank(const double* x, double* y, const int* stop);
	LearnedPreconditioner* learned_ = nullptr;
	LearnedPreconditioner* collector_ = nullptr;
	DeviceArray<double> pair_dinv_, pair_amg_, pair_aamg_;
};

template <> double* Gmres::Basis<double>();
template <> float* Gmres::Basis<float>();

} // namespace tfiga
