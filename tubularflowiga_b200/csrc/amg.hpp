// Point-block (4x4) aggregation multigrid, used as the right preconditioner of
// the flexible GMRES.
//
// Ingredients follow the reference's scalar AggregationAmg
// (solvers/cuda/include/AggregationAmg.hpp:32-436): aggregates built once on
// the host from a strength graph, piecewise-constant prolongation, a Galerkin
// refresh on the device that sums fine entries into coarse entries, and a dense
// inverse at the coarsest level.  Here it works on the 4x4 node blocks of the
// Navier-Stokes system (velocity and pressure aggregated together; strength
// from the trace of the velocity block; Vanek-style greedy aggregation applied
// repeatedly to the aggregated strength graph until a few hundred aggregates
// remain).  Damped Jacobi is not a convergent smoother for these IGA operators
// (cubic B-spline mass matrices have diag/row-sum near 0.1 in 3D), so the
// preconditioner is two-level: the coarse correction x = P Ac^{-1} P^T v
// followed by one block-Jacobi step on the remaining residual, whose residual
// b - A P x_c is evaluated through the product A P (a few 4x4 blocks per fine
// row, formed with the Galerkin refresh) instead of a pass over A.  The coarse
// space carries the long-range (axial) pressure/velocity modes that make
// block-Jacobi GMRES iterations grow with tube length.  Dirichlet degrees of
// freedom are masked out of the prolongation and the coarse operator.  Every
// reduction runs in a fixed order, so an application is deterministic.
#pragma once

#include "common.hpp"
#include "kernels.cuh"

#include <memory>
#include <vector>

namespace tfiga {

struct AmgOptions {
	double strength = 0.08;        // |s_ij| >= theta sqrt(|s_ii s_jj|) is a strong connection
	int coarsest_nodes = 300;      // aggregate until at most this many coarse nodes (dense solve)
	int max_levels = 8;            // aggregation rounds
	double omega = 1.0;            // weight of the block-Jacobi step after the coarse correction
};

class Amg {
public:
	Amg(const DevicePatternView& fine, const std::vector<int32_t>& row_offsets, const std::vector<int32_t>& columns,
		cudaStream_t stream, AmgOptions options = {});
	~Amg();
	Amg(const Amg&) = delete;
	Amg& operator=(const Amg&) = delete;

	// Builds the hierarchy from the strength of `values` (device, fine level, FP64 or FP32).
	template <class T> void Build(const T* values);
	bool built() const { return built_; }
	// Dirichlet masks of the fine level (velocity / pressure constrained per node).
	void SetMasks(const std::vector<int32_t>& velocity_mask, const std::vector<int32_t>& pressure_mask);
	// Refresh from the fine values: A P and the fine block-Jacobi inverses always; the Galerkin
	// coarse operator and its dense inverse when `coarse` (always on the first refresh).
	template <class T> void Refresh(const T* values, bool coarse = true);
	// z = M^{-1} v; kernels skip when *stop is set.  With seg_stop (after SetSegments): the fine
	// nodes and aggregates of segments whose flag is set are skipped (their z is left as it was).
	template <class T> void Apply(const T* fine_values, const double* v, double* z, const int* stop,
		const int* seg_stop = nullptr);
	// Segment of every fine node (independent blocks of the matrix; aggregates never cross them), for
	// the masked Apply; empty: none.
	void SetSegments(const std::vector<int32_t>& node_segment);
	int levels() const { return (int)levels_.size(); }
	std::vector<int> level_nodes() const;
	const std::vector<int>& aggregation_rounds() const { return coarse_history_; }
	std::vector<long long> level_blocks() const;
	long long transfer_blocks() const;
	// Block-Jacobi inverses (4x4 per node, FP64) of the fine level, current after Refresh.
	const double* fine_inverse() const;
	long long launches() const { return launches_; }
	// launches replayed from a captured CUDA graph (counted as if launched)
	void count_launches(long long n) { launches_ += n; }
	void set_profiler(Profiler* p) { profiler_ = p; }

private:
	struct Level;
	template <class T> void Cycle(int level, const T* fine, const double* b, double* x, const int* stop,
		const int* seg_stop);
	void BuildSegmentMaps();           // after the hierarchy exists (Build, or SetSegments once built)
	std::vector<int32_t> node_segment_;                 // host copy until the hierarchy exists
	DeviceArray<int32_t> node_segment_dev_, aggregate_segment_dev_;
	bool segment_maps_ = false;
	template <class T> T* ApValues(Level& level);   // A P blocks in the fine matrix's precision
	void BuildFromStrength(std::vector<double> s);
	std::vector<std::unique_ptr<Level>> levels_;
	DevicePatternView fine_;
	std::vector<int32_t> fine_rows_, fine_columns_;
	std::vector<int32_t> vmask_, pmask_;
	std::vector<int> coarse_history_;
	cudaStream_t stream_;
	AmgOptions options_;
	bool built_ = false;
	bool masks_dirty_ = true;
	bool coarse_ready_ = false;
	long long launches_ = 0;
	Profiler* profiler_ = nullptr;

};

} // namespace tfiga
