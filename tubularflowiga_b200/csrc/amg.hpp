// Point-block (4x4) plain-aggregation algebraic multigrid, used as the right
// preconditioner of the flexible GMRES.
//
// Algorithm: the reference's scalar AggregationAmg
// (solvers/cuda/include/AggregationAmg.hpp:32-436): a hierarchy built once on
// the host from a strength graph, piecewise-constant prolongation, a Galerkin
// refresh on the device that sums fine entries into coarse entries, damped
// Jacobi smoothing and a dense inverse at the coarsest level.  Here it works
// on the 4x4 node blocks of the Navier-Stokes system (velocity and pressure
// aggregated together): strength from the trace of the velocity block,
// Vanek-style greedy aggregation, block-Jacobi smoothing, and Dirichlet
// degrees of freedom masked out of prolongation and of every coarse operator.
// Every reduction (Galerkin sums, restriction) runs in a fixed order, so a
// V-cycle is deterministic.
#pragma once

#include "common.hpp"
#include "kernels.cuh"

#include <memory>
#include <vector>

namespace tfiga {

struct AmgOptions {
	double strength = 0.08;        // |s_ij| >= theta sqrt(|s_ii s_jj|) is a strong connection
	int coarsest_nodes = 160;      // dense inverse at or below this many nodes
	int max_levels = 8;
	int pre_sweeps = 1, post_sweeps = 1;
	double omega = 0.7;            // block-Jacobi damping
};

class Amg {
public:
	Amg(const DevicePatternView& fine, const std::vector<int32_t>& row_offsets, const std::vector<int32_t>& columns,
		cudaStream_t stream, AmgOptions options = {});
	~Amg();
	Amg(const Amg&) = delete;
	Amg& operator=(const Amg&) = delete;

	// Builds the hierarchy from the strength of `values` (device, fine level); masks: 1 = free DOF.
	void Build(const double* values);
	bool built() const { return built_; }
	// Dirichlet masks of the fine level (velocity / pressure constrained per node).
	void SetMasks(const std::vector<int32_t>& velocity_mask, const std::vector<int32_t>& pressure_mask);
	// Galerkin refresh of every coarse operator + smoother inverses from the fine values.
	void Refresh(const double* values);
	// z = M^{-1} v (one V-cycle); kernels skip when *stop is set.
	void Apply(const double* fine_values, const double* v, double* z, const int* stop);
	int levels() const { return (int)levels_.size(); }
	std::vector<int> level_nodes() const;
	std::vector<long long> level_blocks() const;
	long long launches() const { return launches_; }
	void set_profiler(Profiler* p) { profiler_ = p; }

private:
	struct Level;
	void Cycle(int level, const double* b, double* x, const int* stop);
	std::vector<std::unique_ptr<Level>> levels_;
	DevicePatternView fine_;
	std::vector<int32_t> fine_rows_, fine_columns_;
	std::vector<int32_t> vmask_, pmask_;
	cudaStream_t stream_;
	AmgOptions options_;
	bool built_ = false;
	bool masks_dirty_ = true;
	long long launches_ = 0;
	Profiler* profiler_ = nullptr;
	const double* fine_values_ = nullptr;
};

} // namespace tfiga
