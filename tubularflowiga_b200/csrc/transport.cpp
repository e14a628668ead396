// Host side of the two-species transport solver (iga_cuda.cu:621-732).
#include "transport.hpp"

#include "flow_lines.hpp"

#include <cmath>
#include <string>

namespace tfiga {

TransportSolver::TransportSolver(Mesh& mesh, const TransportCoefficients& coefficients, const double* velocity,
	const int32_t* constrained, const double* n0, const double* nplus, int restart, bool fp32_krylov,
	bool flow_lines)
	: mesh_(mesh), nodes_((int)mesh.nodes()), gmres_((int)mesh.nodes(), restart, mesh.stream(), 2)
{
	if (!(coefficients.dt > 0.0) || !std::isfinite(coefficients.dt)) Fail(-1, "transport dt must be positive");
	if (!velocity || !constrained || !n0 || !nplus) Fail(-1, "transport inputs must not be null");
	cudaStream_t s = mesh_.stream();
	const DevicePatternView pattern = mesh_.pattern_view();
	const size_t n = (size_t)nodes_;
	left_.Allocate((size_t)pattern.blocks*4);
	previous_.Allocate((size_t)pattern.blocks*4);
	current_.Allocate(2*n); next_.Allocate(2*n); rhs_.Allocate(2*n);
	n0_.Allocate(n); nplus_.Allocate(n);
	scratch_.Allocate((size_t)PartialSlots()+2);   // LaunchNorm: the partial sums, then (norm, sum)
	left_.Zero(s); previous_.Zero(s); current_.Zero(s); next_.Zero(s); rhs_.Zero(s);
	n0_.Upload(n0, n, s);
	nplus_.Upload(nplus, n, s);

	// Constrained-node list (the reference tests a mask per node in every kernel).
	std::vector<int32_t> mask(n);
	CudaCheck(cudaMemcpyAsync(mask.data(), constrained, n*sizeof(int32_t), cudaMemcpyDefault, s),
		"transport mask");
	CudaCheck(cudaStreamSynchronize(s), "transport mask");
	std::vector<int32_t> list;
	for (size_t i = 0; i < n; ++i)
		if (mask[i]) list.push_back((int32_t)i);
	constrained_count_ = (int)list.size();
	if (constrained_count_) {
		constrained_.Allocate(list.size());
		constrained_.Upload(list.data(), list.size(), s);
	}
	DeviceArray<double> velocity_device(3*n);
	velocity_device.Upload(velocity, 3*n, s);

	cudaEvent_t start, stop;
	CudaCheck(cudaEventCreate(&start), "event");
	CudaCheck(cudaEventCreate(&stop), "event");
	CudaCheck(cudaEventRecord(start, s), "event");
	LaunchTransportAssembly(mesh_.regular_view(), mesh_.phi(), mesh_.qdata(), mesh_.element_blocks(),
		velocity_device.get(), coefficients, left_.get(), previous_.get(), s);
	LaunchTransportAssemblyLarge(mesh_.view(), mesh_.large_first(), mesh_.large_count(), mesh_.phi_large(),
		mesh_.qdata(), mesh_.element_blocks_large(), velocity_device.get(), coefficients, left_.get(), previous_.get(),
		s);
	LaunchTransportBoundaryRows(pattern, constrained_count_, constrained_.get(), left_.get(), previous_.get(), s);
	LaunchTransportBoundaryValues(constrained_count_, constrained_.get(), n0_.get(), nplus_.get(), current_.get(), s);
	if (fp32_krylov) {
		left32_.Allocate((size_t)pattern.blocks*4);
		LaunchToFloat((long long)pattern.blocks*4, left_.get(), left32_.get(), s);
		launches_ += 1;
	}
	CudaCheck(cudaEventRecord(stop, s), "event");
	CudaCheck(cudaStreamSynchronize(s), "transport assembly");
	float ms = 0.0f;
	CudaCheck(cudaEventElapsedTime(&ms, start, stop), "event");
	cudaEventDestroy(start);
	cudaEventDestroy(stop);
	assembly_ms_ = ms;
	launches_ += 3+(mesh_.large_count() > 0 ? 1 : 0);
	gmres_.set_profiler(&profiler_);
	if (flow_lines) {
		// Built once on the host from L after the boundary rows (L is constant over the steps).
		std::vector<double> values((size_t)pattern.blocks*4);
		left_.Download(values.data(), values.size(), s);
		CudaCheck(cudaStreamSynchronize(s), "flow-line matrix");
		const HostPattern& hp = mesh_.pattern();
		const FlowLineFactors f = BuildFlowLines(nodes_, hp.row_offsets.data(), hp.columns.data(), values.data());
		line_offsets_.Allocate(f.line_offsets.size());
		line_offsets_.Upload(f.line_offsets.data(), f.line_offsets.size(), s);
		line_nodes_.Allocate(f.line_nodes.size());
		line_nodes_.Upload(f.line_nodes.data(), f.line_nodes.size(), s);
		band_width_.Allocate(f.band_width.size());
		band_width_.Upload(f.band_width.data(), f.band_width.size(), s);
		band_offsets_.Allocate(f.band_offsets.size());
		band_offsets_.Upload(f.band_offsets.data(), f.band_offsets.size(), s);
		line_factors_.Allocate(f.factors.size());
		line_factors_.Upload(f.factors.data(), f.factors.size(), s);
		CudaCheck(cudaStreamSynchronize(s), "flow-line factors");
		LinePreconditionerView view;
		view.lines = f.lines();
		view.line_offsets = line_offsets_.get();
		view.line_nodes = line_nodes_.get();
		view.band_width = band_width_.get();
		view.band_offsets = band_offsets_.get();
		view.factors = line_factors_.get();
		gmres_.set_line_preconditioner(&view);
		line_view_ = view;
		flow_lines_ = true;
	}
}

TransportStepResult TransportSolver::Step(double rtol, int max_iterations)
{
	cudaStream_t s = mesh_.stream();
	const DevicePatternView pattern = mesh_.pattern_view();
	const size_t n2 = 2*(size_t)nodes_;
	profiler_.Begin(Profiler::kSpmv, s);
	LaunchSpmv2(pattern, previous_.get(), current_.get(), rhs_.get(), s);
	profiler_.End(s);
	LaunchTransportBoundaryValues(constrained_count_, constrained_.get(), n0_.get(), nplus_.get(), rhs_.get(), s);
	launches_ += 2;
	if (steps_ == 0) next_.Zero(s);
	else CudaCheck(cudaMemcpyAsync(next_.get(), current_.get(), n2*sizeof(double), cudaMemcpyDeviceToDevice, s),
		"transport warm start");
	long long launches = 0;
	const GmresResult r = gmres_.Solve(pattern, left_.get(), rhs_.get(), next_.get(), rtol, max_iterations,
		&launches, steps_ == 0, left32_.size() ? left32_.get() : nullptr);
	launches_ += launches;
	if (!r.converged)
		Fail(-6, "transport GMRES did not converge at step "+std::to_string(steps_)+"; residual "
			+std::to_string(r.residual));
	std::swap(current_, next_);
	++steps_;
	TransportStepResult result;
	result.iterations = r.iterations;
	result.residual = r.residual;
	result.singular_blocks = r.singular_blocks;
	return result;
}

void TransportSolver::SetState(const double* state)
{
	current_.Upload(state, 2*(size_t)nodes_, mesh_.stream());
	CudaCheck(cudaStreamSynchronize(mesh_.stream()), "transport state");
}

void TransportSolver::GetState(double* state)
{
	current_.Download(state, 2*(size_t)nodes_, mesh_.stream());
	CudaCheck(cudaStreamSynchronize(mesh_.stream()), "transport state");
}

void TransportSolver::Matrices(double* left, double* previous)
{
	const size_t count = (size_t)mesh_.pattern_view().blocks*4;
	if (left) left_.Download(left, count, mesh_.stream());
	if (previous) previous_.Download(previous, count, mesh_.stream());
	CudaCheck(cudaStreamSynchronize(mesh_.stream()), "transport matrices");
}

void TransportSolver::ApplyLinePreconditioner(const double* x, double* y)
{
	if (!flow_lines_) Fail(-1, "the transport handle has no flow-line preconditioner");
	cudaStream_t s = mesh_.stream();
	const size_t n2 = 2*(size_t)nodes_;
	// rhs_ and next_ are step scratch: Step rewrites both before reading them
	rhs_.Upload(x, n2, s);
	LaunchLineApply(line_view_, rhs_.get(), next_.get(), nullptr, s);
	launches_ += 1;
	next_.Download(y, n2, s);
	CudaCheck(cudaStreamSynchronize(s), "flow-line preconditioner");
}

double TransportSolver::StateNorm()
{
	LaunchNorm(2LL*nodes_, current_.get(), scratch_.get(), scratch_.get()+PartialSlots(), mesh_.stream());
	launches_ += 2;
	double norm[2] = {0.0, 0.0};
	CudaCheck(cudaMemcpyAsync(norm, scratch_.get()+PartialSlots(), 2*sizeof(double), cudaMemcpyDeviceToHost,
		mesh_.stream()),
		"transport norm");
	CudaCheck(cudaStreamSynchronize(mesh_.stream()), "transport norm");
	return norm[0];
}

} // namespace tfiga
