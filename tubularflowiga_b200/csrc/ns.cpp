// Newton iteration and physical step on the device (see ns.hpp).
#include "ns.hpp"

#include "case_input.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <cstdio>
#include <sstream>
#include <string>

namespace tfiga {

namespace {

std::string Precise(double v)
{
	char buffer[64];
	std::snprintf(buffer, sizeof(buffer), "%.16e", v);
	return buffer;
}

// Scalar slots in scalars_ / pinned_.
enum : int { kContinuity = 0 /* sq, sum */, kNorm = 2 /* norm, sum */, kUpdateNorm = 4, kOutletAccepted = 6,
	kSlots = 8 };

} // namespace

NsSolver::NsSolver(Mesh& mesh, const tfiga_ns_params& params)
	: mesh_(mesh), params_(params), n4_(4*mesh.nodes()),
	  gmres_((int)mesh.nodes(), params.gmres_restart > 0 ? params.gmres_restart : 200, mesh.stream())
{
	if (!(params.density > 0.0) || !std::isfinite(params.density) || !(params.viscosity > 0.0)
		|| !std::isfinite(params.viscosity) || !std::isfinite(params.dt) || params.dt < 0.0)
		Fail(-1, "invalid Navier-Stokes density, dynamic viscosity, or time step");
	if (params.dt > 0.0) {
		const double inverse = 1.0/params.dt;
		if (!std::isfinite(4.0*inverse*inverse) || !std::isfinite(params.density*inverse))
			Fail(-1, "transient Navier-Stokes time step is not representable");
	}
	if (mesh.bad_samples() > 0)
		Fail(-5, "mesh has "+std::to_string(mesh.bad_samples())+" non-positive quadrature Jacobians; minimum detJ "
			+std::to_string(mesh.min_detj()));
	stream_ = mesh.stream();
	const int64_t n = mesh.nodes();
	if (params.precision != TFIGA_PRECISION_FP64 && params.precision != TFIGA_PRECISION_MIXED
		&& params.precision != TFIGA_PRECISION_FP32_JACOBIAN && params.precision != TFIGA_PRECISION_MIXED_BF16X3
		&& params.precision != TFIGA_PRECISION_MIXED_TF32)
		Fail(-1, "unknown precision "+std::to_string(params.precision));
	if (!(params.tangent_reuse_factor >= 0.0 && std::isfinite(params.tangent_reuse_factor)))
		Fail(-1, "tangent_reuse_factor must be finite and non-negative");
	if (!tensor_tangent()) values_.Allocate((size_t)blocks()*16);
	rhs_.Allocate(n4_); state_.Allocate(n4_); previous_.Allocate(n4_); update_.Allocate(n4_);
	traction_.Allocate(n4_);
	velocity_bc_.Allocate(3*n); pressure_bc_.Allocate(n);
	vmask_.Allocate(n); pmask_.Allocate(n); constrained_.Allocate(n);
	for (auto* a : {&rhs_, &state_, &previous_, &update_, &traction_, &velocity_bc_, &pressure_bc_}) a->Zero(stream_);
	vmask_.Zero(stream_); pmask_.Zero(stream_);
	partial_.Allocate(PartialSlots());
	scalars_.Allocate(kSlots);
	// Label slots of the boundary faces.
	for (const auto& f : mesh.faces())
		if (!slot_of_label_.count(f.label)) { slot_of_label_[f.label] = 0; }
	int slot = 0;
	for (auto& entry : slot_of_label_) { entry.second = slot++; labels_.push_back(entry.first); }
	for (const auto& f : mesh.faces()) face_slot_host_.push_back(slot_of_label_[f.label]);
	const size_t faces = mesh.faces().size();
	if (faces) {
		face_flow_.Allocate(faces);
		face_pressure_.Allocate(faces);
		face_pressure_.Zero(stream_);
		face_slot_.Allocate(faces);
		face_slot_.Upload(face_slot_host_.data(), faces, stream_);
	}
	label_flow_.Allocate(std::max<size_t>(1, labels_.size()));
	CudaCheck(cudaMallocHost(reinterpret_cast<void**>(&pinned_), sizeof(double)*(kSlots+labels_.size()+1)),
		"pinned scalars");
	for (auto& ev : events_) CudaCheck(cudaEventCreate(&ev), "event");
	gmres_.set_profiler(&profiler_);
	if (mixed() && params.preconditioner != TFIGA_PRECONDITIONER_AMG)
		Fail(-7, "mixed precision requires the AMG-preconditioned flexible GMRES");
	if (mixed()) values32_.Allocate((size_t)blocks()*16);
	if (params.tangent_kernel != TFIGA_TANGENT_AUTO && params.tangent_kernel != TFIGA_TANGENT_COEFFICIENTS
		&& params.tangent_kernel != TFIGA_TANGENT_FUSED && params.tangent_kernel != TFIGA_TANGENT_ELEMENT)
		Fail(-1, "unknown tangent_kernel "+std::to_string(params.tangent_kernel));
	tangent_kernel_ = params.tangent_kernel;
	if (tensor_tangent()) {
		const size_t regular = (size_t)mesh.regular_elements();
		if (coefficient_arrays()) coef32_.Allocate(regular*4*80*64);
		else point_state_.Allocate(regular*kQuad*22);
	}
	if (tensor_tangent()) {
		status_.Allocate(1);
		status_.Zero(stream_);
		CudaCheck(cudaMallocHost(reinterpret_cast<void**>(&pinned_status_), sizeof(int32_t)), "pinned status");
		*pinned_status_ = 0;
	}
	if (params.preconditioner == TFIGA_PRECONDITIONER_AMG) {
		if (params.amg_coarse_nodes < 1 || params.amg_coarse_nodes > 2048)
			Fail(-1, "amg_coarse_nodes must be in [1, 2048]");
		if (params.amg_coarse_period < 1) Fail(-1, "amg_coarse_period must be positive");
		AmgOptions options;
		options.coarsest_nodes = params.amg_coarse_nodes;
		amg_ = std::make_unique<Amg>(mesh.pattern_view(), mesh.pattern().row_offsets, mesh.pattern().columns, stream_,
			options);
		amg_->set_profiler(&profiler_);
	} else if (params.preconditioner != TFIGA_PRECONDITIONER_BLOCK_JACOBI) {
		Fail(-1, "unknown preconditioner "+std::to_string(params.preconditioner));
	}
	CudaCheck(cudaStreamSynchronize(stream_), "solver setup");
}

NsSolver::~NsSolver()
{
	for (auto& ev : events_) if (ev) cudaEventDestroy(ev);
	if (pinned_) cudaFreeHost(pinned_);
	if (pinned_segments_) cudaFreeHost(pinned_segments_);
	if (pinned_status_) cudaFreeHost(pinned_status_);
}

void NsSolver::SetDirichlet(const int32_t* vmask, const int32_t* pmask, const double* velocity, const double* pressure)
{
	const int64_t n = nodes();
	std::vector<int32_t> vm(vmask, vmask+n), pm(n, 0), list;
	if (pmask) pm.assign(pmask, pmask+n);
	for (int64_t i = 0; i < n; ++i) {
		vm[i] = vm[i] ? 1 : 0; pm[i] = pm[i] ? 1 : 0;
		if (vm[i] || pm[i]) list.push_back((int32_t)i);
	}
	vmask_.Upload(vm.data(), n, stream_);
	pmask_.Upload(pm.data(), n, stream_);
	if (amg_) amg_->SetMasks(vm, pm);
	if (!list.empty()) constrained_.Upload(list.data(), list.size(), stream_);
	constrained_count_ = (int)list.size();
	SetDirichletValues(velocity, pressure);
	CudaCheck(cudaStreamSynchronize(stream_), "Dirichlet upload");
	dirichlet_set_ = true;
	tangent_valid_ = false;
	amg_current_ = false;
	lr_dirty_ = true;
}

void NsSolver::SetDirichletValues(const double* velocity, const double* pressure)
{
	const int64_t n = nodes();
	if (velocity) velocity_bc_.Upload(velocity, 3*n, stream_);
	if (pressure) pressure_bc_.Upload(pressure, n, stream_);
}

void NsSolver::SetTractions(const int32_t* labels, const double* pressures, int count)
{
	std::map<int32_t, double> traction;
	for (int i = 0; i < count; ++i) {
		if (!std::isfinite(pressures[i])) Fail(-1, "pressure traction must be finite");
		traction[labels[i]] = pressures[i];
	}
	ApplyTractions(traction);
	tractions_ = traction;
}

void NsSolver::ApplyTractions(const std::map<int32_t, double>& traction)
{
	for (const auto& t : traction) {
		bool found = false;
		for (const auto& f : mesh_.faces()) if (f.label == t.first) { found = true; break; }
		if (!found)
			Fail(-4, "pressure traction label "+std::to_string(t.first)
				+" has no boundary faces in the .ntiga database; repack with iga_pack");
	}
	const auto& faces = mesh_.faces();
	std::vector<double> fp(faces.size(), 0.0);
	for (size_t i = 0; i < faces.size(); ++i) {
		const auto it = traction.find(faces[i].label);
		if (it != traction.end()) fp[i] = it->second;
	}
	traction_.Zero(stream_);
	if (!faces.empty()) {
		face_pressure_.Upload(fp.data(), fp.size(), stream_);
		LaunchFaceTraction((int)faces.size(), mesh_.face_element(), mesh_.face_coef(), mesh_.face_stride(),
			mesh_.view().element_offsets, mesh_.view().connectivity, face_pressure_.get(), traction_.get(), stream_);
		launches_ += 1;
	}
	CudaCheck(cudaStreamSynchronize(stream_), "traction");
}

void NsSolver::SetState(const double* state, const double* previous)
{
	tangent_valid_ = false;
	state_.Upload(state, n4_, stream_);
	previous_.Upload(previous ? previous : state, n4_, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "state upload");
}

void NsSolver::GetState(double* state)
{
	state_.Download(state, n4_, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "state download");
}

void NsSolver::CommitStep()
{
	tangent_valid_ = false;
	CudaCheck(cudaMemcpyAsync(previous_.get(), state_.get(), n4_*sizeof(double), cudaMemcpyDeviceToDevice, stream_),
		"previous-state copy");
}

void NsSolver::AssembleResidualTc()
{
	profiler_.Begin(Profiler::kVector, stream_);
	rhs_.Zero(stream_);
	profiler_.End(stream_);
	profiler_.Begin(Profiler::kResidual, stream_);
	const bool coefficients = coefficient_arrays();
	LaunchTangentPoint(mesh_.regular_view(), mesh_.phi(), mesh_.qdata(), state_.get(), previous_.get(),
		{params_.density, params_.viscosity, params_.dt}, coefficients ? coef32_.get() : nullptr,
		coefficients ? nullptr : point_state_.get(), rhs_.get(), stream_);
	LargeElements<float>(nullptr, rhs_.get());
	profiler_.End(stream_);
	profiler_.Begin(Profiler::kVector, stream_);
	LaunchAxpy(n4_, 1.0, traction_.get(), rhs_.get(), stream_);
	profiler_.End(stream_);
	launches_ += 2;
}

template <class T>
void NsSolver::LargeElements(T* values, double* rhs)
{
	if (mesh_.large_count() == 0) return;
	LaunchAssembleLarge<T>(mesh_.view(), mesh_.large_first(), mesh_.large_count(), mesh_.phi_large(), mesh_.qdata(),
		mesh_.element_blocks_large(), state_.get(), previous_.get(), {params_.density, params_.viscosity, params_.dt},
		values, rhs, stream_);
	launches_ += 1;
}

void NsSolver::AssembleTangentTc()
{
	amg_current_ = false;
	const int operands = tc_operands();
	const AssemblyParams prm{params_.density, params_.viscosity, params_.dt};
	profiler_.Begin(Profiler::kAssembly, stream_);
	if (tangent_kernel_ == TFIGA_TANGENT_AUTO) {
		AutotuneTangent();
	} else {
		values32_.Zero(stream_);
		if (tangent_kernel_ == TFIGA_TANGENT_FUSED)
			LaunchTangentTcFused(mesh_.regular_view(), mesh_.phi(), mesh_.qdata(), point_state_.get(), prm,
				mesh_.element_blocks(), values32_.get(), status_.get(), operands, stream_);
		else if (tangent_kernel_ == TFIGA_TANGENT_ELEMENT)
			LaunchTangentTcElement(mesh_.regular_view(), mesh_.phi32(), coef32_.get(), mesh_.element_blocks(),
				values32_.get(), status_.get(), operands, stream_);
		else
			LaunchTangentTc(mesh_.regular_view(), mesh_.phi32(), coef32_.get(), mesh_.element_blocks(),
				values32_.get(), status_.get(), operands, stream_);
		launches_ += 1;
	}
	LargeElements<float>(values32_.get(), nullptr);
	profiler_.End(stream_);
	if (amg_ && !amg_->built()) amg_->Build(values32_.get());
}

void NsSolver::AutotuneTangent()
{
	const int operands = tc_operands();
	const AssemblyParams prm{params_.density, params_.viscosity, params_.dt};
	const DeviceMeshView view = mesh_.regular_view();
	cudaEvent_t ev[4];
	for (auto& e : ev) CudaCheck(cudaEventCreate(&e), "autotune event");
	struct Events {
		cudaEvent_t* e;
		~Events() { for (int i = 0; i < 4; ++i) cudaEventDestroy(e[i]); }
	} guard{ev};
	// the fused organisation first: the residual pass has just stored its point state
	values32_.Zero(stream_);
	CudaCheck(cudaEventRecord(ev[0], stream_), "event");
	LaunchTangentTcFused(view, mesh_.phi(), mesh_.qdata(), point_state_.get(), prm, mesh_.element_blocks(),
		values32_.get(), status_.get(), operands, stream_);
	CudaCheck(cudaEventRecord(ev[1], stream_), "event");
	launches_ += 1;
	CudaCheck(cudaStreamSynchronize(stream_), "tangent autotune");
	float ms = 0.0f;
	CudaCheck(cudaEventElapsedTime(&ms, ev[0], ev[1]), "event time");
	tune_ms_[1] = ms;
	// the coefficient-array organisation, when its arrays fit with 2 GiB to spare
	const size_t regular = (size_t)mesh_.regular_elements();
	const size_t need = regular*4*80*64*sizeof(float)+regular*kFeatures*kQuad*kMaxBasis*sizeof(float);
	size_t free_bytes = 0, total_bytes = 0;
	CudaCheck(cudaMemGetInfo(&free_bytes, &total_bytes), "device memory");
	if (free_bytes < need+(size_t(2) << 30)) {
		tangent_kernel_ = TFIGA_TANGENT_FUSED;
		return;
	}
	coef32_.Allocate(regular*4*80*64);
	// the same state's coefficients; the residual this pass adds goes to the Newton update vector,
	// which the linear solve clears before use
	LaunchTangentPoint(view, mesh_.phi(), mesh_.qdata(), state_.get(), previous_.get(), prm, coef32_.get(), nullptr,
		update_.get(), stream_);
	const float* phi32 = mesh_.phi32();
	values32_.Zero(stream_);
	CudaCheck(cudaEventRecord(ev[2], stream_), "event");
	LaunchTangentTc(view, phi32, coef32_.get(), mesh_.element_blocks(), values32_.get(), status_.get(), operands,
		stream_);
	CudaCheck(cudaEventRecord(ev[3], stream_), "event");
	launches_ += 2;
	CudaCheck(cudaStreamSynchronize(stream_), "tangent autotune");
	CudaCheck(cudaEventElapsedTime(&ms, ev[2], ev[3]), "event time");
	tune_ms_[0] = ms;
	// the same arrays contracted element by element (its tangent, equal to the others' up to the order
	// of the FP32 additions, is the one kept)
	values32_.Zero(stream_);
	CudaCheck(cudaEventRecord(ev[2], stream_), "event");
	LaunchTangentTcElement(view, phi32, coef32_.get(), mesh_.element_blocks(), values32_.get(), status_.get(),
		operands, stream_);
	CudaCheck(cudaEventRecord(ev[3], stream_), "event");
	launches_ += 1;
	CudaCheck(cudaStreamSynchronize(stream_), "tangent autotune");
	CudaCheck(cudaEventElapsedTime(&ms, ev[2], ev[3]), "event time");
	tune_ms_[2] = ms;
	const double arrays_ms = std::min(tune_ms_[0], tune_ms_[2]);
	if (arrays_ms < tune_ms_[1]) {
		tangent_kernel_ = tune_ms_[2] <= tune_ms_[0] ? TFIGA_TANGENT_ELEMENT : TFIGA_TANGENT_COEFFICIENTS;
		point_state_.Release();
	} else {
		tangent_kernel_ = TFIGA_TANGENT_FUSED;
		coef32_.Release();
		mesh_.ReleasePhi32();
	}
}

void NsSolver::AssembleResidual()
{
	if (tensor_tangent()) {
		AssembleResidualTc();
		return;
	}
	profiler_.Begin(Profiler::kVector, stream_);
	rhs_.Zero(stream_);
	profiler_.End(stream_);
	profiler_.Begin(Profiler::kResidual, stream_);
	LaunchTangentPoint(mesh_.regular_view(), mesh_.phi(), mesh_.qdata(), state_.get(), previous_.get(),
		{params_.density, params_.viscosity, params_.dt}, nullptr, nullptr, rhs_.get(), stream_);
	LargeElements<double>(nullptr, rhs_.get());
	profiler_.End(stream_);
	profiler_.Begin(Profiler::kVector, stream_);
	LaunchAxpy(n4_, 1.0, traction_.get(), rhs_.get(), stream_);
	profiler_.End(stream_);
	launches_ += 2;
}

void NsSolver::AssembleTangent()
{
	if (tensor_tangent()) {
		AssembleTangentTc();
		return;
	}
	amg_current_ = false;
	profiler_.Begin(Profiler::kAssembly, stream_);
	values_.Zero(stream_);
	LaunchAssemble(mesh_.regular_view(), mesh_.phi(), mesh_.qdata(), mesh_.element_blocks(), state_.get(),
		previous_.get(), {params_.density, params_.viscosity, params_.dt}, values_.get(), nullptr, stream_);
	LargeElements<double>(values_.get(), nullptr);
	if (mixed()) {
		LaunchToFloat((long long)blocks()*16, values_.get(), values32_.get(), stream_);
		launches_ += 1;
	}
	profiler_.End(stream_);
	launches_ += 1;
	if (amg_ && !amg_->built()) {
		if (mixed()) amg_->Build(values32_.get());
		else amg_->Build(values_.get());
	}
}

void NsSolver::Assemble()
{
	if (tensor_tangent()) {
		AssembleResidualTc();
		AssembleTangentTc();
		return;
	}
	amg_current_ = false;
	values_.Zero(stream_);
	rhs_.Zero(stream_);
	profiler_.Begin(Profiler::kAssembly, stream_);
	LaunchAssemble(mesh_.regular_view(), mesh_.phi(), mesh_.qdata(), mesh_.element_blocks(), state_.get(),
		previous_.get(), {params_.density, params_.viscosity, params_.dt}, values_.get(), rhs_.get(), stream_);
	LargeElements<double>(values_.get(), rhs_.get());
	profiler_.End(stream_);
	LaunchAxpy(n4_, 1.0, traction_.get(), rhs_.get(), stream_);
	launches_ += 2;
	if (mixed()) {
		LaunchToFloat((long long)blocks()*16, values_.get(), values32_.get(), stream_);
		launches_ += 1;
	}
	// The AMG hierarchy is built once, from the strength of the first raw (pre-Dirichlet) Jacobian.
	if (amg_ && !amg_->built()) {
		if (mixed()) amg_->Build(values32_.get());
		else amg_->Build(values_.get());
	}
}

void NsSolver::ApplyDirichlet()
{
	ApplyDirichletParts(true, true);
}

void NsSolver::LiftDirichletForForcing()
{
	if (!params_.newton_forcing || !dirichlet_set_) return;
	LaunchLiftDirichlet(constrained_count_, constrained_.get(), vmask_.get(), pmask_.get(), velocity_bc_.get(),
		pressure_bc_.get(), state_.get(), stream_);
	launches_ += 1;
}

void NsSolver::ApplyDirichletRhs()
{
	ApplyDirichletParts(false, true);
}

void NsSolver::ApplyDirichletMatrix()
{
	ApplyDirichletParts(true, false);
}

void NsSolver::ApplyDirichletParts(bool matrix, bool rhs)
{
	if (matrix) amg_current_ = false;
	if (!dirichlet_set_) Fail(-1, "Dirichlet conditions have not been set");
	double* r = rhs ? rhs_.get() : nullptr;
	if (mixed())
		LaunchDirichletRows<float>(mesh_.pattern_view(), constrained_count_, constrained_.get(), vmask_.get(),
			pmask_.get(), velocity_bc_.get(), pressure_bc_.get(), state_.get(), matrix ? values32_.get() : nullptr, r,
			stream_);
	else
		LaunchDirichletRows<double>(mesh_.pattern_view(), constrained_count_, constrained_.get(), vmask_.get(),
			pmask_.get(), velocity_bc_.get(), pressure_bc_.get(), state_.get(), matrix ? values_.get() : nullptr, r,
			stream_);
	launches_ += 1;
}

GmresResult NsSolver::SolveLinear(double rtol, int max_iterations)
{
	profiler_.Begin(Profiler::kVector, stream_);
	update_.Zero(stream_);
	profiler_.End(stream_);
	struct Count { long long& n; ~Count() { ++n; } } count{solves_};
	if (amg_) {
		const long long before = amg_->launches();
		GmresResult result;
		auto solve = [&]() {
			// batched tubes: one Arnoldi process per tube over the shared launches
			if (segments_ && mixed())
				return gmres_.SolveFlexibleSegments<float>(mesh_.pattern_view(), values32_.get(), rhs_.get(),
					update_.get(), rtol, max_iterations, *amg_, &launches_, params_.krylov_fp64_basis != 0);
			if (segments_)
				return gmres_.SolveFlexibleSegments<double>(mesh_.pattern_view(), values_.get(), rhs_.get(),
					update_.get(), rtol, max_iterations, *amg_, &launches_);
			if (mixed())
				return gmres_.SolveFlexible<float>(mesh_.pattern_view(), values32_.get(), rhs_.get(), update_.get(),
					rtol, max_iterations, *amg_, &launches_, params_.krylov_fp64_basis != 0);
			return gmres_.SolveFlexible<double>(mesh_.pattern_view(), values_.get(), rhs_.get(), update_.get(), rtol,
				max_iterations, *amg_, &launches_);
		};
		// refresh the AMG data only when the Jacobian changed since the last refresh (a reused
		// tangent keeps them); the dense coarse inverse every amg_coarse_period-th refresh
		if (!amg_current_) {
			const bool coarse = refreshes_ % params_.amg_coarse_period == 0;
			profiler_.Begin(Profiler::kSetup, stream_);
			if (mixed()) {
				if (!amg_->built()) amg_->Build(values32_.get());
				amg_->Refresh(values32_.get(), coarse);
			} else {
				if (!amg_->built()) amg_->Build(values_.get());
				amg_->Refresh(values_.get(), coarse);
			}
			profiler_.End(stream_);
			++refreshes_;
			amg_current_ = true;
		}
		launches_ += amg_->launches()-before;
		result = solve();
		if (!result.converged && gmres_.learned() != nullptr) {
			// the learned stage is only an accelerator: the AMG-only solve is its fallback
			LearnedPreconditioner* learned = gmres_.learned();
			gmres_.set_learned(nullptr);
			update_.Zero(stream_);
			const int spent = result.iterations;
			try {
				result = solve();
			} catch (...) {
				gmres_.set_learned(learned);
				throw;
			}
			gmres_.set_learned(learned);
			result.iterations += spent;
			++learned_fallbacks_;
		}
		return result;
	}
	return gmres_.Solve(mesh_.pattern_view(), values_.get(), rhs_.get(), update_.get(), rtol, max_iterations,
		&launches_);
}

void NsSolver::LaunchDiagnostics(bool flows)
{
	LaunchStridedSums(nodes(), 4, 3, rhs_.get(), partial_.get(), scalars_.get()+kContinuity, stream_);
	launches_ += 2;
	const int faces = (int)mesh_.faces().size();
	if (faces && flows) {
		LaunchFaceFlows(faces, mesh_.face_element(), mesh_.face_coef(), mesh_.face_stride(),
			mesh_.view().element_offsets, mesh_.view().connectivity, state_.get(), face_flow_.get(), stream_);
		LaunchSegmentSums((int)labels_.size(), face_slot_.get(), faces, face_flow_.get(), label_flow_.get(), stream_);
		launches_ += 2;
	}
}

NsSolver::Diagnostics NsSolver::ReadDiagnostics()
{
	// pinned_ already holds the downloaded values (see NewtonIteration).
	Diagnostics d{};
	d.continuity_l2 = std::sqrt(pinned_[kContinuity]);
	d.continuity_sum = pinned_[kContinuity+1];
	for (size_t i = 0; i < labels_.size(); ++i) {
		d.net_flow += pinned_[kSlots+i];
		d.absolute_flow += std::fabs(pinned_[kSlots+i]);
	}
	d.imbalance = d.absolute_flow > 0.0 ? 2.0*std::fabs(d.net_flow)/d.absolute_flow : 0.0;
	return d;
}

tfiga_newton_report NsSolver::NewtonIteration(double initial_residual)
{
	tfiga_newton_report report{};
	// Residual first (every precision mode): the FP64 residual comes from its own kernel, so the
	// convergence test runs before the tangent, and an iteration that passes it assembles no
	// tangent at all.  The residual is the one the combined assembly computes (same point
	// formulas, FP64), so only the order of the floating-point sums differs.
	const bool tc = tensor_tangent();
	CudaCheck(cudaEventRecord(events_[0], stream_), "event");
	const bool outlets = outlet_count_ >= 0;
	if (outlets) {
		profiler_.Begin(Profiler::kVector, stream_);
		CoupleOutletsOnDevice();
		profiler_.End(stream_);
	}
	AssembleResidual();
	profiler_.Begin(Profiler::kVector, stream_);
	LaunchDiagnostics(!outlets);
	ApplyDirichletRhs();
	LaunchNorm(n4_, rhs_.get(), partial_.get(), scalars_.get()+kNorm, stream_);
	launches_ += 2;
	if (segments_) {
		LaunchSegmentSquares(segments_, segment_entries_.get(), rhs_.get(), segment_sq_.get(), stream_);
		segment_sq_.Download(pinned_segments_, segments_, stream_);
		launches_ += 1;
	}
	profiler_.End(stream_);
	CudaCheck(cudaEventRecord(events_[1], stream_), "event");
	scalars_.Download(pinned_, kSlots, stream_);
	if (!labels_.empty()) label_flow_.Download(pinned_+kSlots, labels_.size(), stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "Navier-Stokes assembly");
	float ms = 0.0f;
	CudaCheck(cudaEventElapsedTime(&ms, events_[0], events_[1]), "event time");
	report.assembly_ms = ms;
	if (outlets) last_outlet_ok_ = pinned_[kOutletAccepted] != 0.0;
	const Diagnostics d = ReadDiagnostics();
	report.continuity_l2 = d.continuity_l2;
	report.continuity_sum = d.continuity_sum;
	report.net_boundary_flow = d.net_flow;
	report.absolute_boundary_flow = d.absolute_flow;
	report.relative_mass_imbalance = d.imbalance;
	const double norm = pinned_[kNorm];
	report.residual_l2 = norm;
	if (!std::isfinite(norm)) Fail(-6, "Navier-Stokes residual is not finite");
	const double initial = initial_residual < 0.0 ? norm : initial_residual;
	const double scale = std::sqrt((double)n4_);
	report.tolerance = std::max(params_.nonlinear_atol*scale, params_.nonlinear_rtol*initial);
	bool residual_ok = norm <= report.tolerance;
	double floor_ratio = report.tolerance/norm;       // reduction the open Newton tests still ask for
	if (segments_) {
		// per-segment Newton tests; a segment that passed stays frozen for the rest of the step
		if (initial_residual < 0.0) std::fill(segment_done_host_.begin(), segment_done_host_.end(), 0);
		residual_ok = true;
		floor_ratio = std::numeric_limits<double>::infinity();
		for (int k = 0; k < segments_; ++k) {
			segment_norm_[k] = std::sqrt(pinned_segments_[k]);
			if (initial_residual < 0.0) segment_initial_[k] = segment_norm_[k];
			const double tol = std::max(params_.nonlinear_atol*std::sqrt(4.0*(segment_nodes_[k+1]-segment_nodes_[k])),
				params_.nonlinear_rtol*segment_initial_[k]);
			if (segment_norm_[k] <= tol) segment_done_host_[k] = 1;
			if (!segment_done_host_[k]) {
				residual_ok = false;
				floor_ratio = std::min(floor_ratio, tol/segment_norm_[k]);
			}
		}
		if (!std::isfinite(floor_ratio)) floor_ratio = report.tolerance/norm;
	}
	if (residual_ok && d.imbalance <= params_.mass_rtol) {
		report.converged = 1;
		return report;
	}
	if (segments_) {
		// Frozen segments take no update: their rhs rows vanish before the linear solve.  Each open
		// segment's rhs is scaled to unit norm, so that the union's Krylov solve weighs every segment
		// alike instead of resolving the small ones only to the large ones' absolute accuracy; the
		// Jacobian is block diagonal over the segments, so a segment's solution scales by the same
		// factor and is scaled back after the solve.
		for (int k = 0; k < segments_; ++k) {
			const bool open = !segment_done_host_[k] && segment_norm_[k] > 0.0;
			segment_scale_host_[k] = open ? 1.0/segment_norm_[k] : 0.0;
			segment_scale_host_[segments_+k] = open ? segment_norm_[k] : 0.0;
		}
		profiler_.Begin(Profiler::kVector, stream_);
		segment_scale_.Upload(segment_scale_host_.data(), 2*segments_, stream_);
		LaunchScaleSegments(segments_, segment_entries_.get(), segment_scale_.get(), rhs_.get(), stream_);
		profiler_.End(stream_);
		launches_ += 1;
	}
	// Tangent reuse: keep the previous iteration's tangent while that iteration contracted the
	// residual about as far as its linear tolerance allowed.
	const bool reuse = params_.tangent_reuse_factor > 0.0 && tangent_valid_ && initial_residual >= 0.0
		&& norm <= params_.tangent_reuse_factor*reuse_eta_*reuse_norm_;
	reuse_norm_ = norm;
	if (!reuse) {
		CudaCheck(cudaEventRecord(events_[4], stream_), "event");
		AssembleTangent();
		profiler_.Begin(Profiler::kVector, stream_);
		ApplyDirichletMatrix();
		profiler_.End(stream_);
		tangent_valid_ = true;
		++tangent_contractions_;
		CudaCheck(cudaEventRecord(events_[5], stream_), "event");
		if (tc) status_.Download(pinned_status_, 1, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "tangent assembly");
		if (tc && *pinned_status_ != 0)
			Fail(-2, "tensor-core tangent: an MMA completion wait expired (status "+std::to_string(*pinned_status_)+")");
		CudaCheck(cudaEventElapsedTime(&ms, events_[4], events_[5]), "event time");
		report.assembly_ms += ms;
	}
	CudaCheck(cudaEventRecord(events_[2], stream_), "event");
	// Linear tolerance: gmres_rtol, or the Eisenstat-Walker forcing term (choice 2, gamma 0.9,
	// alpha 2) with its safeguard, capped at 1e-3, floored at gmres_rtol and at half of what the
	// Newton test still asks for, so the last solve does not oversolve.
	double eta = params_.gmres_rtol;
	if (params_.newton_forcing) {
		constexpr double kEtaMax = 1e-3;
		if (initial_residual < 0.0) eta = kEtaMax;
		else {
			// with segments, the slowest-contracting open segment's ratio (each is solved at unit scale)
			double ratio = norm/forcing_norm_;
			if (segments_) {
				ratio = 0.0;
				for (int k = 0; k < segments_; ++k)
					if (!segment_done_host_[k] && segment_forcing_[k] > 0.0)
						ratio = std::max(ratio, segment_norm_[k]/segment_forcing_[k]);
			}
			eta = 0.9*ratio*ratio;
			const double safeguard = 0.9*forcing_eta_*forcing_eta_;
			if (safeguard > 0.1) eta = std::max(eta, safeguard);
			eta = std::min(eta, kEtaMax);
		}
		eta = std::max(eta, params_.gmres_rtol);
		eta = std::max(eta, std::min(0.1, 0.5*floor_ratio));
		forcing_norm_ = norm;
		forcing_eta_ = eta;
		if (segments_) segment_forcing_ = segment_norm_;
	}
	reuse_eta_ = eta;
	const GmresResult linear = SolveLinear(eta, params_.gmres_max_iterations);
	CudaCheck(cudaEventRecord(events_[3], stream_), "event");
	report.linear_iterations = linear.iterations;
	report.linear_residual = linear.residual;
	report.singular_diagonal_blocks = (int32_t)linear.singular_blocks;
	if (!linear.converged)
		Fail(-6, "Navier-Stokes GMRES failed (residual="+Precise(linear.residual)+", nonlinear_residual="
			+Precise(norm)+", continuity_l2="+Precise(d.continuity_l2)+", net_boundary_flow="+Precise(d.net_flow)
			+", relative_mass_imbalance="+Precise(d.imbalance)+")");
	if (collect_pairs_) {
		// training pair of this solved system, with the AMG data of this Jacobian
		LaunchApplyBlockInverse((int)nodes(), amg_->fine_inverse(), rhs_.get(), pair_dinv_.get(), stream_);
		if (mixed()) {
			amg_->Apply(values32_.get(), rhs_.get(), pair_amg_.get(), zero_flag_.get());
			LaunchSpmv<float>(mesh_.pattern_view(), values32_.get(), pair_amg_.get(), pair_aamg_.get(), stream_);
		} else {
			amg_->Apply(values_.get(), rhs_.get(), pair_amg_.get(), zero_flag_.get());
			LaunchSpmv<double>(mesh_.pattern_view(), values_.get(), pair_amg_.get(), pair_aamg_.get(), stream_);
		}
		learned_->AddSolvedPair(pair_dinv_.get(), update_.get(), pair_amg_.get(), rhs_.get(), pair_aamg_.get(), norm);
		launches_ += 6;
	}
	profiler_.Begin(Profiler::kVector, stream_);
	if (segments_) {
		LaunchScaleSegments(segments_, segment_entries_.get(), segment_scale_.get()+segments_, update_.get(), stream_);
		launches_ += 1;
	}
	LaunchNorm(n4_, update_.get(), partial_.get(), scalars_.get()+kUpdateNorm, stream_);
	LaunchAxpy(n4_, 1.0, update_.get(), state_.get(), stream_);
	profiler_.End(stream_);
	launches_ += 3;
	scalars_.Download(pinned_+kUpdateNorm, 1, stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "Navier-Stokes update");
	CudaCheck(cudaEventElapsedTime(&ms, events_[2], events_[3]), "event time");
	report.linear_ms = ms;
	report.update_l2 = pinned_[kUpdateNorm];
	return report;
}

tfiga_step_report NsSolver::Step()
{
	tfiga_step_report step{};
	double initial = -1.0;
	LiftDirichletForForcing();
	const int max_newton = params_.max_newton > 0 ? params_.max_newton : 12;
	tfiga_newton_report last{};
	for (int k = 0; k < max_newton; ++k) {
		last = NewtonIteration(initial);
		if (initial < 0.0) { initial = last.residual_l2; step.initial_residual_l2 = initial; }
		step.assembly_ms += last.assembly_ms;
		step.linear_ms += last.linear_ms;
		step.linear_iterations += last.linear_iterations;
		step.residual_l2 = last.residual_l2;
		step.relative_mass_imbalance = last.relative_mass_imbalance;
		step.newton_iterations = k;
		if (last.converged) { step.converged = 1; return step; }
	}
	Fail(-6, "Navier-Stokes nonlinear solve reached MAX_NEWTON (nonlinear_residual="+Precise(last.residual_l2)
		+", continuity_l2="+Precise(last.continuity_l2)+", net_boundary_flow="+Precise(last.net_boundary_flow)
		+", relative_mass_imbalance="+Precise(last.relative_mass_imbalance)+")");
}

tfiga_step_report NsSolver::StepOutlets(tfiga_outlet* outlets, int count, double relaxation, int max_iterations,
	int* iterations)
{
	if (!(relaxation > 0.0 && relaxation <= 1.0)) Fail(-1, "invalid outlet coupling relaxation");
	if (max_iterations < 1) Fail(-1, "outlet coupling needs at least one iteration");
	std::vector<OutletModel> models = OutletModels(outlets, count);
	std::vector<int32_t> labels(count);
	std::vector<double> previous_capacitor(count), flows(count);
	for (int i = 0; i < count; ++i) {
		labels[i] = outlets[i].label;
		previous_capacitor[i] = outlets[i].capacitor_pressure;
	}
	tfiga_step_report total{};
	for (int coupling = 0; coupling < max_iterations; ++coupling) {
		auto traction = tractions_;
		for (const auto& m : models) traction[m.label] = m.pressure;
		ApplyTractions(traction);
		const tfiga_step_report r = Step();
		if (coupling == 0) total.initial_residual_l2 = r.initial_residual_l2;
		total.converged = r.converged;
		total.newton_iterations += r.newton_iterations;
		total.linear_iterations += r.linear_iterations;
		total.residual_l2 = r.residual_l2;
		total.relative_mass_imbalance = r.relative_mass_imbalance;
		total.assembly_ms += r.assembly_ms;
		total.linear_ms += r.linear_ms;
		if (count == 0) { if (iterations) *iterations = 1; return total; }
		BoundaryFlows(labels.data(), count, flows.data());
		double change = 0.0, scale = 1.0;
		std::vector<std::array<double, 2>> evaluated(count);
		for (int i = 0; i < count; ++i) {
			OutletModel m = models[i];
			m.capacitor_pressure = previous_capacitor[i];
			evaluated[i] = EvaluateOutletModel(m, flows[i], params_.dt);
			change = std::max(change, std::fabs(evaluated[i][0]-models[i].pressure));
			scale = std::max(scale, std::fabs(evaluated[i][0]));
		}
		if (change <= 1e-8+1e-6*scale) {
			for (int i = 0; i < count; ++i) {
				outlets[i].flow = flows[i];
				outlets[i].pressure = evaluated[i][0];
				outlets[i].capacitor_pressure = evaluated[i][1];
			}
			if (iterations) *iterations = coupling+1;
			return total;
		}
		for (int i = 0; i < count; ++i) {
			models[i].flow = flows[i];
			models[i].pressure = (1.0-relaxation)*models[i].pressure+relaxation*evaluated[i][0];
			outlets[i].flow = flows[i];
			outlets[i].pressure = models[i].pressure;
		}
	}
	if (iterations) *iterations = max_iterations;
	Fail(-6, "outlet fixed-point iteration did not converge");
}

std::vector<OutletModel> NsSolver::OutletModels(const tfiga_outlet* outlets, int count) const
{
	std::vector<OutletModel> models(count);
	for (int i = 0; i < count; ++i) {
		const tfiga_outlet& o = outlets[i];
		OutletModel& m = models[i];
		m.label = o.label;
		if (o.kind == TFIGA_OUTLET_RESISTANCE) m.kind = "resistance";
		else if (o.kind == TFIGA_OUTLET_RC) m.kind = "windkessel_rc";
		else if (o.kind == TFIGA_OUTLET_RCR) m.kind = "windkessel_rcr";
		else Fail(-1, "unknown outlet model kind "+std::to_string(o.kind));
		m.resistance = o.resistance;
		m.proximal = o.proximal_resistance;
		m.distal = o.distal_resistance;
		m.capacitance = o.capacitance;
		m.reference_pressure = o.reference_pressure;
		m.capacitor_pressure = o.capacitor_pressure;
		m.flow = o.flow;
		m.pressure = o.pressure;
		if (!std::isfinite(m.pressure)) Fail(-1, "outlet pressure must be finite");
	}
	return models;
}

void NsSolver::CoupleOutletsOnDevice()
{
	const int faces = (int)mesh_.faces().size();
	if (faces) {
		LaunchFaceFlows(faces, mesh_.face_element(), mesh_.face_coef(), mesh_.face_stride(),
			mesh_.view().element_offsets, mesh_.view().connectivity, state_.get(), face_flow_.get(), stream_);
		LaunchSegmentSums((int)labels_.size(), face_slot_.get(), faces, face_flow_.get(), label_flow_.get(), stream_);
		launches_ += 2;
	}
	LaunchOutletUpdate(outlet_count_, outlets_dev_.get(), label_flow_.get(), params_.dt, outlet_relaxation_,
		outlet_iteration_ > 0, scalars_.get()+kOutletAccepted, outlet_updates_.get(), stream_);
	launches_ += 1;
	traction_.Zero(stream_);
	if (faces) {
		LaunchFacePressures(faces, face_slot_.get(), slot_outlet_.get(), face_base_.get(), outlets_dev_.get(),
			face_pressure_.get(), stream_);
		LaunchFaceTraction(faces, mesh_.face_element(), mesh_.face_coef(), mesh_.face_stride(),
			mesh_.view().element_offsets, mesh_.view().connectivity, face_pressure_.get(), traction_.get(), stream_);
		launches_ += 2;
	}
	++outlet_iteration_;
}

tfiga_step_report NsSolver::StepOutletsCoupled(tfiga_outlet* outlets, int count, double relaxation, int max_newton,
	int* updates)
{
	if (!(relaxation > 0.0 && relaxation <= 1.0)) Fail(-1, "invalid outlet coupling relaxation");
	if (max_newton < 1) Fail(-1, "outlet coupling needs at least one Newton iteration");
	const std::vector<OutletModel> models = OutletModels(outlets, count);
	// The models, the label slot -> outlet map and the fixed per-face tractions go to the device once;
	// every Newton iteration then updates the outlets there (CoupleOutletsOnDevice).
	std::vector<DeviceOutlet> host(count);
	std::vector<int32_t> slot_outlet(std::max<size_t>(1, labels_.size()), -1);
	for (int i = 0; i < count; ++i) {
		const tfiga_outlet& o = outlets[i];
		if (o.kind != TFIGA_OUTLET_RESISTANCE && !(params_.dt > 0.0))
			Fail(-4, "RC/RCR outlets require positive transient dt");
		DeviceOutlet& d = host[i];
		d.kind = o.kind;
		const auto it = slot_of_label_.find(o.label);
		d.slot = it == slot_of_label_.end() ? -1 : it->second;
		if (d.slot >= 0) slot_outlet[d.slot] = i;
		d.resistance = o.resistance; d.proximal = o.proximal_resistance; d.distal = o.distal_resistance;
		d.capacitance = o.capacitance; d.reference_pressure = o.reference_pressure;
		d.capacitor_pressure = o.capacitor_pressure;
		d.pressure = models[i].pressure;
		d.flow = o.flow; d.evaluated = d.pressure; d.evaluated_capacitor = o.capacitor_pressure;
	}
	const auto& faces = mesh_.faces();
	std::vector<double> base(faces.size(), 0.0);
	for (size_t f = 0; f < faces.size(); ++f) {
		const auto it = tractions_.find(faces[f].label);
		if (it != tractions_.end()) base[f] = it->second;
	}
	if (outlets_dev_.size() < (size_t)std::max(1, count)) outlets_dev_.Allocate(std::max(1, count));
	if (slot_outlet_.size() < slot_outlet.size()) slot_outlet_.Allocate(slot_outlet.size());
	if (outlet_updates_.size() == 0) outlet_updates_.Allocate(1);
	if (!faces.empty() && face_base_.size() < faces.size()) face_base_.Allocate(faces.size());
	if (count) outlets_dev_.Upload(host.data(), count, stream_);
	slot_outlet_.Upload(slot_outlet.data(), slot_outlet.size(), stream_);
	if (!faces.empty()) face_base_.Upload(base.data(), base.size(), stream_);
	outlet_updates_.Zero(stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "outlet upload");
	// The coupling's share of the Newton Jacobian: the residual carries P_k(Q_k(u)) g_k with
	// Q_k = g_k . u the outward flow of outlet k (g_k the face coefficients of its label on the free
	// velocity unknowns), so its derivative is sum_k dP_k/dQ_k g_k g_k^T, with dP/dQ = relaxation x
	// (R | 1 / (C/dt + 1/R) | R1 + 1 / (C/dt + 1/R2)) for the resistance / RC / RCR models.  The flexible
	// GMRES applies it next to the SpMV, so Newton converges on the coupled system instead of lagging
	// the pressures one iteration behind.
	std::vector<int32_t> lr_labels;
	std::vector<double> lr_coef;
	for (int i = 0; i < count; ++i) {
		if (host[i].slot < 0) continue;
		const DeviceOutlet& d = host[i];
		double dpdq = 0.0;
		if (d.kind == TFIGA_OUTLET_RESISTANCE) dpdq = d.resistance;
		else if (d.kind == TFIGA_OUTLET_RC) dpdq = 1.0/(d.capacitance/params_.dt+1.0/d.resistance);
		else dpdq = d.proximal+1.0/(d.capacitance/params_.dt+1.0/d.distal);
		lr_labels.push_back(outlets[i].label);
		lr_coef.push_back(relaxation*dpdq);
	}
	if (amg_ && !lr_labels.empty()) {
		if (lr_dirty_ || lr_labels != lr_labels_) BuildOutletFlowVectors(lr_labels);
		lr_coef_.Upload(lr_coef.data(), lr_coef.size(), stream_);
		const Gmres::LowRank term{(int)lr_labels.size(), lr_ptr_.get(), lr_idx_.get(), lr_val_.get(), lr_coef_.get()};
		gmres_.set_low_rank(&term);
	}
	struct Deactivate {
		int& count;
		Gmres& gmres;
		~Deactivate() { count = -1; gmres.set_low_rank(nullptr); }
	} deactivate{outlet_count_, gmres_};
	outlet_count_ = count;
	outlet_relaxation_ = relaxation;
	outlet_iteration_ = 0;
	tfiga_step_report step{};
	double initial = -1.0;
	LiftDirichletForForcing();
	tfiga_newton_report last{};
	auto read_back = [&](bool accepted) {
		int32_t changes = 0;
		if (count) outlets_dev_.Download(host.data(), count, stream_);
		outlet_updates_.Download(&changes, 1, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "outlet read-back");
		for (int i = 0; i < count; ++i) {
			outlets[i].flow = host[i].flow;
			outlets[i].pressure = accepted ? host[i].evaluated : host[i].pressure;
			if (accepted) outlets[i].capacitor_pressure = host[i].evaluated_capacitor;
		}
		if (updates) *updates = changes;
	};
	for (int k = 0; k < max_newton; ++k) {
		last = NewtonIteration(initial);
		if (initial < 0.0) { initial = last.residual_l2; step.initial_residual_l2 = initial; }
		step.assembly_ms += last.assembly_ms;
		step.linear_ms += last.linear_ms;
		step.linear_iterations += last.linear_iterations;
		step.residual_l2 = last.residual_l2;
		step.relative_mass_imbalance = last.relative_mass_imbalance;
		if (!last.converged) ++step.newton_iterations;
		if (last.converged && last_outlet_ok_) {
			read_back(true);
			step.converged = 1;
			return step;
		}
	}
	read_back(false);
	Fail(-6, "Navier-Stokes nonlinear solve with coupled outlets reached MAX_NEWTON (nonlinear_residual="
		+Precise(last.residual_l2)+", relative_mass_imbalance="+Precise(last.relative_mass_imbalance)+")");
}

void NsSolver::BuildOutletFlowVectors(const std::vector<int32_t>& labels)
{
	const auto& faces = mesh_.faces();
	const int64_t n = nodes();
	std::vector<int32_t> vm(n);
	vmask_.Download(vm.data(), n, stream_);
	std::vector<int32_t> ptr{0}, idx;
	std::vector<double> val, g(n4_);
	std::vector<double> fp(faces.size());
	for (const int32_t label : labels) {
		// -F per unknown for a unit pressure on the label's faces (the traction kernel), i.e. -g
		for (size_t f = 0; f < faces.size(); ++f) fp[f] = faces[f].label == label ? 1.0 : 0.0;
		face_pressure_.Upload(fp.data(), fp.size(), stream_);
		update_.Zero(stream_);
		LaunchFaceTraction((int)faces.size(), mesh_.face_element(), mesh_.face_coef(), mesh_.face_stride(),
			mesh_.view().element_offsets, mesh_.view().connectivity, face_pressure_.get(), update_.get(), stream_);
		launches_ += 1;
		update_.Download(g.data(), n4_, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "outlet flow vector");
		for (int64_t i = 0; i < n; ++i) {
			if (vm[i]) continue;                              // Dirichlet velocity: no update, no flow change
			for (int c = 0; c < 3; ++c)
				if (g[4*i+c] != 0.0) { idx.push_back((int32_t)(4*i+c)); val.push_back(-g[4*i+c]); }
		}
		ptr.push_back((int32_t)idx.size());
	}
	lr_ptr_.Allocate(ptr.size());
	lr_ptr_.Upload(ptr.data(), ptr.size(), stream_);
	lr_idx_.Allocate(std::max<size_t>(1, idx.size()));
	lr_val_.Allocate(std::max<size_t>(1, val.size()));
	if (!idx.empty()) {
		lr_idx_.Upload(idx.data(), idx.size(), stream_);
		lr_val_.Upload(val.data(), val.size(), stream_);
	}
	lr_coef_.Allocate(labels.size());
	// (the face pressures are rebuilt from the outlet pressures before every coupled residual)
	CudaCheck(cudaStreamSynchronize(stream_), "outlet flow vectors");
	lr_labels_ = labels;
	lr_dirty_ = false;
}

void NsSolver::BoundaryFlows(const int32_t* labels, int count, double* flows)
{
	const int faces = (int)mesh_.faces().size();
	std::vector<double> per_label(labels_.size(), 0.0);
	if (faces) {
		LaunchFaceFlows(faces, mesh_.face_element(), mesh_.face_coef(), mesh_.face_stride(),
			mesh_.view().element_offsets, mesh_.view().connectivity, state_.get(), face_flow_.get(), stream_);
		LaunchSegmentSums((int)labels_.size(), face_slot_.get(), faces, face_flow_.get(), label_flow_.get(), stream_);
		launches_ += 2;
		label_flow_.Download(per_label.data(), labels_.size(), stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "boundary flows");
	}
	for (int i = 0; i < count; ++i) {
		const auto it = slot_of_label_.find(labels[i]);
		flows[i] = it == slot_of_label_.end() ? 0.0 : per_label[it->second];
	}
}

void NsSolver::SetSegments(const int64_t* node_offsets, int count)
{
	if (count < 0) Fail(-1, "segment count must be non-negative");
	if (count == 0) {
		segments_ = 0;
		gmres_.SetSegments({});
		if (amg_) amg_->SetSegments({});
		return;
	}
	if (node_offsets == nullptr) Fail(-1, "null segment offsets");
	if (node_offsets[0] != 0 || node_offsets[count] != nodes()) Fail(-1, "segments must cover the nodes from 0");
	for (int k = 0; k < count; ++k)
		if (!(node_offsets[k+1] > node_offsets[k])) Fail(-1, "segment offsets must increase");
	segment_nodes_.assign(node_offsets, node_offsets+count+1);
	std::vector<int64_t> entries(count+1), blocks(count);
	for (int k = 0; k <= count; ++k) entries[k] = 4*node_offsets[k];
	const auto& rows = mesh_.pattern().row_offsets;
	for (int k = 0; k < count; ++k) blocks[k] = (int64_t)rows[node_offsets[k+1]]-rows[node_offsets[k]];
	gmres_.SetSegments(entries, blocks);
	if (amg_) {
		std::vector<int32_t> node_segment((size_t)nodes());
		for (int k = 0; k < count; ++k)
			for (int64_t i = node_offsets[k]; i < node_offsets[k+1]; ++i) node_segment[i] = k;
		amg_->SetSegments(node_segment);
	}
	segment_entries_.Allocate(count+1);
	segment_entries_.Upload(entries.data(), count+1, stream_);
	segment_sq_.Allocate(count);
	segment_scale_.Allocate(2*(size_t)count);
	segment_scale_host_.assign(2*(size_t)count, 0.0);
	segment_initial_.assign(count, 0.0);
	segment_forcing_.assign(count, 0.0);
	segment_norm_.assign(count, 0.0);
	segment_done_host_.assign(count, 0);
	if (pinned_segments_) cudaFreeHost(pinned_segments_);
	pinned_segments_ = nullptr;
	CudaCheck(cudaMallocHost(reinterpret_cast<void**>(&pinned_segments_), sizeof(double)*count), "pinned segments");
	CudaCheck(cudaStreamSynchronize(stream_), "segments");
	segments_ = count;
}

void NsSolver::SegmentStatus(int32_t* done, double* residuals) const
{
	for (int k = 0; k < segments_; ++k) {
		if (done) done[k] = segment_done_host_[k];
		if (residuals) residuals[k] = segment_norm_[k];
	}
}

void NsSolver::DownloadValues(double* out)
{
	const size_t count = (size_t)blocks()*16;
	if (mixed()) {
		std::vector<float> tmp(count);
		values32_.Download(tmp.data(), count, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "download values");
		for (size_t i = 0; i < count; ++i) out[i] = tmp[i];
	} else {
		values_.Download(out, count, stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "download values");
	}
}

void NsSolver::SetLearned(LearnedPreconditioner* learned, bool use, bool collect)
{
	if (learned != nullptr && !amg_) Fail(-7, "the learned preconditioner stage needs the AMG-preconditioned FGMRES");
	learned_ = learned;
	collect_pairs_ = learned != nullptr && collect;
	gmres_.set_learned(learned != nullptr && use ? learned : nullptr);
	gmres_.set_collector(collect_pairs_ ? learned : nullptr);
	if (collect_pairs_ && pair_dinv_.size() == 0) {
		pair_dinv_.Allocate(n4_);
		pair_amg_.Allocate(n4_);
		pair_aamg_.Allocate(n4_);
		zero_flag_.Allocate(1);
		zero_flag_.Zero(stream_);
	}
}

void NsSolver::BindLearnedOperator(LearnedPreconditioner& learned)
{
	if (mixed()) learned.SetOperator(mesh_.pattern_view(), values32_.get(), nullptr);
	else learned.SetOperator(mesh_.pattern_view(), nullptr, values_.get());
}

void NsSolver::Synchronize()
{
	CudaCheck(cudaStreamSynchronize(stream_), "synchronize");
}

} // namespace tfiga
