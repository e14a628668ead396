// extern "C" boundary: every entry point converts exceptions into a status
// code plus a thread-local message (tfiga_last_error).
#include "case_input.hpp"
#include "flow_lines.hpp"
#include "learned.hpp"
#include "mesh.hpp"
#include "ns.hpp"
#include "transport.hpp"

#include "../../include/tfiga.h"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <filesystem>
#include <cstring>
#include <fstream>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <vector>

struct tfiga_mesh {
	std::unique_ptr<tfiga::Mesh> mesh;
};

struct tfiga_learned;

struct tfiga_ns {
	tfiga_mesh* mesh = nullptr;
	std::unique_ptr<tfiga::NsSolver> solver;
	tfiga_learned* learned = nullptr;       // attached learned stage (not owned)
};

struct tfiga_transport {
	tfiga_mesh* mesh = nullptr;
	std::unique_ptr<tfiga::TransportSolver> solver;
	tfiga_transport_params params;
};

struct tfiga_learned {
	std::unique_ptr<tfiga::LearnedPreconditioner> net;
	tfiga_ns* owner = nullptr;              // the ns handle it was created on (its mesh and stream)
	tfiga_ns* attached = nullptr;
	int32_t loss = TFIGA_LEARNED_RESIDUAL_LOSS;
};

namespace {

thread_local std::string g_error;

template <class F>
int Guard(F&& body)
{
	try {
		body();
		return TFIGA_OK;
	} catch (const tfiga::Error& error) {
		g_error = error.what();
		return error.status;
	} catch (const std::bad_alloc&) {
		g_error = "host allocation failed";
		return TFIGA_E_MEMORY;
	} catch (const std::exception& error) {
		g_error = error.what();
		return TFIGA_E_INVALID;
	} catch (...) {
		g_error = "unknown error";
		return TFIGA_E_INVALID;
	}
}

void Require(bool condition, const char* message)
{
	if (!condition) tfiga::Fail(TFIGA_E_INVALID, message);
}

tfiga::HostMesh FromDesc(const tfiga_mesh_desc* d)
{
	Require(d && d->nodes > 0 && d->elements > 0, "mesh descriptor needs nodes and elements");
	Require(d->element_offsets && d->connectivity && d->extraction_offsets && d->extraction_columns
		&& d->extraction_values && d->bezier_points, "mesh descriptor has a null array");
	tfiga::HostMesh m;
	m.nodes = d->nodes;
	const int64_t E = d->elements;
	m.element_offsets.assign(d->element_offsets, d->element_offsets+E+1);
	Require(m.element_offsets[0] == 0, "element_offsets must start at 0");
	const int64_t entries = m.element_offsets[E];
	m.connectivity.assign(d->connectivity, d->connectivity+entries);
	m.extraction_offsets.assign(d->extraction_offsets, d->extraction_offsets+entries+1);
	const int64_t nnz = m.extraction_offsets[entries];
	m.extraction_columns.assign(d->extraction_columns, d->extraction_columns+nnz);
	m.extraction_values.assign(d->extraction_values, d->extraction_values+nnz);
	m.bezier_points.assign(d->bezier_points, d->bezier_points+E*192);
	if (d->boundary_labels) m.boundary_labels.assign(d->boundary_labels, d->boundary_labels+E*6);
	else m.boundary_labels.assign(E*6, -1);
	for (int64_t e = 0; e < E; ++e)
		m.max_basis = std::max<int32_t>(m.max_basis, m.element_offsets[e+1]-m.element_offsets[e]);
	return m;
}

} // namespace

namespace tfiga {
// Lets entry points outside this file (which do not go through Guard) set the message.
void RecordLastError(const char* message) { g_error = message; }
}

extern "C" {

size_t tfiga_last_error(char* buffer, size_t capacity)
{
	if (buffer && capacity) {
		const size_t n = std::min(capacity-1, g_error.size());
		std::memcpy(buffer, g_error.data(), n);
		buffer[n] = '\0';
	}
	return g_error.size();
}

const char* tfiga_version(void)
{
	return "tubularflowiga-b200 0.2 sm_100a (FP64; tcgen05 split-BF16 tangent)";
}

int tfiga_mesh_create(const tfiga_mesh_desc* desc, tfiga_mesh** out)
{
	return Guard([&] {
		Require(out != nullptr, "out is null");
		*out = nullptr;
		auto handle = std::make_unique<tfiga_mesh>();
		handle->mesh = std::make_unique<tfiga::Mesh>(FromDesc(desc));
		*out = handle.release();
	});
}

int tfiga_batch_mesh_create(const tfiga_mesh_desc* tubes, int32_t count, tfiga_mesh** out, int64_t* node_offsets,
	int64_t* element_offsets)
{
	return Guard([&] {
		Require(out != nullptr && tubes != nullptr && count > 0, "batch needs tubes and an out handle");
		*out = nullptr;
		tfiga::HostMesh all;
		int64_t nodes = 0, elements = 0;
		if (node_offsets) node_offsets[0] = 0;
		if (element_offsets) element_offsets[0] = 0;
		for (int32_t k = 0; k < count; ++k) {
			const tfiga::HostMesh m = FromDesc(tubes+k);
			const int32_t entry0 = all.element_offsets.back();
			const int32_t nnz0 = all.extraction_offsets.back();
			Require(nodes+m.nodes < INT32_MAX && (int64_t)entry0+(int64_t)m.connectivity.size() < INT32_MAX
				&& (int64_t)nnz0+(int64_t)m.extraction_values.size() < INT32_MAX, "batch exceeds 32-bit indices");
			for (int64_t e = 1; e <= m.elements(); ++e) all.element_offsets.push_back(entry0+m.element_offsets[e]);
			for (const int32_t node : m.connectivity) all.connectivity.push_back((int32_t)(node+nodes));
			for (size_t i = 1; i < m.extraction_offsets.size(); ++i)
				all.extraction_offsets.push_back(nnz0+m.extraction_offsets[i]);
			all.extraction_columns.insert(all.extraction_columns.end(), m.extraction_columns.begin(),
				m.extraction_columns.end());
			all.extraction_values.insert(all.extraction_values.end(), m.extraction_values.begin(),
				m.extraction_values.end());
			all.bezier_points.insert(all.bezier_points.end(), m.bezier_points.begin(), m.bezier_points.end());
			all.boundary_labels.insert(all.boundary_labels.end(), m.boundary_labels.begin(), m.boundary_labels.end());
			all.max_basis = std::max(all.max_basis, m.max_basis);
			nodes += m.nodes;
			elements += m.elements();
			if (node_offsets) node_offsets[k+1] = nodes;
			if (element_offsets) element_offsets[k+1] = elements;
		}
		all.nodes = nodes;
		auto handle = std::make_unique<tfiga_mesh>();
		handle->mesh = std::make_unique<tfiga::Mesh>(std::move(all));
		*out = handle.release();
	});
}

int tfiga_mesh_load_ntiga(const char* path, tfiga_mesh** out)
{
	return Guard([&] {
		Require(path && out, "null argument");
		*out = nullptr;
		auto handle = std::make_unique<tfiga_mesh>();
		handle->mesh = std::make_unique<tfiga::Mesh>(tfiga::ReadNtiga(path));
		*out = handle.release();
	});
}

int tfiga_mesh_destroy(tfiga_mesh* mesh)
{
	return Guard([&] { delete mesh; });
}

int tfiga_mesh_info_get(const tfiga_mesh* mesh, tfiga_mesh_info* info)
{
	return Guard([&] {
		Require(mesh && info, "null argument");
		const auto& m = *mesh->mesh;
		info->nodes = m.host().nodes;
		info->elements = m.host().elements();
		info->max_basis = m.host().max_basis;
		info->basis_entries = (int64_t)m.host().connectivity.size();
		info->extraction_nonzeros = (int64_t)m.host().extraction_values.size();
		info->block_nonzeros = (int64_t)m.pattern().columns.size();
		info->max_block_row = m.pattern().max_row;
		info->min_detj = m.min_detj();
		info->bad_samples = m.bad_samples();
		info->device_bytes = m.device_bytes();
	});
}

int tfiga_mesh_pattern(const tfiga_mesh* mesh, int32_t* row_offsets, int32_t* columns, int32_t* diagonal)
{
	return Guard([&] {
		Require(mesh != nullptr, "null mesh");
		const auto& p = mesh->mesh->pattern();
		if (row_offsets) std::memcpy(row_offsets, p.row_offsets.data(), p.row_offsets.size()*sizeof(int32_t));
		if (columns) std::memcpy(columns, p.columns.data(), p.columns.size()*sizeof(int32_t));
		if (diagonal) std::memcpy(diagonal, p.diagonal.data(), p.diagonal.size()*sizeof(int32_t));
	});
}

void tfiga_ns_default_params(tfiga_ns_params* p)
{
	if (!p) return;
	p->density = 1.0;
	p->viscosity = 0.1;
	p->dt = 0.0;
	p->max_newton = 12;
	p->nonlinear_rtol = 1e-5;
	p->nonlinear_atol = 1e-10;
	p->mass_rtol = 1e-3;
	p->gmres_restart = 200;
	p->gmres_max_iterations = 5000;
	p->gmres_rtol = 1e-8;
	p->preconditioner = TFIGA_PRECONDITIONER_BLOCK_JACOBI;
	p->precision = TFIGA_PRECISION_FP64;
	p->amg_coarse_nodes = 300;
	p->amg_coarse_period = 1;
	p->krylov_fp64_basis = 0;
	p->newton_forcing = 0;
	p->tangent_reuse_factor = 0.0;
	p->tangent_kernel = TFIGA_TANGENT_AUTO;
}

int tfiga_ns_create(tfiga_mesh* mesh, const tfiga_ns_params* params, tfiga_ns** out)
{
	return Guard([&] {
		Require(mesh && params && out, "null argument");
		*out = nullptr;
		auto handle = std::make_unique<tfiga_ns>();
		handle->mesh = mesh;
		handle->solver = std::make_unique<tfiga::NsSolver>(*mesh->mesh, *params);
		*out = handle.release();
	});
}

int tfiga_ns_destroy(tfiga_ns* ns)
{
	return Guard([&] {
		if (ns && ns->learned) {
			if (ns->learned->attached == ns) ns->learned->attached = nullptr;
			if (ns->learned->owner == ns) ns->learned->owner = nullptr;
		}
		delete ns;
	});
}

int tfiga_ns_set_dirichlet(tfiga_ns* ns, const int32_t* vmask, const int32_t* pmask, const double* velocity,
	const double* pressure)
{
	return Guard([&] {
		Require(ns && vmask && velocity, "null argument");
		std::vector<double> zeros;
		if (!pressure) { zeros.assign(ns->solver->nodes(), 0.0); pressure = zeros.data(); }
		ns->solver->SetDirichlet(vmask, pmask, velocity, pressure);
	});
}

int tfiga_ns_set_dirichlet_values(tfiga_ns* ns, const double* velocity, const double* pressure)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		ns->solver->SetDirichletValues(velocity, pressure);
	});
}

int tfiga_ns_set_tractions(tfiga_ns* ns, const int32_t* labels, const double* pressures, int32_t count)
{
	return Guard([&] {
		Require(ns && (count == 0 || (labels && pressures)), "null argument");
		ns->solver->SetTractions(labels, pressures, count);
	});
}

int tfiga_ns_set_state(tfiga_ns* ns, const double* state, const double* previous)
{
	return Guard([&] {
		Require(ns && state, "null argument");
		ns->solver->SetState(state, previous);
	});
}

int tfiga_ns_get_state(tfiga_ns* ns, double* state)
{
	return Guard([&] {
		Require(ns && state, "null argument");
		ns->solver->GetState(state);
	});
}

int tfiga_ns_commit_step(tfiga_ns* ns)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		ns->solver->CommitStep();
	});
}

int tfiga_ns_assemble(tfiga_ns* ns, double* values, double* rhs)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		auto& s = *ns->solver;
		s.Assemble();
		if (values) s.DownloadValues(values);
		if (rhs) tfiga::CudaCheck(cudaMemcpyAsync(rhs, s.rhs(), (size_t)s.nodes()*4*sizeof(double),
			cudaMemcpyDeviceToHost, s.stream()), "download rhs");
		s.Synchronize();
	});
}

int tfiga_ns_apply_dirichlet(tfiga_ns* ns, double* values, double* rhs)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		auto& s = *ns->solver;
		s.ApplyDirichlet();
		if (values) s.DownloadValues(values);
		if (rhs) tfiga::CudaCheck(cudaMemcpyAsync(rhs, s.rhs(), (size_t)s.nodes()*4*sizeof(double),
			cudaMemcpyDeviceToHost, s.stream()), "download rhs");
		s.Synchronize();
	});
}

int tfiga_ns_solve_linear(tfiga_ns* ns, double rtol, int32_t max_iterations, double* update, int32_t* iterations,
	double* residual)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		auto& s = *ns->solver;
		const auto result = s.SolveLinear(rtol, max_iterations);
		if (iterations) *iterations = result.iterations;
		if (residual) *residual = result.residual;
		if (update) {
			tfiga::CudaCheck(cudaMemcpyAsync(update, s.update(), (size_t)s.nodes()*4*sizeof(double),
				cudaMemcpyDeviceToHost, s.stream()), "download update");
			s.Synchronize();
		}
		if (!result.converged) tfiga::Fail(TFIGA_E_NOT_CONVERGED, "GMRES did not reach the requested tolerance");
	});
}

int tfiga_ns_newton_iteration(tfiga_ns* ns, double initial_residual, tfiga_newton_report* report)
{
	return Guard([&] {
		Require(ns && report, "null argument");
		*report = ns->solver->NewtonIteration(initial_residual);
	});
}

int tfiga_ns_step(tfiga_ns* ns, tfiga_step_report* report)
{
	return Guard([&] {
		Require(ns && report, "null argument");
		*report = ns->solver->Step();
	});
}

int tfiga_ns_step_outlets(tfiga_ns* ns, tfiga_outlet* outlets, int32_t count, double relaxation,
	int32_t max_iterations, tfiga_step_report* report, int32_t* outlet_iterations)
{
	return Guard([&] {
		Require(ns && report && count >= 0 && (count == 0 || outlets), "null argument");
		int iterations = 0;
		*report = ns->solver->StepOutlets(outlets, count, relaxation, max_iterations, &iterations);
		if (outlet_iterations) *outlet_iterations = iterations;
	});
}

int tfiga_ns_step_outlets_coupled(tfiga_ns* ns, tfiga_outlet* outlets, int32_t count, double relaxation,
	int32_t max_newton, tfiga_step_report* report, int32_t* pressure_updates)
{
	return Guard([&] {
		Require(ns && report && count >= 0 && (count == 0 || outlets), "null argument");
		int updates = 0;
		*report = ns->solver->StepOutletsCoupled(outlets, count, relaxation, max_newton, &updates);
		if (pressure_updates) *pressure_updates = updates;
	});
}

int tfiga_ns_set_segments(tfiga_ns* ns, const int64_t* node_offsets, int32_t count)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		ns->solver->SetSegments(node_offsets, count);
	});
}

int tfiga_ns_segment_status(tfiga_ns* ns, int32_t* done, double* residuals)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		ns->solver->SegmentStatus(done, residuals);
	});
}

int tfiga_ns_tangent_kernel(tfiga_ns* ns, int32_t* kernel, double* coefficients_ms, double* fused_ms)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		if (kernel) *kernel = ns->solver->tangent_kernel();
		if (coefficients_ms) *coefficients_ms = ns->solver->tune_ms(TFIGA_TANGENT_COEFFICIENTS);
		if (fused_ms) *fused_ms = ns->solver->tune_ms(TFIGA_TANGENT_FUSED);
	});
}

int tfiga_ns_tangent_element_ms(tfiga_ns* ns, double* element_ms)
{
	return Guard([&] {
		Require(ns && element_ms, "null argument");
		*element_ms = ns->solver->tune_ms(TFIGA_TANGENT_ELEMENT);
	});
}

int tfiga_ns_amg_info(tfiga_ns* ns, tfiga_amg_info* info)
{
	return Guard([&] {
		Require(ns && info, "null argument");
		*info = tfiga_amg_info{};
		const auto* amg = ns->solver->amg();
		if (!amg || !amg->built()) return;
		const auto nodes = amg->level_nodes();
		const auto blocks = amg->level_blocks();
		info->levels = (int32_t)std::min<size_t>(8, nodes.size());
		for (int l = 0; l < info->levels; ++l) { info->nodes[l] = nodes[l]; info->blocks[l] = blocks[l]; }
		info->transfer_blocks = amg->transfer_blocks();
	});
}

int tfiga_ns_boundary_flows(tfiga_ns* ns, const int32_t* labels, int32_t count, double* flows)
{
	return Guard([&] {
		Require(ns && (count == 0 || (labels && flows)), "null argument");
		ns->solver->BoundaryFlows(labels, count, flows);
	});
}

int tfiga_ns_spmv_device(tfiga_ns* ns, const double* x, double* y)
{
	return Guard([&] {
		Require(ns && x && y, "null argument");
		if (ns->solver->mixed())
			tfiga::LaunchSpmv(ns->solver->pattern(), ns->solver->values32(), x, y, ns->solver->stream());
		else
			tfiga::LaunchSpmv(ns->solver->pattern(), ns->solver->values(), x, y, ns->solver->stream());
		ns->solver->AddLaunches(1);
	});
}

int tfiga_ns_device_buffers(tfiga_ns* ns, double** values, double** state, double** rhs)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		if (values) *values = ns->solver->values();
		if (state) *state = ns->solver->state();
		if (rhs) *rhs = ns->solver->rhs();
	});
}

int64_t tfiga_ns_launch_count(const tfiga_ns* ns)
{
	return ns ? ns->solver->launches() : -1;
}

int tfiga_ns_synchronize(tfiga_ns* ns)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		ns->solver->Synchronize();
	});
}

int tfiga_ns_stream(tfiga_ns* ns, void** stream)
{
	return Guard([&] {
		Require(ns && stream, "null argument");
		*stream = (void*)ns->solver->stream();
	});
}

int tfiga_ns_set_profiling(tfiga_ns* ns, int enable)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		ns->solver->profiler().Enable(enable != 0);
	});
}

int tfiga_ns_profile(tfiga_ns* ns, double* milliseconds, int64_t* launches, int32_t reset)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		long long counts[tfiga::Profiler::kFamilies];
		ns->solver->profiler().Totals(milliseconds, counts, reset != 0);
		if (launches) for (int f = 0; f < tfiga::Profiler::kFamilies; ++f) launches[f] = counts[f];
	});
}

void tfiga_transport_default_params(tfiga_transport_params* params)
{
	if (!params) return;
	std::memset(params, 0, sizeof(*params));
	params->restart = 50;
	params->gmres_rtol = 1e-8;
	params->gmres_max_iterations = 10000;
}

int tfiga_transport_read_params(const char* path, tfiga_transport_params* params)
{
	return Guard([&] {
		Require(path && params, "null argument");
		const tfiga::TransportParameters p = tfiga::ReadTransportParameters(path);
		params->diffusion = p.diffusion;
		params->vplus = p.vplus;
		params->vminus = p.vminus;
		params->kplus = p.kplus;
		params->kminus = p.kminus;
		params->detach_plus = p.detach_plus;
		params->detach_minus = p.detach_minus;
		params->dt = p.dt;
		params->steps = p.steps;
		params->n0_bc = p.n0_bc;
		params->nplus_bc = p.nplus_bc;
		params->nminus_bc = p.nminus_bc;
		params->artificial_diffusion = p.artificial_diffusion;
	});
}

int tfiga_resolve_flow_boundaries(const char* config_path, const char* system, double time, int64_t nodes,
	const int32_t* labels, const double* reference_velocity, int32_t* velocity_mask, double* velocity,
	int32_t* pressure_mask, double* pressure, int64_t* counts, int32_t* traction_labels, double* traction_values,
	int32_t* traction_count, double* physics)
{
	return Guard([&] {
		Require(config_path && nodes > 0 && labels && reference_velocity, "null argument");
		const std::string name = system ? system : "";
		const tfiga::SimulationConfig config = tfiga::ReadSimulationConfig(config_path);
		const tfiga::FlowSystem& flow = tfiga::FindNavierStokesSystem(config, name);
		const bool transient = flow.time_integration == "backward_euler";
		const auto models = tfiga::InitializeOutletModels(config, flow);
		const tfiga::SimulationConfig materialized = tfiga::MaterializeOutletPressures(
			transient ? tfiga::MaterializeWaveforms(config,
				std::filesystem::path(config_path).parent_path().string(), time) : config, models);
		const tfiga::FlowSystem& resolved_system = tfiga::FindNavierStokesSystem(materialized, name);
		const auto tractions = tfiga::ExtractPressureTractions(materialized, resolved_system);
		std::vector<int> label(labels, labels+nodes);
		std::vector<std::array<double, 3>> reference((size_t)nodes);
		for (int64_t i = 0; i < nodes; ++i)
			for (int d = 0; d < 3; ++d) reference[(size_t)i][d] = reference_velocity[3*i+d];
		const auto r = tfiga::ResolveFlowBoundaries(materialized, resolved_system, label, reference);
		if (velocity_mask) std::copy(r.velocity_mask.begin(), r.velocity_mask.end(), velocity_mask);
		if (velocity) std::copy(r.velocity.begin(), r.velocity.end(), velocity);
		if (pressure_mask) std::copy(r.pressure_mask.begin(), r.pressure_mask.end(), pressure_mask);
		if (pressure) std::copy(r.pressure.begin(), r.pressure.end(), pressure);
		if (counts) { counts[0] = (int64_t)r.velocity_nodes; counts[1] = (int64_t)r.pressure_nodes; }
		if (traction_count) {
			int32_t n = 0;
			for (const auto& t : tractions) {
				if (n < *traction_count && traction_labels && traction_values) {
					traction_labels[n] = t.first;
					traction_values[n] = t.second;
				}
				++n;
			}
			*traction_count = n;
		}
		if (physics) {
			physics[0] = flow.viscosity;
			physics[1] = flow.density;
			physics[2] = transient ? config.dt : 0.0;
			physics[3] = transient ? config.steps : 1;
			physics[4] = transient ? 1.0 : 0.0;
		}
	});
}

int tfiga_resolve_legacy_boundaries(int64_t nodes, const int32_t* labels, const double* reference_velocity,
	const tfiga_transport_params* params, const char* case_config_path, int32_t* velocity_mask, double* velocity,
	int32_t* pressure_mask, double* pressure, int32_t* transport_mask, double* n0, double* nplus, int64_t* counts)
{
	return Guard([&] {
		Require(nodes > 0 && labels && reference_velocity && params, "null argument");
		tfiga::TransportParameters p;
		p.vplus = params->vplus;
		p.n0_bc = params->n0_bc;
		p.nplus_bc = params->nplus_bc;
		std::vector<int> label(labels, labels+nodes);
		std::vector<std::array<double, 3>> reference((size_t)nodes);
		for (int64_t i = 0; i < nodes; ++i)
			for (int d = 0; d < 3; ++d) reference[(size_t)i][d] = reference_velocity[3*i+d];
		const tfiga::CaseConfiguration configuration = case_config_path
			? tfiga::ReadCaseConfiguration(case_config_path) : tfiga::CaseConfiguration{};
		const auto r = tfiga::ResolveLegacyBoundaries(configuration, label, reference, p);
		if (velocity_mask) std::copy(r.velocity_mask.begin(), r.velocity_mask.end(), velocity_mask);
		if (velocity) std::copy(r.velocity.begin(), r.velocity.end(), velocity);
		if (pressure_mask) std::copy(r.pressure_mask.begin(), r.pressure_mask.end(), pressure_mask);
		if (pressure) std::copy(r.pressure.begin(), r.pressure.end(), pressure);
		if (transport_mask) std::copy(r.transport_mask.begin(), r.transport_mask.end(), transport_mask);
		if (n0) std::copy(r.n0.begin(), r.n0.end(), n0);
		if (nplus) std::copy(r.nplus.begin(), r.nplus.end(), nplus);
		if (counts) {
			counts[0] = (int64_t)r.velocity_nodes;
			counts[1] = (int64_t)r.pressure_nodes;
			counts[2] = (int64_t)r.transport_nodes;
		}
	});
}

int tfiga_transport_resolve_boundaries(int64_t nodes, const int32_t* labels, const double* reference_velocity,
	const tfiga_transport_params* params, const char* case_config_path, int32_t* constrained, double* n0,
	double* nplus, int64_t* transport_nodes)
{
	int64_t counts[3] = {0, 0, 0};
	const int status = tfiga_resolve_legacy_boundaries(nodes, labels, reference_velocity, params, case_config_path,
		nullptr, nullptr, nullptr, nullptr, constrained, n0, nplus, counts);
	if (status == TFIGA_OK && transport_nodes) *transport_nodes = counts[2];
	return status;
}

int tfiga_transport_flow_lines(int64_t nodes, const int32_t* row_offsets, const int32_t* columns,
	const double* values, int32_t* line_offsets, int32_t* line_nodes, int32_t* band_width, int64_t* band_offsets,
	double* factors, int32_t* lines, int64_t* factor_count)
{
	return Guard([&] {
		Require(nodes > 0 && nodes < INT32_MAX && row_offsets && columns && values, "null argument");
		const tfiga::FlowLineFactors f = tfiga::BuildFlowLines((int32_t)nodes, row_offsets, columns, values);
		if (lines) *lines = f.lines();
		if (factor_count) *factor_count = (int64_t)f.factors.size();
		if (line_offsets) std::copy(f.line_offsets.begin(), f.line_offsets.end(), line_offsets);
		if (line_nodes) std::copy(f.line_nodes.begin(), f.line_nodes.end(), line_nodes);
		if (band_width) std::copy(f.band_width.begin(), f.band_width.end(), band_width);
		if (band_offsets) std::copy(f.band_offsets.begin(), f.band_offsets.end(), band_offsets);
		if (factors) std::copy(f.factors.begin(), f.factors.end(), factors);
	});
}

int tfiga_transport_create(tfiga_mesh* mesh, const tfiga_transport_params* params, const double* velocity,
	const int32_t* constrained, const double* n0, const double* nplus, tfiga_transport** out)
{
	return Guard([&] {
		Require(mesh && params && out, "null argument");
		*out = nullptr;
		Require(params->restart > 0, "restart must be positive");
		Require(params->gmres_rtol > 0.0 && params->gmres_max_iterations > 0, "GMRES tolerance and limit must be positive");
		Require(params->precision == TFIGA_PRECISION_FP64 || params->precision == TFIGA_PRECISION_MIXED,
			"transport precision must be TFIGA_PRECISION_FP64 or TFIGA_PRECISION_MIXED");
		Require(params->preconditioner == TFIGA_TRANSPORT_BLOCK_JACOBI
			|| params->preconditioner == TFIGA_TRANSPORT_FLOW_LINES, "unknown transport preconditioner");
		tfiga::RequireDevice();
		const tfiga::TransportCoefficients c{params->diffusion, params->vplus, params->kplus, params->kminus,
			params->detach_plus, params->dt, params->artificial_diffusion};
		auto handle = std::make_unique<tfiga_transport>();
		handle->mesh = mesh;
		handle->params = *params;
		handle->solver = std::make_unique<tfiga::TransportSolver>(*mesh->mesh, c, velocity, constrained, n0, nplus,
			params->restart, params->precision == TFIGA_PRECISION_MIXED,
			params->preconditioner == TFIGA_TRANSPORT_FLOW_LINES);
		*out = handle.release();
	});
}

int tfiga_transport_destroy(tfiga_transport* transport)
{
	return Guard([&] { delete transport; });
}

int tfiga_transport_step(tfiga_transport* transport, int32_t steps, tfiga_transport_report* report)
{
	return Guard([&] {
		Require(transport != nullptr, "null handle");
		Require(steps >= 0, "steps must be non-negative");
		tfiga_transport_report r;
		std::memset(&r, 0, sizeof(r));
		for (int32_t k = 0; k < steps; ++k) {
			const auto step = transport->solver->Step(transport->params.gmres_rtol,
				transport->params.gmres_max_iterations);
			r.steps += 1;
			r.last_iterations = step.iterations;
			r.total_iterations += step.iterations;
			r.last_residual = step.residual;
			r.singular_blocks = std::max(r.singular_blocks, step.singular_blocks);
		}
		if (report) {
			r.final_l2 = transport->solver->StateNorm();
			*report = r;
		}
	});
}

int tfiga_transport_set_state(tfiga_transport* transport, const double* state)
{
	return Guard([&] {
		Require(transport && state, "null argument");
		transport->solver->SetState(state);
	});
}

int tfiga_transport_get_state(tfiga_transport* transport, double* state)
{
	return Guard([&] {
		Require(transport && state, "null argument");
		transport->solver->GetState(state);
	});
}

int tfiga_transport_matrices(tfiga_transport* transport, double* left, double* previous)
{
	return Guard([&] {
		Require(transport != nullptr, "null handle");
		transport->solver->Matrices(left, previous);
	});
}

int tfiga_transport_apply_preconditioner(tfiga_transport* transport, const double* x, double* y)
{
	return Guard([&] {
		Require(transport && x && y, "null argument");
		transport->solver->ApplyLinePreconditioner(x, y);
	});
}

int tfiga_transport_info(const tfiga_transport* transport, double* assembly_ms, int32_t* steps, int64_t* launches)
{
	return Guard([&] {
		Require(transport != nullptr, "null handle");
		if (assembly_ms) *assembly_ms = transport->solver->assembly_ms();
		if (steps) *steps = transport->solver->steps();
		if (launches) *launches = transport->solver->launches();
	});
}

int tfiga_transport_stream(tfiga_transport* transport, void** stream)
{
	return Guard([&] {
		Require(transport && stream, "null argument");
		*stream = (void*)transport->solver->stream();
	});
}

int tfiga_transport_set_profiling(tfiga_transport* transport, int enable)
{
	return Guard([&] {
		Require(transport != nullptr, "null handle");
		transport->solver->profiler().Enable(enable != 0);
	});
}

int tfiga_transport_profile(tfiga_transport* transport, double* milliseconds, int64_t* launches, int32_t reset)
{
	return Guard([&] {
		Require(transport != nullptr, "null handle");
		long long counts[tfiga::Profiler::kFamilies];
		transport->solver->profiler().Totals(milliseconds, counts, reset != 0);
		if (launches) for (int f = 0; f < tfiga::Profiler::kFamilies; ++f) launches[f] = counts[f];
	});
}

int tfiga_learned_create(tfiga_ns* ns, int32_t layers, uint64_t seed, int32_t linear, tfiga_learned** out)
{
	return Guard([&] {
		Require(ns && out, "null argument");
		*out = nullptr;
		if (!ns->solver->amg()) tfiga::Fail(TFIGA_E_UNSUPPORTED, "the learned stage needs TFIGA_PRECONDITIONER_AMG");
		auto handle = std::make_unique<tfiga_learned>();
		handle->net = std::make_unique<tfiga::LearnedPreconditioner>(*ns->mesh->mesh, layers, seed,
			ns->solver->stream(), linear != 0);
		handle->owner = ns;
		*out = handle.release();
	});
}

int tfiga_learned_destroy(tfiga_learned* learned)
{
	return Guard([&] {
		if (!learned) return;
		if (learned->attached) {
			learned->attached->solver->SetLearned(nullptr, false, false);
			learned->attached->learned = nullptr;
		}
		delete learned;
	});
}

int tfiga_learned_info(const tfiga_learned* learned, int64_t* parameters, int64_t* elements, int32_t* pairs)
{
	return Guard([&] {
		Require(learned != nullptr, "null handle");
		if (parameters) *parameters = learned->net->parameter_count();
		if (elements) *elements = learned->net->elements();
		if (pairs) *pairs = learned->net->pair_count();
	});
}

int tfiga_ns_set_learned(tfiga_ns* ns, tfiga_learned* learned, int32_t use, int32_t collect)
{
	return Guard([&] {
		Require(ns != nullptr, "null handle");
		if (learned && learned->owner != ns)
			tfiga::Fail(TFIGA_E_INVALID, "the learned stage belongs to another solver handle");
		ns->solver->SetLearned(learned ? learned->net.get() : nullptr, use != 0, collect != 0);
		if (ns->learned && ns->learned != learned) ns->learned->attached = nullptr;
		ns->learned = learned;
		if (learned) learned->attached = ns;
	});
}

int tfiga_ns_learned_fallbacks(const tfiga_ns* ns, int64_t* count)
{
	return Guard([&] {
		Require(ns && count, "null argument");
		*count = ns->solver->learned_fallbacks();
	});
}

namespace {

// The residual loss trains through the owner's current Jacobian; the error loss through none.
void BindLoss(tfiga_learned* learned)
{
	if (learned->loss == TFIGA_LEARNED_ERROR_LOSS) learned->net->SetOperator({}, nullptr, nullptr);
	else if (learned->owner) learned->owner->solver->BindLearnedOperator(*learned->net);
}

} // namespace

int tfiga_learned_set_loss(tfiga_learned* learned, int32_t loss)
{
	return Guard([&] {
		Require(learned != nullptr, "null handle");
		Require(loss == TFIGA_LEARNED_RESIDUAL_LOSS || loss == TFIGA_LEARNED_ERROR_LOSS, "unknown learned loss");
		learned->loss = loss;
	});
}

int tfiga_learned_set_capacity(tfiga_learned* learned, int32_t capacity)
{
	return Guard([&] {
		Require(learned != nullptr && capacity > 0, "invalid argument");
		learned->net->SetCapacity(capacity);
	});
}

int tfiga_learned_fit_scales(tfiga_learned* learned)
{
	return Guard([&] { Require(learned != nullptr, "null handle"); BindLoss(learned);
		learned->net->FitScales(); });
}

int tfiga_learned_train(tfiga_learned* learned, int32_t steps, double learning_rate, double* loss)
{
	return Guard([&] {
		Require(learned != nullptr && steps >= 0, "invalid argument");
		Require(learning_rate > 0.0 && std::isfinite(learning_rate), "learning rate must be positive");
		BindLoss(learned);
		const double l = learned->net->Train(steps, learning_rate);
		if (loss) *loss = l;
	});
}

int tfiga_learned_evaluate(tfiga_learned* learned, double* loss)
{
	return Guard([&] {
		Require(learned && loss, "null argument");
		BindLoss(learned);
		*loss = learned->net->EvaluatePairs();
	});
}

int tfiga_learned_fit_gain(tfiga_learned* learned, double* gain)
{
	return Guard([&] {
		Require(learned != nullptr, "null handle");
		BindLoss(learned);
		const double g = learned->net->FitGain();
		if (gain) *gain = g;
	});
}

int tfiga_learned_get_parameters(const tfiga_learned* learned, float* parameters)
{
	return Guard([&] { Require(learned && parameters, "null argument"); learned->net->GetParameters(parameters); });
}

int tfiga_learned_set_parameters(tfiga_learned* learned, const float* parameters)
{
	return Guard([&] { Require(learned && parameters, "null argument"); learned->net->SetParameters(parameters); });
}

int tfiga_learned_get_scales(const tfiga_learned* learned, double* scales)
{
	return Guard([&] {
		Require(learned && scales, "null argument");
		learned->net->GetScales(scales, scales+4, scales+8);
	});
}

int tfiga_learned_set_scales(tfiga_learned* learned, const double* scales)
{
	return Guard([&] {
		Require(learned && scales, "null argument");
		learned->net->SetScales(scales, scales+4, scales+8);
	});
}

int tfiga_learned_neighbours(const tfiga_learned* learned, int32_t* neighbours)
{
	return Guard([&] {
		Require(learned && neighbours, "null argument");
		const auto& nb = learned->net->neighbours();
		std::memcpy(neighbours, nb.data(), nb.size()*sizeof(int32_t));
	});
}

int tfiga_learned_forward_device(tfiga_learned* learned, const double* x_device, double* o_device)
{
	return Guard([&] {
		Require(learned && x_device && o_device, "null argument");
		learned->net->Forward(x_device, o_device);
		tfiga::CudaCheck(cudaStreamSynchronize(learned->net->stream()), "learned forward");
	});
}

int tfiga_learned_apply_device(tfiga_learned* learned, const double* x_device, double* z_device)
{
	return Guard([&] {
		Require(learned && x_device && z_device, "null argument");
		learned->net->Apply(x_device, z_device, nullptr);
		tfiga::CudaCheck(cudaStreamSynchronize(learned->net->stream()), "learned apply");
	});
}

int tfiga_learned_loss_gradient_device(tfiga_learned* learned, const double* x_device, const double* target_device,
	double* loss, float* gradient)
{
	return Guard([&] {
		Require(learned && x_device && target_device, "null argument");
		const double l = learned->net->LossAndGradient(x_device, target_device);
		if (loss) *loss = l;
		if (gradient) {
			tfiga::CudaCheck(cudaMemcpyAsync(gradient, learned->net->gradient(),
				sizeof(float)*(size_t)learned->net->parameter_count(), cudaMemcpyDeviceToHost, learned->net->stream()),
				"learned gradient");
			tfiga::CudaCheck(cudaStreamSynchronize(learned->net->stream()), "learned gradient");
		}
	});
}

namespace {
const char kLearnedMagic[8] = {'T', 'F', 'L', 'R', 'N', '0', '0', '1'};
}

int tfiga_learned_save(const tfiga_learned* learned, const char* path)
{
	return Guard([&] {
		Require(learned && path, "null argument");
		const auto& net = *learned->net;
		std::vector<float> theta(net.parameter_count());
		net.GetParameters(theta.data());
		double scales[12];
		net.GetScales(scales, scales+4, scales+8);
		std::ofstream f(path, std::ios::binary);
		if (!f) tfiga::Fail(TFIGA_E_IO, std::string("cannot write ")+path);
		const int32_t layers = net.layers();
		const int64_t count = net.parameter_count();
		f.write(kLearnedMagic, 8);
		f.write(reinterpret_cast<const char*>(&layers), sizeof(layers));
		f.write(reinterpret_cast<const char*>(&count), sizeof(count));
		f.write(reinterpret_cast<const char*>(theta.data()), sizeof(float)*theta.size());
		f.write(reinterpret_cast<const char*>(scales), sizeof(scales));
		if (!f) tfiga::Fail(TFIGA_E_IO, std::string("write failed: ")+path);
	});
}

int tfiga_learned_load(tfiga_learned* learned, const char* path)
{
	return Guard([&] {
		Require(learned && path, "null argument");
		auto& net = *learned->net;
		std::ifstream f(path, std::ios::binary);
		if (!f) tfiga::Fail(TFIGA_E_IO, std::string("cannot read ")+path);
		char magic[8];
		int32_t layers = 0;
		int64_t count = 0;
		f.read(magic, 8);
		f.read(reinterpret_cast<char*>(&layers), sizeof(layers));
		f.read(reinterpret_cast<char*>(&count), sizeof(count));
		if (!f || std::memcmp(magic, kLearnedMagic, 8) != 0) tfiga::Fail(TFIGA_E_FORMAT, "not a learned-stage file");
		if (layers != net.layers() || count != net.parameter_count())
			tfiga::Fail(TFIGA_E_FORMAT, "learned-stage file has a different architecture");
		std::vector<float> theta(count);
		double scales[12];
		f.read(reinterpret_cast<char*>(theta.data()), sizeof(float)*theta.size());
		f.read(reinterpret_cast<char*>(scales), sizeof(scales));
		if (!f) tfiga::Fail(TFIGA_E_FORMAT, "truncated learned-stage file");
		net.SetParameters(theta.data());
		net.SetScales(scales, scales+4, scales+8);
	});
}

int tfiga_ns_profile_bytes(tfiga_ns* ns, double* bytes)
{
	return Guard([&] {
		Require(ns && bytes, "null argument");
		ns->solver->profiler().Totals(nullptr, nullptr, false, bytes, bytes+tfiga::Profiler::kFamilies);
	});
}

} // extern "C"
