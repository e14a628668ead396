// ref_shim.cpp -- C entry points around the reference's own header-only
// element code, compiled unmodified from the reference sources (see
// oracle/Makefile) into oracle/_ref/libtfiga_ref.so.  TEST INFRASTRUCTURE
// ONLY: it pins the C restatement in ns_oracle.c and serves as the reference
// CPU arm of the bench.  Nothing in the product links it.
//
// Wrapped reference routines:
//   iga::BuildNavierStokesElement      solvers/cpu/include/NavierStokesElement.hpp:390-397
//   iga::EvaluateBasis                 solvers/cpu/include/TransportElement.hpp:118-206
//   iga::IntegrateBoundaryFlow         solvers/cpu/include/BoundaryFlow.hpp:165-200
//   iga::IntegrateBoundaryPressureTraction solvers/cpu/include/BoundaryFlow.hpp:445-475
//   iga::EvaluateOutletModel           include/OutletModel.hpp:70-90
//   iga::Database::Load                solvers/cpu/include/IgaDatabase.hpp:124-161
//   iga::WallTraceBasis                solvers/cpu/include/BoundarySupport.hpp:134-150
//   iga::BuildTransportElement         solvers/cpu/include/TransportElement.hpp:213-260
//   iga::ParseCaseConfiguration        include/CaseConfig.hpp:340-371
//   iga::ReadTransportParameters       solvers/cpu/include/CaseInput.hpp:85-118
//   iga::WriteFlowCheckpointMetadata / ReadFlowCheckpointMetadata / ValidateFlowCheckpoint
//                                      include/FlowCheckpoint.hpp:176-211, with the raw state
//                                      file of solvers/cuda/src/iga_cuda.cu:566-602
//   iga::WriteVtu                      include/VtkOutput.hpp:107-155 (the arrays of
//                                      WriteNavierStokesVtu, solvers/cuda/src/iga_cuda.cu:366-388)
//   the flow boundary set-up of NavierStokes (solvers/cuda/src/iga_cuda.cu:766-790):
//   ReadSimulationConfiguration, FindNavierStokesSystem, InitializeOutletModels,
//   MaterializeBoundaryWaveforms, MaterializeOutletPressures, ExtractPressureTractions,
//   ResolveFlowBoundaries
//   iga::ResolveBoundaryConditions     solvers/cpu/include/CaseInput.hpp:162-258
//   iga::WomersleyAxialVelocity        solvers/cpu/include/WomersleyReference.hpp:150-189
#include "BoundaryFlow.hpp"
#include "BoundarySupport.hpp"
#include "FlowCheckpoint.hpp"
#include "GenericCaseInput.hpp"
#include "NavierStokesElement.hpp"
#include "OutletModel.hpp"
#include "PressureTraction.hpp"
#include "TemporalFunction.hpp"
#include "VtkOutput.hpp"
#include "WomersleyReference.hpp"

#include <omp.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <exception>
#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

namespace {

iga::Element MakeElement(const double* C, const double* X, int nen)
{
	iga::Element element;
	element.connectivity.resize(static_cast<std::size_t>(nen));
	element.extraction.resize(static_cast<std::size_t>(nen));
	for (int a = 0; a < nen; ++a) {
		element.connectivity[static_cast<std::size_t>(a)] = a;
		for (int p = 0; p < 64; ++p) element.extraction[static_cast<std::size_t>(a)][static_cast<std::size_t>(p)] = C[a*64+p];
	}
	for (int p = 0; p < 64; ++p)
		for (int d = 0; d < 3; ++d) element.bezier_points[static_cast<std::size_t>(p)][static_cast<std::size_t>(d)] = X[p*3+d];
	return element;
}

std::vector<std::array<double, 4>> Nodal(const double* values, int nen)
{
	std::vector<std::array<double, 4>> result(static_cast<std::size_t>(nen));
	for (int a = 0; a < nen; ++a)
		for (int f = 0; f < 4; ++f) result[static_cast<std::size_t>(a)][static_cast<std::size_t>(f)] = values ? values[a*4+f] : 0.0;
	return result;
}

thread_local std::string last_error;

} // namespace

extern "C" {

const char* ref_last_error() { return last_error.c_str(); }

// Element residual (-r) and exact tangent at the reference 4x4x4 rule.
// jac may be null (residual only).  Returns 0 or -1 on a reference exception.
int ref_ns_element(const double* C, const double* X, int nen, const double* state,
	const double* previous, double density, double viscosity, double dt, double* jac, double* negres)
{
	try {
		const auto element = MakeElement(C, X, nen);
		const auto nodal = Nodal(state, nen);
		const auto prev = dt > 0.0 ? Nodal(previous, nen) : std::vector<std::array<double, 4>>{};
		iga::FullCell4x4x4VolumeQuadratureProvider quadrature(element);
		const auto system = iga::BuildNavierStokesElement(element, nodal, prev,
			{density, viscosity, dt}, quadrature.Rule(),
			jac ? iga::NavierStokesAssemblyRequest::ResidualAndJacobian
				: iga::NavierStokesAssemblyRequest::ResidualOnly);
		if (jac) std::memcpy(jac, system.jacobian.data(), sizeof(double)*system.jacobian.size());
		std::memcpy(negres, system.negative_residual.data(), sizeof(double)*system.negative_residual.size());
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// Element residual with an explicit single-point rule (reference test form).
int ref_ns_element_points(const double* C, const double* X, int nen, const double* state,
	const double* previous, double density, double viscosity, double dt,
	const double* points, const double* weights, int count, double* jac, double* negres)
{
	try {
		const auto element = MakeElement(C, X, nen);
		std::vector<iga::VolumeQuadraturePoint> rule;
		for (int q = 0; q < count; ++q)
			rule.push_back({{points[3*q], points[3*q+1], points[3*q+2]}, weights[q]});
		const auto system = iga::BuildNavierStokesElement(element, Nodal(state, nen),
			dt > 0.0 ? Nodal(previous, nen) : std::vector<std::array<double, 4>>{},
			{density, viscosity, dt}, iga::VolumeQuadratureRule(rule));
		if (jac) std::memcpy(jac, system.jacobian.data(), sizeof(double)*system.jacobian.size());
		std::memcpy(negres, system.negative_residual.data(), sizeof(double)*system.negative_residual.size());
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

int ref_basis(const double* C, const double* X, int nen, double u, double v, double w,
	double* N, double* dN, double* H, double* inverse, double* raw_det)
{
	try {
		const auto basis = iga::EvaluateBasis(MakeElement(C, X, nen), u, v, w, true);
		for (int a = 0; a < nen; ++a) {
			N[a] = basis.value[static_cast<std::size_t>(a)];
			for (int i = 0; i < 3; ++i) {
				dN[a*3+i] = basis.gradient[static_cast<std::size_t>(a)][static_cast<std::size_t>(i)];
				for (int j = 0; j < 3; ++j)
					H[a*9+i*3+j] = basis.hessian[static_cast<std::size_t>(a)][static_cast<std::size_t>(i)][static_cast<std::size_t>(j)];
			}
		}
		for (int i = 0; i < 3; ++i)
			for (int j = 0; j < 3; ++j) inverse[i*3+j] = basis.inverse_jacobian[static_cast<std::size_t>(i)][static_cast<std::size_t>(j)];
		*raw_det = basis.raw_determinant;
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

double ref_boundary_flow(const double* C, const double* X, int nen, int face, const double* state)
{
	return iga::IntegrateBoundaryFlow(MakeElement(C, X, nen), static_cast<std::size_t>(face), Nodal(state, nen));
}

int ref_pressure_traction(const double* C, const double* X, int nen, int face, double pressure, double* out)
{
	try {
		const auto local = iga::IntegrateBoundaryPressureTraction(MakeElement(C, X, nen),
			static_cast<std::size_t>(face), pressure);
		std::memcpy(out, local.data(), sizeof(double)*local.size());
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

int ref_outlet_model(int kind, double resistance, double proximal, double distal, double capacitance,
	double reference_pressure, double capacitor_pressure, double flow, double dt,
	double* pressure, double* new_capacitor_pressure)
{
	try {
		iga::OutletModelState model;
		model.kind = kind == 0 ? iga::FieldBoundaryKind::Resistance
			: kind == 1 ? iga::FieldBoundaryKind::WindkesselRC : iga::FieldBoundaryKind::WindkesselRCR;
		model.resistance = resistance;
		model.proximal_resistance = proximal;
		model.distal_resistance = distal;
		model.capacitance = capacitance;
		model.reference_pressure = reference_pressure;
		model.capacitor_pressure = capacitor_pressure;
		const auto result = iga::EvaluateOutletModel(model, flow, dt);
		*pressure = result.pressure;
		*new_capacitor_pressure = result.capacitor_pressure;
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// Database header (version, ranks, elements, nodes) through iga::Database.
int ref_ntiga_header(const char* path, std::uint64_t* out)
{
	try {
		iga::Database database(path);
		const auto& h = database.header();
		out[0] = h.version; out[1] = h.ranks; out[2] = h.elements; out[3] = h.nodes;
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// One element through iga::Database::Load: nen, labels[6], connectivity,
// dense extraction [nen*64] and Bezier points [192].
int ref_ntiga_element(const char* path, std::uint64_t index, int* nen, int* labels,
	int* connectivity, double* extraction, double* bezier)
{
	try {
		iga::Database database(path);
		const auto element = database.Load(index);
		*nen = static_cast<int>(element.connectivity.size());
		for (int k = 0; k < 6; ++k) labels[k] = element.boundary_labels[static_cast<std::size_t>(k)];
		for (std::size_t a = 0; a < element.connectivity.size(); ++a) {
			connectivity[a] = element.connectivity[a];
			for (std::size_t p = 0; p < 64; ++p) extraction[a*64+p] = element.extraction[a][p];
		}
		for (std::size_t p = 0; p < 64; ++p)
			for (std::size_t d = 0; d < 3; ++d) bezier[p*3+d] = element.bezier_points[p][d];
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// Wall-trace no-slip basis set (iga_cuda.cu:748 -> BoundarySupport.hpp:134-150).
// Writes up to `capacity` node ids (sorted) and returns the count, or -1.
long long ref_wall_trace(const char* database_path, const char* vtk_path, int* out, long long capacity)
{
	try {
		iga::Database database(database_path);
		const auto mesh = iga::ReadLabeledHexMesh(vtk_path, database.header().nodes, database.header().elements);
		const auto nodes = iga::WallTraceBasis(database, mesh);
		long long count = 0;
		for (const auto node : nodes) {
			if (count < capacity) out[count] = node;
			++count;
		}
		return count;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// Global assembly with the reference's own element code: an OpenMP loop over
// elements [first, last) of a flattened mesh, each element built by
// iga::BuildNavierStokesElement (exact tangent, 4x4x4 rule) and added into
// 4x4 block CSR as OwnedRowAssembler::AddElementMatrix does
// (solvers/cpu/include/OwnedRowAssembler.hpp:210-236).  values may be null
// (residual only).  Returns 0 or -1.
int ref_assemble(int first, int last, const int* element_offsets, const int* connectivity,
	const int* extraction_offsets, const std::uint8_t* extraction_columns, const double* extraction_values,
	const double* bezier_points, const int* row_offsets, const int* columns, const double* state,
	const double* previous, double density, double viscosity, double dt, double* values, double* rhs)
{
	std::atomic<int> failed{0};
#pragma omp parallel for schedule(dynamic, 2)
	for (int e = first; e < last; ++e) {
		if (failed.load()) continue;
		try {
			const int begin = element_offsets[e];
			const int nen = element_offsets[e+1]-begin;
			iga::Element element;
			element.connectivity.resize(static_cast<std::size_t>(nen));
			element.extraction.assign(static_cast<std::size_t>(nen), std::array<double, 64>{});
			std::vector<std::array<double, 4>> nodal(static_cast<std::size_t>(nen)), prev(static_cast<std::size_t>(nen));
			for (int a = 0; a < nen; ++a) {
				const int node = connectivity[begin+a];
				element.connectivity[static_cast<std::size_t>(a)] = node;
				for (int k = extraction_offsets[begin+a]; k < extraction_offsets[begin+a+1]; ++k)
					element.extraction[static_cast<std::size_t>(a)][extraction_columns[k]] = extraction_values[k];
				for (int f = 0; f < 4; ++f) {
					nodal[static_cast<std::size_t>(a)][static_cast<std::size_t>(f)] = state[4*static_cast<std::size_t>(node)+f];
					prev[static_cast<std::size_t>(a)][static_cast<std::size_t>(f)] = previous[4*static_cast<std::size_t>(node)+f];
				}
			}
			for (int p = 0; p < 64; ++p)
				for (int d = 0; d < 3; ++d)
					element.bezier_points[static_cast<std::size_t>(p)][static_cast<std::size_t>(d)] = bezier_points[static_cast<std::size_t>(e)*192+p*3+d];
			iga::FullCell4x4x4VolumeQuadratureProvider quadrature(element);
			const auto system = iga::BuildNavierStokesElement(element, nodal,
				dt > 0.0 ? prev : std::vector<std::array<double, 4>>{}, {density, viscosity, dt}, quadrature.Rule(),
				values ? iga::NavierStokesAssemblyRequest::ResidualAndJacobian
					: iga::NavierStokesAssemblyRequest::ResidualOnly);
			const int ndof = 4*nen;
			for (int a = 0; a < nen; ++a) {
				const int row = element.connectivity[static_cast<std::size_t>(a)];
				for (int f = 0; f < 4; ++f) {
#pragma omp atomic
					rhs[4*static_cast<std::size_t>(row)+f] += system.negative_residual[static_cast<std::size_t>(4*a+f)];
				}
				if (!values) continue;
				for (int b = 0; b < nen; ++b) {
					const int column = element.connectivity[static_cast<std::size_t>(b)];
					const int* lo = columns+row_offsets[row];
					const int* hi = columns+row_offsets[row+1];
					const int* it = std::lower_bound(lo, hi, column);
					double* block = values+static_cast<std::size_t>(it-columns)*16;
					for (int i = 0; i < 4; ++i)
						for (int f = 0; f < 4; ++f) {
#pragma omp atomic
							block[i*4+f] += system.jacobian[static_cast<std::size_t>((4*a+i)*ndof+4*b+f)];
						}
				}
			}
		} catch (const std::exception& error) {
#pragma omp critical
			last_error = error.what();
			failed.store(1);
		}
	}
	return failed.load() ? -1 : 0;
}

int ref_max_threads() { return omp_get_max_threads(); }

// Boundary resolution of a legacy case: labels[nodes], reference velocity [3 nodes], the transport
// parameters it reads (vplus, N0bc, Nplusbc) and case_config.json text (NULL: absent).  Outputs
// [nodes] (velocity [3 nodes]); counts[3] = velocity, pressure, transport nodes.
int ref_resolve_boundaries(long long nodes, const int* labels, const double* velocity, double vplus, double n0_bc,
	double nplus_bc, const char* case_config, int* velocity_mask, int* pressure_mask, int* transport_mask,
	double* velocity_out, double* pressure, double* n0, double* nplus, long long* counts)
{
	try {
		std::vector<int> label(labels, labels+nodes);
		std::vector<std::array<double, 3>> reference(static_cast<std::size_t>(nodes));
		for (long long i = 0; i < nodes; ++i)
			for (int d = 0; d < 3; ++d) reference[static_cast<std::size_t>(i)][static_cast<std::size_t>(d)] = velocity[3*i+d];
		iga::TransportParameters parameters;
		parameters.vplus = vplus;
		parameters.n0_bc = n0_bc;
		parameters.nplus_bc = nplus_bc;
		const iga::CaseConfiguration configuration = case_config ? iga::ParseCaseConfiguration(case_config)
			: iga::CaseConfiguration{};
		const auto r = iga::ResolveBoundaryConditions(configuration, label, reference, parameters);
		for (long long i = 0; i < nodes; ++i) {
			const auto k = static_cast<std::size_t>(i);
			velocity_mask[i] = r.velocity_constrained[k];
			pressure_mask[i] = r.pressure_constrained[k];
			transport_mask[i] = r.transport_constrained[k];
			for (int d = 0; d < 3; ++d) velocity_out[3*i+d] = r.velocity[k][static_cast<std::size_t>(d)];
			pressure[i] = r.pressure[k];
			n0[i] = r.n0[k];
			nplus[i] = r.nplus[k];
		}
		counts[0] = static_cast<long long>(r.velocity_nodes);
		counts[1] = static_cast<long long>(r.pressure_nodes);
		counts[2] = static_cast<long long>(r.transport_nodes);
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// Flow boundary conditions of a simulation_config.json case at physical time t, outlet models at
// their initial state.  physics[5] = viscosity, density, dt, steps, transient; counts[2] = velocity,
// pressure nodes; tractions: labels / values up to *traction_count entries (in: capacity, out: count).
int ref_flow_boundaries(const char* config_path, const char* system, double time, long long nodes, const int* labels,
	const double* velocity, int* velocity_mask, double* velocity_out, int* pressure_mask, double* pressure,
	long long* counts, int* traction_labels, double* traction_values, int* traction_count, double* physics)
{
	try {
		const std::filesystem::path path(config_path);
		const auto configuration = iga::ReadSimulationConfiguration(path.string());
		const auto& flow = iga::FindNavierStokesSystem(configuration, system);
		const bool transient = flow.time_integration == "backward_euler";
		const auto models = iga::InitializeOutletModels(configuration, flow);
		const auto waveform = transient
			? iga::MaterializeBoundaryWaveforms(configuration, path.parent_path(), time) : configuration;
		const auto materialized = iga::MaterializeOutletPressures(waveform, models);
		const auto& resolved_system = iga::FindNavierStokesSystem(materialized, system);
		const auto tractions = iga::ExtractPressureTractions(materialized, resolved_system);
		std::vector<int> label(labels, labels+nodes);
		std::vector<std::array<double, 3>> reference(static_cast<std::size_t>(nodes));
		for (long long i = 0; i < nodes; ++i)
			for (int d = 0; d < 3; ++d) reference[static_cast<std::size_t>(i)][static_cast<std::size_t>(d)] = velocity[3*i+d];
		const auto r = iga::ResolveFlowBoundaries(materialized, resolved_system, label, reference);
		for (long long i = 0; i < nodes; ++i) {
			const auto k = static_cast<std::size_t>(i);
			velocity_mask[i] = r.velocity_constrained[k];
			pressure_mask[i] = r.pressure_constrained[k];
			for (int d = 0; d < 3; ++d) velocity_out[3*i+d] = r.velocity[k][static_cast<std::size_t>(d)];
			pressure[i] = r.pressure[k];
		}
		counts[0] = static_cast<long long>(r.velocity_nodes);
		counts[1] = static_cast<long long>(r.pressure_nodes);
		int n = 0;
		for (const auto& t : tractions) {
			if (n < *traction_count) { traction_labels[n] = t.first; traction_values[n] = t.second; }
			++n;
		}
		*traction_count = n;
		physics[0] = flow.viscosity;
		physics[1] = flow.density;
		physics[2] = transient ? configuration.time.dt : 0.0;
		physics[3] = transient ? configuration.time.steps : 1;
		physics[4] = transient ? 1.0 : 0.0;
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// Flow checkpoint as the CUDA command writes it: raw state + metadata.  outlets: count entries of
// (label, kind 0/1/2 = resistance / windkessel_rc / windkessel_rcr) and (flow, pressure, capacitor).
int ref_write_flow_checkpoint(const char* prefix, long long nodes, int completed, double time, double dt,
	double density, double viscosity, const int* outlet_ints, const double* outlet_values, int count,
	const double* state)
{
	try {
		static const char* kinds[3] = {"resistance", "windkessel_rc", "windkessel_rcr"};
		const auto state_path = iga::FlowCheckpointStatePath(prefix);
		std::ofstream output(state_path, std::ios::binary);
		output.write(reinterpret_cast<const char*>(state), static_cast<std::streamsize>(4*nodes*sizeof(double)));
		output.close();
		iga::FlowCheckpointMetadata metadata;
		metadata.nodes = static_cast<std::uint64_t>(nodes);
		metadata.completed_step = completed;
		metadata.physical_time = time;
		metadata.dt = dt;
		metadata.density = density;
		metadata.viscosity = viscosity;
		metadata.state_file = state_path.filename().string();
		metadata.state_format = "raw_float64";
		for (int i = 0; i < count; ++i)
			metadata.outlets.push_back({outlet_ints[2*i], kinds[outlet_ints[2*i+1]], outlet_values[3*i],
				outlet_values[3*i+1], outlet_values[3*i+2]});
		iga::WriteFlowCheckpointMetadata(prefix, metadata);
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// The reference's restart path: metadata, validation against (nodes, steps, dt, density, viscosity),
// and the raw state.  outlet_values[3*i]: flow, pressure, capacitor pressure of metadata outlet i.
int ref_read_flow_checkpoint(const char* prefix, long long nodes, int steps, double dt, double density,
	double viscosity, double* state, int* completed, double* time, int* outlet_labels, double* outlet_values,
	int* count)
{
	try {
		const auto metadata = iga::ReadFlowCheckpointMetadata(prefix);
		iga::ValidateFlowCheckpoint(metadata, static_cast<std::uint64_t>(nodes), steps, dt, density, viscosity);
		if (metadata.state_format != "raw_float64") throw std::runtime_error("not raw_float64");
		std::filesystem::path path(metadata.state_file);
		if (path.is_relative()) path = iga::FlowCheckpointMetadataPath(prefix).parent_path()/path;
		std::ifstream input(path, std::ios::binary);
		input.read(reinterpret_cast<char*>(state), static_cast<std::streamsize>(4*nodes*sizeof(double)));
		char extra = 0;
		if (!input || input.read(&extra, 1)) throw std::runtime_error("state is truncated or has trailing data");
		*completed = metadata.completed_step;
		*time = metadata.physical_time;
		const int n = std::min<int>(*count, static_cast<int>(metadata.outlets.size()));
		for (int i = 0; i < n; ++i) {
			outlet_labels[i] = metadata.outlets[static_cast<std::size_t>(i)].label;
			outlet_values[3*i] = metadata.outlets[static_cast<std::size_t>(i)].flow;
			outlet_values[3*i+1] = metadata.outlets[static_cast<std::size_t>(i)].pressure;
			outlet_values[3*i+2] = metadata.outlets[static_cast<std::size_t>(i)].capacitor_pressure;
		}
		*count = static_cast<int>(metadata.outlets.size());
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// VTU snapshot of a Navier-Stokes state [4 nodes] on the control mesh of mesh_vtk.
int ref_write_vtu(const char* mesh_vtk, const char* output, const double* state, long long nodes, double time)
{
	try {
		std::vector<double> velocity(static_cast<std::size_t>(3*nodes)), pressure(static_cast<std::size_t>(nodes));
		for (long long node = 0; node < nodes; ++node) {
			for (int c = 0; c < 3; ++c) velocity[static_cast<std::size_t>(3*node+c)] = state[4*node+c];
			pressure[static_cast<std::size_t>(node)] = state[4*node+3];
		}
		std::vector<iga::VtkPointArray> arrays{{"velocity", 3, std::move(velocity)}, {"pressure", 1, std::move(pressure)}};
		iga::WriteVtu(mesh_vtk, output, arrays, time);
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// simulation_parameter.txt: out[13] = D, vplus, vminus, kplus, kminus, k'plus, k'minus, dt, nstep,
// N0bc, Nplusbc, Nminusbc, artificial_diffusion.
int ref_read_transport_parameters(const char* path, double* out)
{
	try {
		const auto p = iga::ReadTransportParameters(path);
		const double values[13] = {p.diffusion, p.vplus, p.vminus, p.kplus, p.kminus, p.detach_plus, p.detach_minus,
			p.dt, static_cast<double>(p.steps), p.n0_bc, p.nplus_bc, p.nminus_bc, p.artificial_diffusion};
		std::memcpy(out, values, sizeof(values));
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// Two-species transport element (left and previous matrices, dense (2 nen)^2).
// p: D, vplus, kplus, kminus, k'plus, dt, artificial_diffusion.
int ref_transport_element(const double* C, const double* X, int nen, const double* velocity,
	const double* p, double* left, double* previous)
{
	try {
		const auto element = MakeElement(C, X, nen);
		std::vector<std::array<double, 3>> nodal(static_cast<std::size_t>(nen));
		for (int a = 0; a < nen; ++a)
			for (int d = 0; d < 3; ++d) nodal[static_cast<std::size_t>(a)][static_cast<std::size_t>(d)] = velocity[a*3+d];
		iga::TransportParameters parameters;
		parameters.diffusion = p[0];
		parameters.vplus = p[1];
		parameters.kplus = p[2];
		parameters.kminus = p[3];
		parameters.detach_plus = p[4];
		parameters.dt = p[5];
		parameters.artificial_diffusion = p[6];
		const auto matrices = iga::BuildTransportElement(element, nodal, parameters);
		std::memcpy(left, matrices.left.data(), sizeof(double)*matrices.left.size());
		std::memcpy(previous, matrices.previous.data(), sizeof(double)*matrices.previous.size());
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

// Axial Womersley velocity at radial distance r and time t of a pipe of the given radius driven by
// the pressure gradient mean + sum_k cosine[k] cos((k+1) w t) + sine[k] sin((k+1) w t).
int ref_womersley_axial_velocity(double radius, double density, double viscosity, double period,
	double mean_gradient, const double* cosine, const double* sine, int harmonics, double r, double t,
	double* velocity)
{
	try {
		iga::WomersleyReferenceConfiguration configuration;
		configuration.radius = radius;
		configuration.density = density;
		configuration.dynamic_viscosity = viscosity;
		configuration.period = period;
		configuration.mean_pressure_gradient = mean_gradient;
		configuration.cosine_pressure_gradient.assign(cosine, cosine+harmonics);
		configuration.sine_pressure_gradient.assign(sine, sine+harmonics);
		*velocity = iga::WomersleyAxialVelocity(configuration, r, t);
		return 0;
	} catch (const std::exception& error) {
		last_error = error.what();
		return -1;
	}
}

} // extern "C"
