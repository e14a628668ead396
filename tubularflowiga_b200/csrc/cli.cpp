// The drop-in command (tfiga_main): device-info, mesh-check, navier-stokes and
// transport with the reference's arguments, log lines, outputs and exit codes
// (solvers/cuda/src/iga_cuda.cu:278-303, 327-400, 389-498, 566-1195).
#include "case_input.hpp"
#include "json.hpp"
#include "mesh.hpp"
#include "ns.hpp"
#include "transport.hpp"

#include "../../include/tfiga.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <exception>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>

namespace fs = std::filesystem;

namespace tfiga {
namespace {

using Clock = std::chrono::steady_clock;

void PrintDevice()
{
	int device = 0;
	CudaCheck(cudaGetDevice(&device), "cudaGetDevice");
	cudaDeviceProp prop{};
	CudaCheck(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
	size_t free_bytes = 0, total = 0;
	CudaCheck(cudaMemGetInfo(&free_bytes, &total), "cudaMemGetInfo");
	int runtime = 0, driver = 0;
	cudaRuntimeGetVersion(&runtime);
	cudaDriverGetVersion(&driver);
	std::cout << "device=" << device << " name=\"" << prop.name << "\" compute_capability=" << prop.major << '.'
		<< prop.minor << " sms=" << prop.multiProcessorCount
		<< " memory_free_gib=" << free_bytes/1073741824.0 << " memory_total_gib=" << total/1073741824.0 << '\n';
	std::cout << "cuda_capabilities runtime_build=" << CUDART_VERSION << " runtime_linked=" << runtime
		<< " driver=" << driver << " arch=sm_100a precision=fp64\n";
}

void PrintMesh(const Mesh& mesh)
{
	const auto& h = mesh.host();
	std::cout << "mesh nodes=" << h.nodes << " elements=" << h.elements() << " basis_entries=" << h.connectivity.size()
		<< " extraction_nonzeros=" << h.extraction_values.size() << " max_basis=" << h.max_basis
		<< " block_nonzeros=" << mesh.pattern().columns.size()
		<< " mean_block_row=" << (double)mesh.pattern().columns.size()/h.nodes << '\n';
}

int MeshCheck(const std::string& path)
{
	Mesh mesh(ReadNtiga(path));
	PrintMesh(mesh);
	std::cout << "geometry min_detJ=" << std::setprecision(17) << mesh.min_detj() << " bad_samples="
		<< mesh.bad_samples() << " device_mesh_gib=" << mesh.device_bytes()/1073741824.0 << '\n';
	return mesh.bad_samples() ? 1 : 0;
}

struct Options {
	std::string database, case_dir, system;
	int max_newton = 12;
	double rtol = 1e-5, atol = 1e-10, mass_rtol = 1e-3;
	std::string output, checkpoint, restart;
	int output_every = 0, checkpoint_every = 0, stop_after_step = 0;
	std::string visualization = "auto";
};

int PositiveInt(const std::string& text, const std::string& option)
{
	size_t used = 0;
	int v = 0;
	try { v = std::stoi(text, &used); } catch (const std::exception&) { Fail(-1, option+" requires a positive integer"); }
	if (used != text.size() || v <= 0) Fail(-1, option+" requires a positive integer");
	return v;
}

double PositiveDouble(const std::string& text, const std::string& option)
{
	size_t used = 0;
	double v = 0.0;
	try { v = std::stod(text, &used); } catch (const std::exception&) { Fail(-1, option+" requires a finite positive value"); }
	if (used != text.size() || !std::isfinite(v) || v <= 0.0) Fail(-1, option+" requires a finite positive value");
	return v;
}

// ParseCudaFlowOptions (iga_cuda.cu:447-498).
Options ParseOptions(int argc, char** argv)
{
	if (argc < 4) Fail(-1, "usage: iga_cuda navier-stokes DATABASE.ntiga CASE_DIR [MAX_NEWTON] [OUTPUT] "
		"[--system NAME] [--max-newton N] [--output PATH] [--output-every N] [--checkpoint PREFIX] "
		"[--checkpoint-every N] [--restart PREFIX] [--stop-after-step N] [--nonlinear-rtol R] "
		"[--nonlinear-atol A] [--mass-rtol R] [--visualization-format auto|vtu|vtkhdf]");
	Options o;
	o.database = argv[2];
	o.case_dir = argv[3];
	int positional = 0;
	for (int i = 4; i < argc; ++i) {
		const std::string arg(argv[i]);
		if (arg.rfind("--", 0) != 0) {
			if (positional == 0) o.max_newton = PositiveInt(arg, "MAX_NEWTON");
			else if (positional == 1) o.output = arg;
			else Fail(-1, "too many positional arguments");
			++positional;
			continue;
		}
		if (i+1 >= argc) Fail(-1, arg+" requires a value");
		const std::string v(argv[++i]);
		if (arg == "--system") o.system = v;
		else if (arg == "--max-newton") o.max_newton = PositiveInt(v, arg);
		else if (arg == "--output") o.output = v;
		else if (arg == "--output-every") o.output_every = PositiveInt(v, arg);
		else if (arg == "--checkpoint") o.checkpoint = v;
		else if (arg == "--checkpoint-every") o.checkpoint_every = PositiveInt(v, arg);
		else if (arg == "--restart") o.restart = v;
		else if (arg == "--stop-after-step") o.stop_after_step = PositiveInt(v, arg);
		else if (arg == "--nonlinear-rtol") o.rtol = PositiveDouble(v, arg);
		else if (arg == "--nonlinear-atol") o.atol = PositiveDouble(v, arg);
		else if (arg == "--mass-rtol") o.mass_rtol = PositiveDouble(v, arg);
		else if (arg == "--visualization-format") {
			// ParseVisualizationFormat (include/VtkOutput.hpp:17-25)
			if (v != "auto" && v != "vtu" && v != "vtkhdf" && v != "bezier-vtkhdf")
				Fail(-1, "--visualization-format must be auto, vtu, or vtkhdf");
			if (v == "vtkhdf" || v == "bezier-vtkhdf")
				Fail(-4, "--visualization-format vtkhdf needs HDF5, which this build does not include; use vtu");
			o.visualization = v;
		} else Fail(-1, "unknown option: "+arg);
	}
	if (o.output_every > 0 && o.output.empty()) Fail(-1, "--output-every requires --output or legacy OUTPUT");
	if (o.checkpoint_every > 0 && o.checkpoint.empty()) Fail(-1, "--checkpoint-every requires --checkpoint");
	return o;
}

std::string Precise(double v)
{
	std::ostringstream s;
	s << std::scientific << std::setprecision(16) << v;
	return s.str();
}

// TimeIndexedPath (include/FlowCheckpoint.hpp).
fs::path TimeIndexed(const fs::path& base, int step)
{
	std::ostringstream suffix;
	suffix << ".step" << std::setw(6) << std::setfill('0') << step;
	const auto ext = base.extension().string();
	if (ext.empty()) return base.string()+suffix.str();
	return base.parent_path()/(base.stem().string()+suffix.str()+ext);
}

// WriteNavierStokes (iga_cuda.cu:389-400): "u v w" rows and <out>.pressure rows.
void WriteText(const fs::path& path, const std::vector<double>& state)
{
	std::ofstream velocity(path), pressure(path.string()+".pressure");
	if (!velocity || !pressure) Fail(-3, "cannot create Navier-Stokes output");
	velocity << std::setprecision(17);
	pressure << std::setprecision(17);
	for (size_t node = 0; node < state.size()/4; ++node) {
		velocity << state[4*node] << ' ' << state[4*node+1] << ' ' << state[4*node+2] << '\n';
		pressure << state[4*node+3] << '\n';
	}
}

// WriteNavierStokesVtk (iga_cuda.cu:351-364): control mesh + velocity/pressure point data.
void WriteVtk(const fs::path& mesh_path, const fs::path& path, const std::vector<double>& state)
{
	std::ifstream mesh(mesh_path);
	std::ofstream out(path);
	if (!mesh) Fail(-3, "cannot open VTK mesh "+mesh_path.string());
	if (!out) Fail(-3, "cannot create "+path.string());
	out << mesh.rdbuf() << "\nVECTORS Velocity double\n" << std::setprecision(17);
	for (size_t node = 0; node < state.size()/4; ++node)
		out << state[4*node] << ' ' << state[4*node+1] << ' ' << state[4*node+2] << '\n';
	out << "SCALARS Pressure double 1\nLOOKUP_TABLE default\n";
	for (size_t node = 0; node < state.size()/4; ++node) out << state[4*node+3] << '\n';
}

// ASCII legacy unstructured grid of controlmesh.vtk (ReadLegacyUnstructuredGrid,
// include/VtkOutput.hpp:61-105): points, cell connectivity, offsets and types.
struct VtkGrid {
	std::vector<double> points;
	std::vector<int64_t> connectivity, offsets;
	std::vector<unsigned> types;
};

VtkGrid ReadVtkGrid(const fs::path& path)
{
	std::ifstream in(path);
	if (!in) Fail(-3, "cannot open VTK mesh: "+path.string());
	VtkGrid g;
	std::string token;
	size_t points = 0, cells = 0;
	while (in >> token) {
		if (token == "POINTS") {
			std::string type;
			in >> points >> type;
			g.points.resize(3*points);
			for (auto& v : g.points)
				if (!(in >> v)) Fail(-4, "truncated VTK points: "+path.string());
		} else if (token == "CELLS") {
			size_t entries = 0;
			in >> cells >> entries;
			for (size_t c = 0; c < cells; ++c) {
				size_t count = 0;
				if (!(in >> count)) Fail(-4, "truncated VTK cells: "+path.string());
				for (size_t k = 0; k < count; ++k) {
					int64_t index = -1;
					if (!(in >> index) || index < 0 || (size_t)index >= points)
						Fail(-4, "invalid VTK cell connectivity: "+path.string());
					g.connectivity.push_back(index);
				}
				g.offsets.push_back((int64_t)g.connectivity.size());
			}
		} else if (token == "CELL_TYPES") {
			size_t count = 0;
			in >> count;
			g.types.resize(count);
			for (auto& t : g.types)
				if (!(in >> t)) Fail(-4, "truncated VTK cell types: "+path.string());
			break;
		}
	}
	if (points == 0 || cells == 0 || g.offsets.size() != cells || g.types.size() != cells)
		Fail(-4, "VTK mesh is not a complete ASCII unstructured grid: "+path.string());
	return g;
}

// VTK XML unstructured grid with velocity (3) and pressure (1) point arrays and the
// physical time as TimeValue field data (WriteVtu, include/VtkOutput.hpp:107-155).
void WriteVtuFile(const VtkGrid& g, const fs::path& path, const std::vector<double>& state, double time)
{
	const size_t points = g.points.size()/3;
	if (state.size() != 4*points) Fail(-4, "VTU point-array size mismatch for 'velocity'");
	if (!path.parent_path().empty()) fs::create_directories(path.parent_path());
	std::ofstream out(path);
	if (!out) Fail(-3, "cannot create VTU output: "+path.string());
	out << std::setprecision(17) << "<?xml version=\"1.0\"?>\n"
		<< "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
		<< "  <UnstructuredGrid>\n"
		<< "    <FieldData><DataArray type=\"Float64\" Name=\"TimeValue\" NumberOfTuples=\"1\" format=\"ascii\">"
		<< time << "</DataArray></FieldData>\n"
		<< "    <Piece NumberOfPoints=\"" << points << "\" NumberOfCells=\"" << g.offsets.size() << "\">\n"
		<< "      <PointData>\n"
		<< "        <DataArray type=\"Float64\" Name=\"velocity\" NumberOfComponents=\"3\" format=\"ascii\">\n          ";
	for (size_t node = 0; node < points; ++node)
		out << state[4*node] << ' ' << state[4*node+1] << ' ' << state[4*node+2] << ' ';
	out << "\n        </DataArray>\n"
		<< "        <DataArray type=\"Float64\" Name=\"pressure\" NumberOfComponents=\"1\" format=\"ascii\">\n          ";
	for (size_t node = 0; node < points; ++node) out << state[4*node+3] << ' ';
	out << "\n        </DataArray>\n      </PointData>\n"
		<< "      <Points><DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n        ";
	for (double v : g.points) out << v << ' ';
	out << "\n      </DataArray></Points>\n      <Cells>\n"
		<< "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n          ";
	for (auto v : g.connectivity) out << v << ' ';
	out << "\n        </DataArray>\n        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n          ";
	for (auto v : g.offsets) out << v << ' ';
	out << "\n        </DataArray>\n        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n          ";
	for (auto v : g.types) out << v << ' ';
	out << "\n        </DataArray>\n      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n";
	out.close();
	if (!out) Fail(-3, "cannot write VTU output: "+path.string());
}

// <stem>.stepNNNNNN.vtu, <stem>.vtu, <stem>.pvd, <stem>.series.csv next to the output
// (VtuStepPath / VtuFinalPath / PvdPath, VtkOutput.hpp:157-174; VelocityManifestPath,
// VelocitySeries.hpp:87-90).
fs::path SiblingPath(const fs::path& base, const std::string& suffix)
{
	return base.parent_path()/(base.stem().string()+suffix);
}

fs::path VtuStep(const fs::path& base, int step)
{
	std::ostringstream name;
	name << ".step" << std::setw(6) << std::setfill('0') << step << ".vtu";
	return SiblingPath(base, name.str());
}

// XML attribute text (EscapeVtkXml, VtkOutput.hpp:48-59).
std::string XmlEscape(const std::string& value)
{
	std::string out;
	for (char c : value) {
		if (c == '&') out += "&amp;";
		else if (c == '<') out += "&lt;";
		else if (c == '>') out += "&gt;";
		else if (c == '"') out += "&quot;";
		else out.push_back(c);
	}
	return out;
}

// ParaView collection of the VTU snapshots (WritePvd, VtkOutput.hpp:176-191).
void WritePvdFile(const fs::path& path, const std::vector<std::pair<double, fs::path>>& snapshots)
{
	std::ofstream out(path);
	if (!out) Fail(-3, "cannot create PVD output: "+path.string());
	out << "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
		<< "  <Collection>\n";
	for (const auto& s : snapshots)
		out << "    <DataSet timestep=\"" << std::setprecision(17) << s.first << "\" group=\"\" part=\"0\" file=\""
			<< XmlEscape(s.second.filename().string()) << "\"/>\n";
	out << "  </Collection>\n</VTKFile>\n";
	out.close();
	if (!out) Fail(-3, "cannot write PVD output: "+path.string());
}

// time,file rows of the text velocity snapshots (WriteVelocityManifest, VelocitySeries.hpp:92-103).
void WriteManifest(const fs::path& path, const std::vector<std::pair<double, fs::path>>& snapshots)
{
	std::ofstream out(path);
	if (!out) Fail(-3, "cannot create velocity manifest: "+path.string());
	out << "time,file\n";
	for (const auto& s : snapshots) out << std::setprecision(17) << s.first << ',' << s.second.filename().string() << '\n';
	out.close();
	if (!out) Fail(-3, "cannot write velocity manifest: "+path.string());
}

// Flow checkpoint: raw float64 state + JSON metadata (FlowCheckpoint.hpp, iga_cuda.cu:566-602).
void WriteCheckpoint(const fs::path& prefix, int64_t nodes, int completed, double time, double dt, double density,
	double viscosity, const std::vector<OutletModel>& outlets, const std::vector<double>& state)
{
	const fs::path state_path = prefix.string()+".state";
	{
		std::ofstream out(state_path, std::ios::binary);
		if (!out) Fail(-3, "cannot create CUDA flow checkpoint state: "+state_path.string());
		out.write(reinterpret_cast<const char*>(state.data()), (std::streamsize)(state.size()*sizeof(double)));
		if (!out) Fail(-3, "cannot write CUDA flow checkpoint state: "+state_path.string());
	}
	std::ofstream meta(prefix.string()+".json");
	if (!meta) Fail(-3, "cannot create checkpoint metadata");
	meta << std::setprecision(17) << "{\n  \"schema_version\": 1,\n  \"nodes\": " << nodes << ",\n  \"fields\": 4,\n"
		<< "  \"completed_step\": " << completed << ",\n  \"physical_time\": " << time << ",\n  \"dt\": " << dt
		<< ",\n  \"density\": " << density << ",\n  \"viscosity\": " << viscosity << ",\n  \"state_file\": \""
		<< state_path.filename().string() << "\",\n  \"state_format\": \"raw_float64\",\n  \"outlets\": [";
	for (size_t i = 0; i < outlets.size(); ++i)
		meta << (i == 0 ? "\n" : ",\n") << "    {\"label\": " << outlets[i].label << ", \"kind\": \"" << outlets[i].kind
			<< "\", \"flow\": " << outlets[i].flow << ", \"pressure\": " << outlets[i].pressure
			<< ", \"capacitor_pressure\": " << outlets[i].capacitor_pressure << "}";
	if (!outlets.empty()) meta << '\n';
	meta << "  ]\n}\n";
}

struct Restart {
	int completed = 0;
	double time = 0.0;
	std::vector<double> state;
};

Restart ReadCheckpoint(const fs::path& prefix, int64_t nodes, double dt, double density, double viscosity,
	std::vector<OutletModel>& outlets)
{
	std::ifstream in(prefix.string()+".json");
	if (!in) Fail(-3, "cannot open flow checkpoint metadata: "+prefix.string()+".json");
	std::stringstream ss;
	ss << in.rdbuf();
	const auto root = json::Parse(ss.str());
	if (root.At("state_format", "flow checkpoint").String("state_format") != "raw_float64")
		Fail(-4, "CUDA flow restart requires raw_float64 checkpoint state");
	if ((int64_t)root.At("nodes", "flow checkpoint").Number("nodes") != nodes)
		Fail(-4, "flow checkpoint node count does not match the database");
	if (root.At("fields", "flow checkpoint").Integer("fields") != 4) Fail(-4, "flow checkpoint must have 4 fields");
	auto same = [](double a, double b) { return std::fabs(a-b) <= 1e-12*std::max(1.0, std::max(std::fabs(a), std::fabs(b))); };
	if (!same(root.At("dt", "flow checkpoint").Number("dt"), dt)
		|| !same(root.At("density", "flow checkpoint").Number("density"), density)
		|| !same(root.At("viscosity", "flow checkpoint").Number("viscosity"), viscosity))
		Fail(-4, "flow checkpoint dt, density or viscosity does not match the case");
	Restart r;
	r.completed = root.At("completed_step", "flow checkpoint").Integer("completed_step");
	r.time = root.At("physical_time", "flow checkpoint").Number("physical_time");
	if (const auto* list = root.Find("outlets"))
		for (const auto& item : list->Array("outlets")) {
			const int label = item.At("label", "outlet").Integer("outlet.label");
			for (auto& m : outlets)
				if (m.label == label) {
					m.flow = item.At("flow", "outlet").Number("outlet.flow");
					m.pressure = item.At("pressure", "outlet").Number("outlet.pressure");
					m.capacitor_pressure = item.At("capacitor_pressure", "outlet").Number("outlet.capacitor_pressure");
				}
		}
	fs::path state_path(root.At("state_file", "flow checkpoint").String("state_file"));
	if (state_path.is_relative()) state_path = fs::path(prefix.string()+".json").parent_path()/state_path;
	std::ifstream sin(state_path, std::ios::binary);
	if (!sin) Fail(-3, "cannot open CUDA flow checkpoint state: "+state_path.string());
	r.state.resize((size_t)nodes*4);
	sin.read(reinterpret_cast<char*>(r.state.data()), (std::streamsize)(r.state.size()*sizeof(double)));
	char extra = 0;
	if (!sin || sin.read(&extra, 1)) Fail(-4, "CUDA flow checkpoint state is truncated or has trailing data");
	return r;
}

int NavierStokes(int argc, char** argv)
{
	const Options options = ParseOptions(argc, argv);
	const auto total_start = Clock::now();
	const fs::path case_dir(options.case_dir);
	HostMesh host = ReadNtiga(options.database);
	const auto labeled = ReadLabeledHexMesh((case_dir/"controlmesh.vtk").string(), host.nodes, host.elements());
	const auto wall = WallTraceBasis(host, labeled);
	const auto reference_velocity = ReadVelocity((case_dir/"initial_velocityfield.txt").string(), host.nodes);
	// simulation_config.json, or a legacy case: simulation_parameter.txt (+ case_config.json) with the
	// reference's legacy flow defaults, steady, viscosity 0.1, density 1, Dirichlet pressure on the
	// outlet labels (iga_cuda.cu:761-795).
	const bool legacy = !fs::exists(case_dir/"simulation_config.json");
	const SimulationConfig config = legacy ? SimulationConfig{}
		: ReadSimulationConfig((case_dir/"simulation_config.json").string());
	bool transient = false;
	double viscosity = 0.1, density = 1.0, dt = 0.0;
	int physical_steps = 1;
	std::vector<OutletModel> outlets;
	std::string boundary_source = "simulation_config.json";
	ResolvedBoundaries legacy_boundaries;
	if (!legacy) {
		const FlowSystem& flow = FindNavierStokesSystem(config, options.system);
		transient = flow.time_integration == "backward_euler";
		viscosity = flow.viscosity;
		density = flow.density;
		dt = transient ? config.dt : 0.0;
		physical_steps = transient ? config.steps : 1;
		outlets = InitializeOutletModels(config, flow);
	} else {
		const TransportParameters parameters = ReadTransportParameters((case_dir/"simulation_parameter.txt").string());
		const CaseConfiguration case_configuration = ReadCaseConfiguration((case_dir/"case_config.json").string());
		const LegacyBoundaries lb = ResolveLegacyBoundaries(case_configuration, labeled.labels, reference_velocity,
			parameters);
		legacy_boundaries.velocity_mask = lb.velocity_mask;
		legacy_boundaries.pressure_mask = lb.pressure_mask;
		legacy_boundaries.velocity = lb.velocity;
		legacy_boundaries.pressure = lb.pressure;
		legacy_boundaries.velocity_nodes = lb.velocity_nodes;
		legacy_boundaries.pressure_nodes = lb.pressure_nodes;
		boundary_source = case_configuration.present ? "case_config.json" : "legacy-defaults";
	}
	auto resolve = [&](const SimulationConfig& step_config, std::map<int, double>& tractions) {
		ResolvedBoundaries r;
		if (legacy) {
			tractions.clear();
			r = legacy_boundaries;
		} else {
			const auto boundary_config = MaterializeOutletPressures(step_config, outlets);
			const auto& system = FindNavierStokesSystem(boundary_config, options.system);
			tractions = ExtractPressureTractions(boundary_config, system);
			r = ResolveFlowBoundaries(boundary_config, system, labeled.labels, reference_velocity);
		}
		for (const int32_t node : wall) {
			if (!r.velocity_mask.at(node)) ++r.velocity_nodes;
			r.velocity_mask[node] = 1;
			for (int d = 0; d < 3; ++d) r.velocity[3*node+d] = 0.0;
		}
		return r;
	};
	std::map<int, double> tractions;
	auto boundaries = resolve(transient ? MaterializeWaveforms(config, case_dir.string(), 0.0) : config, tractions);
	if (!transient)
		for (const auto& m : outlets)
			if (m.kind != "resistance") Fail(-4, "RC/RCR outlets require backward_euler flow");
	if (options.stop_after_step > physical_steps) Fail(-1, "--stop-after-step exceeds configured physical steps");
	const int run_end = options.stop_after_step > 0 ? options.stop_after_step : physical_steps;
	std::cout << "boundary_config=" << boundary_source << " viscosity=" << viscosity << " density=" << density
		<< " time_integration=" << (transient ? "backward_euler" : "steady") << " dt=" << dt
		<< " steps=" << physical_steps << " run_end_step=" << run_end
		<< " velocity_nodes=" << boundaries.velocity_nodes << " pressure_nodes=" << boundaries.pressure_nodes << '\n';
	if (!transient && (!options.restart.empty() || !options.checkpoint.empty() || options.output_every > 0
		|| options.checkpoint_every > 0))
		Fail(-1, "restart, checkpoint, and time-indexed output require transient flow");
	const int64_t nodes = host.nodes;
	Mesh mesh(std::move(host));
	PrintMesh(mesh);
	if (mesh.bad_samples())
		Fail(-5, "mesh has "+std::to_string(mesh.bad_samples())+" non-positive quadrature Jacobians; minimum detJ "
			+std::to_string(mesh.min_detj()));
	const auto preprocess_end = Clock::now();
	tfiga_ns_params params;
	tfiga_ns_default_params(&params);
	params.density = density;
	params.viscosity = viscosity;
	params.dt = dt;
	params.max_newton = options.max_newton;
	params.nonlinear_rtol = options.rtol;
	params.nonlinear_atol = options.atol;
	params.mass_rtol = options.mass_rtol;
	NsSolver solver(mesh, params);
	std::vector<int32_t> traction_labels;
	std::vector<double> traction_values;
	auto upload_boundaries = [&]() {
		solver.SetDirichlet(boundaries.velocity_mask.data(), boundaries.pressure_mask.data(),
			boundaries.velocity.data(), boundaries.pressure.data());
		traction_labels.clear(); traction_values.clear();
		for (const auto& t : tractions) { traction_labels.push_back(t.first); traction_values.push_back(t.second); }
		solver.SetTractions(traction_labels.data(), traction_values.data(), (int)traction_labels.size());
	};
	upload_boundaries();
	int start_step = 0;
	std::vector<double> state((size_t)nodes*4, 0.0);
	if (transient && !options.restart.empty()) {
		auto r = ReadCheckpoint(options.restart, nodes, dt, density, viscosity, outlets);
		state = r.state;
		start_step = r.completed;
		std::cout << "restart=" << options.restart << " completed_step=" << start_step << " physical_time=" << r.time << '\n';
	} else if (transient) {
		for (int64_t node = 0; node < nodes; ++node) {
			if (boundaries.velocity_mask[node]) for (int d = 0; d < 3; ++d) state[4*node+d] = boundaries.velocity[3*node+d];
			if (boundaries.pressure_mask[node]) state[4*node+3] = boundaries.pressure[node];
		}
	}
	solver.SetState(state.data(), state.data());
	long long total_iterations = 0;
	double total_assembly = 0.0, total_linear = 0.0;
	// VTU snapshots and the PVD collection (iga_cuda.cu:902-916, 1086-1100, 1126-1141); "auto"
	// resolves to VTU in this build (the Bezier VTKHDF format needs HDF5).
	const VtkGrid grid = options.output.empty() ? VtkGrid{} : ReadVtkGrid(case_dir/"controlmesh.vtk");
	std::vector<std::pair<double, fs::path>> vtu_snapshots, velocity_snapshots;
	if (transient && options.output_every > 0) {
		const fs::path text = TimeIndexed(options.output, start_step);
		WriteText(text, state);
		const fs::path vtu = VtuStep(options.output, start_step);
		WriteVtuFile(grid, vtu, state, start_step*dt);
		vtu_snapshots.push_back({start_step*dt, vtu});
		velocity_snapshots.push_back({start_step*dt, text});
	}
	for (int step = start_step; step < run_end; ++step) {
		if (step > start_step) solver.CommitStep();
		const double physical_time = transient ? (step+1)*dt : 0.0;
		const SimulationConfig step_config = transient ? MaterializeWaveforms(config, case_dir.string(), physical_time)
			: config;
		std::vector<double> previous_capacitor(outlets.size());
		for (size_t i = 0; i < outlets.size(); ++i) previous_capacitor[i] = outlets[i].capacitor_pressure;
		const int max_outlet = outlets.empty() ? 1 : 12;
		bool outlet_converged = false;
		for (int coupling = 0; coupling < max_outlet; ++coupling) {
			boundaries = resolve(step_config, tractions);
			upload_boundaries();
			double initial = -1.0;
			bool converged = false;
			tfiga_newton_report last{};
			for (int k = 0; k < options.max_newton; ++k) {
				last = solver.NewtonIteration(initial);
				if (initial < 0.0) initial = last.residual_l2;
				total_assembly += last.assembly_ms/1e3;
				const double rms = last.residual_l2/std::sqrt(4.0*nodes);
				if (last.converged) {
					std::cout << "step=" << step+1 << " time=" << physical_time << " converged newton=" << k
						<< " residual_l2=" << last.residual_l2 << " residual_rms=" << rms << " tolerance=" << last.tolerance
						<< " absolute_rms_tolerance=" << options.atol << " continuity_l2=" << last.continuity_l2
						<< " continuity_sum=" << last.continuity_sum << " net_boundary_flow=" << last.net_boundary_flow
						<< " relative_mass_imbalance=" << last.relative_mass_imbalance
						<< " mass_tolerance=" << options.mass_rtol << '\n';
					converged = true;
					break;
				}
				total_linear += last.linear_ms/1e3;
				total_iterations += last.linear_iterations;
				std::cout << "step=" << step+1 << " time=" << physical_time << " newton=" << k
					<< " residual_l2=" << last.residual_l2 << " residual_rms=" << rms
					<< " continuity_l2=" << last.continuity_l2 << " continuity_sum=" << last.continuity_sum
					<< " net_boundary_flow=" << last.net_boundary_flow
					<< " relative_mass_imbalance=" << last.relative_mass_imbalance << " update_l2=" << last.update_l2
					<< " linear_iterations=" << last.linear_iterations << " linear_residual=" << last.linear_residual
					<< " singular_diagonal_blocks=" << last.singular_diagonal_blocks
					<< " assembly_s=" << last.assembly_ms/1e3 << " linear_s=" << last.linear_ms/1e3 << '\n';
			}
			if (!converged)
				Fail(-6, "Navier-Stokes nonlinear solve reached MAX_NEWTON at physical step "+std::to_string(step+1)
					+" (nonlinear_residual="+Precise(last.residual_l2)+", continuity_l2="+Precise(last.continuity_l2)
					+", net_boundary_flow="+Precise(last.net_boundary_flow)+", relative_mass_imbalance="
					+Precise(last.relative_mass_imbalance)+")");
			if (outlets.empty()) { outlet_converged = true; break; }
			// Outlet fixed point (iga_cuda.cu:1059-1082, OutletModel.hpp:92-150).
			std::vector<int32_t> labels;
			for (const auto& m : outlets) labels.push_back(m.label);
			std::vector<double> flows(outlets.size());
			solver.BoundaryFlows(labels.data(), (int)labels.size(), flows.data());
			double change = 0.0, scale = 1.0;
			std::vector<std::array<double, 2>> evaluated(outlets.size());
			for (size_t i = 0; i < outlets.size(); ++i) {
				auto m = outlets[i];
				m.capacitor_pressure = previous_capacitor[i];
				evaluated[i] = EvaluateOutletModel(m, flows[i], dt);
				change = std::max(change, std::fabs(evaluated[i][0]-outlets[i].pressure));
				scale = std::max(scale, std::fabs(evaluated[i][0]));
			}
			const double tolerance = 1e-8+1e-6*scale;
			std::cout << "step=" << step+1 << " time=" << physical_time << " outlet_iteration=" << coupling
				<< " pressure_change=" << change << " tolerance=" << tolerance << '\n';
			if (change <= tolerance) {
				for (size_t i = 0; i < outlets.size(); ++i) {
					outlets[i].flow = flows[i];
					outlets[i].pressure = evaluated[i][0];
					outlets[i].capacitor_pressure = evaluated[i][1];
					std::cout << "outlet label=" << outlets[i].label << " flow=" << outlets[i].flow
						<< " pressure=" << outlets[i].pressure << " capacitor_pressure="
						<< outlets[i].capacitor_pressure << '\n';
				}
				outlet_converged = true;
				break;
			}
			for (size_t i = 0; i < outlets.size(); ++i) {
				outlets[i].flow = flows[i];
				outlets[i].pressure = 0.5*outlets[i].pressure+0.5*evaluated[i][0];
			}
		}
		if (!outlet_converged)
			Fail(-6, "outlet fixed-point iteration did not converge at physical step "+std::to_string(step+1));
		const int completed = step+1;
		if (options.output_every > 0 && completed%options.output_every == 0) {
			solver.GetState(state.data());
			const fs::path text = TimeIndexed(options.output, completed);
			WriteText(text, state);
			const fs::path vtu = VtuStep(options.output, completed);
			WriteVtuFile(grid, vtu, state, completed*dt);
			vtu_snapshots.push_back({completed*dt, vtu});
			velocity_snapshots.push_back({completed*dt, text});
		}
		if (!options.checkpoint.empty()
			&& (completed == run_end || (options.checkpoint_every > 0 && completed%options.checkpoint_every == 0))) {
			solver.GetState(state.data());
			WriteCheckpoint(options.checkpoint, nodes, completed, completed*dt, dt, density, viscosity, outlets, state);
			std::cout << "checkpoint=" << options.checkpoint << " completed_step=" << completed << '\n';
		}
	}
	solver.GetState(state.data());
	double vsq = 0.0, psq = 0.0;
	for (int64_t node = 0; node < nodes; ++node) {
		for (int d = 0; d < 3; ++d) vsq += state[4*node+d]*state[4*node+d];
		psq += state[4*node+3]*state[4*node+3];
	}
	if (!options.output.empty()) {
		WriteText(options.output, state);
		WriteVtk(case_dir/"controlmesh.vtk", options.output+".vtk", state);
		const double final_time = transient ? run_end*dt : 0.0;
		const fs::path vtu = SiblingPath(options.output, ".vtu");
		WriteVtuFile(grid, vtu, state, final_time);
		if (vtu_snapshots.empty()) vtu_snapshots.push_back({final_time, vtu});
		WritePvdFile(SiblingPath(options.output, ".pvd"), vtu_snapshots);
		if (!velocity_snapshots.empty())
			WriteManifest(SiblingPath(options.output, ".series.csv"), velocity_snapshots);
	}
	std::cout << "navier_stokes_cuda nodes=" << nodes << " elements=" << mesh.host().elements()
		<< " steps=" << physical_steps << " run_end_step=" << run_end
		<< " preprocess_s=" << std::chrono::duration<double>(preprocess_end-total_start).count()
		<< " assembly_s=" << total_assembly << " linear_s=" << total_linear
		<< " total_linear_iterations=" << total_iterations << " state_l2=" << std::sqrt(vsq+psq)
		<< " velocity_l2=" << std::sqrt(vsq) << " pressure_l2=" << std::sqrt(psq)
		<< " gpu_used_gib=" << DeviceBytesPeak()/1073741824.0 << '\n';
	return 0;
}

// WriteTransport (iga_cuda.cu:327-335): "node N0 N+" rows.
void WriteTransportText(const fs::path& path, const std::vector<double>& values)
{
	std::ofstream out(path);
	if (!out) Fail(-3, "cannot create "+path.string());
	out << std::setprecision(17);
	for (size_t node = 0; node < values.size()/2; ++node)
		out << node << ' ' << values[2*node] << ' ' << values[2*node+1] << '\n';
}

// WriteTransportVtk (iga_cuda.cu:337-349): control mesh + N0 / Nplus point scalars.
void WriteTransportVtk(const fs::path& mesh_path, const fs::path& path, const std::vector<double>& values)
{
	std::ifstream mesh(mesh_path);
	std::ofstream out(path);
	if (!mesh) Fail(-3, "cannot open VTK mesh "+mesh_path.string());
	if (!out) Fail(-3, "cannot create "+path.string());
	out << mesh.rdbuf() << "\nSCALARS N0 double 1\nLOOKUP_TABLE default\n" << std::setprecision(17);
	for (size_t node = 0; node < values.size()/2; ++node) out << values[2*node] << '\n';
	out << "SCALARS Nplus double 1\nLOOKUP_TABLE default\n";
	for (size_t node = 0; node < values.size()/2; ++node) out << values[2*node+1] << '\n';
}

// `transport DATABASE CASE_DIR [STEPS] [OUTPUT] [VELOCITY]` (Transport, iga_cuda.cu:621-732).
int Transport(int argc, char** argv)
{
	if (argc < 4) Fail(-1, "usage: iga_cuda transport DATABASE.ntiga CASE_DIR [STEPS] [OUTPUT] [VELOCITY]");
	const auto total_start = Clock::now();
	const fs::path case_dir(argv[3]);
	HostMesh host = ReadNtiga(argv[2]);
	TransportParameters parameters = ReadTransportParameters((case_dir/"simulation_parameter.txt").string());
	if (argc >= 5) parameters.steps = std::stoi(argv[4]);
	const auto labeled = ReadLabeledHexMesh((case_dir/"controlmesh.vtk").string(), host.nodes, host.elements());
	const fs::path velocity_path = argc >= 7 ? fs::path(argv[6]) : case_dir/"initial_velocityfield.txt";
	const auto velocity_host = ReadVelocity(velocity_path.string(), host.nodes);
	const auto configuration = ReadCaseConfiguration((case_dir/"case_config.json").string());
	const auto boundaries = ResolveLegacyBoundaries(configuration, labeled.labels, velocity_host, parameters);
	std::cout << "boundary_config=" << (configuration.present ? "case_config.json" : "legacy-defaults")
		<< " transport_nodes=" << boundaries.transport_nodes << '\n';
	Mesh mesh(std::move(host));
	PrintMesh(mesh);
	const auto preprocess_end = Clock::now();
	if (mesh.bad_samples())
		Fail(-5, "geometry has "+std::to_string(mesh.bad_samples())+" non-positive Jacobian samples");
	std::vector<double> velocity(3*(size_t)mesh.nodes());
	for (size_t node = 0; node < velocity_host.size(); ++node)
		for (int d = 0; d < 3; ++d) velocity[3*node+d] = velocity_host[node][d];
	const TransportCoefficients coefficients{parameters.diffusion, parameters.vplus, parameters.kplus,
		parameters.kminus, parameters.detach_plus, parameters.dt, parameters.artificial_diffusion};
	constexpr int kRestart = 50;
	const auto assembly_start = Clock::now();
	TransportSolver solver(mesh, coefficients, velocity.data(), boundaries.transport_mask.data(),
		boundaries.n0.data(), boundaries.nplus.data(), kRestart);
	const auto assembly_end = Clock::now();
	long long total_iterations = 0;
	unsigned singular = 0;
	const auto solve_start = Clock::now();
	for (int step = 0; step < parameters.steps; ++step) {
		const TransportStepResult r = solver.Step(1e-8, 10000);
		total_iterations += r.iterations;
		singular = std::max(singular, r.singular_blocks);
		if ((step+1)%25 == 0 || step+1 == parameters.steps)
			std::cout << "transport step=" << step+1 << '/' << parameters.steps << " iterations=" << r.iterations
				<< " residual=" << r.residual << '\n';
	}
	CudaCheck(cudaStreamSynchronize(solver.stream()), "transport solve");
	const auto solve_end = Clock::now();
	const double norm = solver.StateNorm();
	if (argc >= 6) {
		std::vector<double> output(2*(size_t)mesh.nodes());
		solver.GetState(output.data());
		WriteTransportText(argv[5], output);
		WriteTransportVtk(case_dir/"controlmesh.vtk", std::string(argv[5])+".vtk", output);
	}
	std::cout << "transport_cuda nodes=" << mesh.nodes() << " elements=" << mesh.host().elements()
		<< " steps=" << parameters.steps
		<< " preprocess_s=" << std::chrono::duration<double>(preprocess_end-total_start).count()
		<< " assembly_s=" << std::chrono::duration<double>(assembly_end-assembly_start).count()
		<< " solve_s=" << std::chrono::duration<double>(solve_end-solve_start).count()
		<< " total_iterations=" << total_iterations << " final_l2=" << norm
		<< " singular_diagonal_blocks=" << singular << " gpu_used_gib=" << DeviceBytesPeak()/1073741824.0 << '\n';
	return 0;
}

} // namespace
} // namespace tfiga

namespace tfiga {
void RecordLastError(const char* message);
}

namespace {

const char* OutletKindName(int32_t kind)
{
	switch (kind) {
	case TFIGA_OUTLET_RESISTANCE: return "resistance";
	case TFIGA_OUTLET_RC: return "windkessel_rc";
	case TFIGA_OUTLET_RCR: return "windkessel_rcr";
	default: tfiga::Fail(TFIGA_E_INVALID, "unknown outlet kind");
	}
}

template <class F>
int HostGuard(F&& body)
{
	try {
		body();
		return TFIGA_OK;
	} catch (const tfiga::Error& error) {
		tfiga::RecordLastError(error.what());
		return error.status;
	} catch (const std::exception& error) {
		tfiga::RecordLastError(error.what());
		return TFIGA_E_INVALID;
	}
}

} // namespace

// The no-slip bases of the navier-stokes command (WallTraceBasis, BoundarySupport.hpp:82-150) from
// the database (this library's .ntiga reader) and controlmesh.vtk: sorted node indices.
extern "C" int tfiga_wall_trace_basis(const char* database, const char* controlmesh_vtk, int32_t* nodes_out,
	int64_t capacity, int64_t* count)
{
	return HostGuard([&] {
		if (!database || !controlmesh_vtk || !count) tfiga::Fail(TFIGA_E_INVALID, "null argument");
		const tfiga::HostMesh host = tfiga::ReadNtiga(database);
		const auto labeled = tfiga::ReadLabeledHexMesh(controlmesh_vtk, host.nodes, host.elements());
		const auto wall = tfiga::WallTraceBasis(host, labeled);
		*count = (int64_t)wall.size();
		int64_t i = 0;
		for (const int32_t node : wall) {
			if (i < capacity && nodes_out) nodes_out[i] = node;
			++i;
		}
	});
}

// The navier-stokes command's checkpoint (WriteCudaFlowCheckpoint, iga_cuda.cu:584-602).
extern "C" int tfiga_write_flow_checkpoint(const char* prefix, int64_t nodes, int32_t completed_step,
	double physical_time, double dt, double density, double viscosity, const tfiga_outlet* outlets, int32_t count,
	const double* state)
{
	return HostGuard([&] {
		if (!prefix || !state || nodes <= 0 || count < 0 || (count > 0 && !outlets))
			tfiga::Fail(TFIGA_E_INVALID, "null argument");
		std::vector<tfiga::OutletModel> models((size_t)count);
		for (int32_t i = 0; i < count; ++i) {
			models[i].label = outlets[i].label;
			models[i].kind = OutletKindName(outlets[i].kind);
			models[i].flow = outlets[i].flow;
			models[i].pressure = outlets[i].pressure;
			models[i].capacitor_pressure = outlets[i].capacitor_pressure;
		}
		tfiga::WriteCheckpoint(prefix, nodes, completed_step, physical_time, dt, density, viscosity, models,
			std::vector<double>(state, state+4*nodes));
	});
}

// Restart from a checkpoint (ReadFlowCheckpointMetadata, ValidateFlowCheckpoint, ReadCudaFlowCheckpoint,
// include/FlowCheckpoint.hpp:186-211, iga_cuda.cu:566-582): the outlets whose labels appear in the
// metadata take its flow, pressure and capacitor pressure.
extern "C" int tfiga_read_flow_checkpoint(const char* prefix, int64_t nodes, double dt, double density,
	double viscosity, tfiga_outlet* outlets, int32_t count, double* state, int32_t* completed_step,
	double* physical_time)
{
	return HostGuard([&] {
		if (!prefix || !state || nodes <= 0 || count < 0 || (count > 0 && !outlets))
			tfiga::Fail(TFIGA_E_INVALID, "null argument");
		std::vector<tfiga::OutletModel> models((size_t)count);
		for (int32_t i = 0; i < count; ++i) {
			models[i].label = outlets[i].label;
			models[i].flow = outlets[i].flow;
			models[i].pressure = outlets[i].pressure;
			models[i].capacitor_pressure = outlets[i].capacitor_pressure;
		}
		const auto r = tfiga::ReadCheckpoint(prefix, nodes, dt, density, viscosity, models);
		std::copy(r.state.begin(), r.state.end(), state);
		for (int32_t i = 0; i < count; ++i) {
			outlets[i].flow = models[i].flow;
			outlets[i].pressure = models[i].pressure;
			outlets[i].capacitor_pressure = models[i].capacitor_pressure;
		}
		if (completed_step) *completed_step = r.completed;
		if (physical_time) *physical_time = r.time;
	});
}

// The VTU snapshot writer of the navier-stokes command (WriteNavierStokesVtu, iga_cuda.cu:366-388:
// the control mesh of mesh_vtk with velocity and pressure point arrays and the physical time).
extern "C" int tfiga_write_vtu(const char* mesh_vtk, const char* output, const double* state, int64_t nodes,
	double time)
{
	try {
		if (!mesh_vtk || !output || !state || nodes <= 0) tfiga::Fail(TFIGA_E_INVALID, "null argument");
		const tfiga::VtkGrid grid = tfiga::ReadVtkGrid(mesh_vtk);
		const std::vector<double> values(state, state+4*nodes);
		tfiga::WriteVtuFile(grid, output, values, time);
		return TFIGA_OK;
	} catch (const tfiga::Error& error) {
		tfiga::RecordLastError(error.what());
		return error.status;
	} catch (const std::exception& error) {
		tfiga::RecordLastError(error.what());
		return TFIGA_E_INVALID;
	}
}

extern "C" int tfiga_main(int argc, char** argv)
{
	try {
		if (argc < 2) throw std::runtime_error("usage: iga_cuda device-info|mesh-check|navier-stokes|transport ...");
		tfiga::RequireDevice();
		const std::string command(argv[1]);
		tfiga::PrintDevice();
		int status = 0;
		if (command == "device-info") return 0;
		if (command == "mesh-check") {
			if (argc != 3) throw std::runtime_error("usage: iga_cuda mesh-check DATABASE.ntiga");
			status = tfiga::MeshCheck(argv[2]);
		} else if (command == "navier-stokes") {
			status = tfiga::NavierStokes(argc, argv);
		} else if (command == "transport") {
			status = tfiga::Transport(argc, argv);
		} else {
			throw std::runtime_error("unknown command: "+command);
		}
		std::cout << "cuda_allocations scope=project_device_buffers requested_peak_bytes=" << tfiga::DeviceBytesPeak()
			<< " requested_live_bytes=" << tfiga::DeviceBytesLive() << '\n';
		std::cout.flush();
		return status;
	} catch (const std::exception& error) {
		std::cerr << "iga_cuda: " << error.what() << '\n';
		std::cerr << "cuda_allocations scope=project_device_buffers requested_peak_bytes=" << tfiga::DeviceBytesPeak()
			<< " requested_live_bytes=" << tfiga::DeviceBytesLive() << '\n';
		return 1;
	}
}
