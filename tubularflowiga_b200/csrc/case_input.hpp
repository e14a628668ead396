// Case-directory inputs of the navier-stokes command and the host-side
// boundary physics: simulation_config.json (schema v4 subset used by the flow
// path), controlmesh.vtk labels, initial_velocityfield.txt, the wall-trace
// no-slip basis, Dirichlet resolution, waveforms and 0D outlet models.
#pragma once

#include "mesh.hpp"

#include <array>
#include <map>
#include <set>
#include <string>
#include <vector>

namespace tfiga {

struct Condition {
	std::string field, type;
	std::vector<double> value;
	std::string profile;
	double scale = 1.0;
	std::string waveform;
	double resistance = 0.0, proximal_resistance = 0.0, distal_resistance = 0.0, capacitance = 0.0;
	double reference_pressure = 0.0, initial_pressure = 0.0;
	bool pressure_gauge = false;
};

struct Boundary {
	int label = -1;
	std::string name;
	std::vector<Condition> conditions;
};

struct TemporalFunction {
	std::string name, kind;
	double value = 0.0, mean = 0.0, amplitude = 0.0, period = 0.0, phase = 0.0;
	std::vector<double> cosine, sine;
	std::string file;
};

struct FlowSystem {
	std::string name, kind;
	std::vector<std::string> unknowns;
	double viscosity = 0.0, density = 1.0;
	std::string time_integration = "steady";
};

struct SimulationConfig {
	double dt = 0.0;
	int steps = 1;
	std::vector<FlowSystem> systems;
	std::vector<Boundary> boundaries;
	std::vector<TemporalFunction> temporal;
};

// ReadSimulationConfiguration (include/SimulationConfig.hpp), flow subset.
SimulationConfig ReadSimulationConfig(const std::string& path);
// FindNavierStokesSystem (solvers/cpu/include/GenericCaseInput.hpp:153-172).
const FlowSystem& FindNavierStokesSystem(const SimulationConfig& config, const std::string& name);
// One (time, value) sample of a periodic_table waveform.
struct TemporalSample {
	double time = 0.0, value = 0.0;
};
// ParseTemporalCsv / ReadTemporalCsv (include/TemporalFunction.hpp:45-88): `time,value` lines ('#'
// comments, blank lines and a leading `time,value` header skipped), times strictly increasing in
// [0, period), at least two samples starting at 0; the reference's messages.
std::vector<TemporalSample> ParseTemporalCsv(const std::string& text, double period, const std::string& context);
std::vector<TemporalSample> ReadTemporalCsv(const std::string& path, double period);
// EvaluateTemporalFunction (include/TemporalFunction.hpp:97-134): constant, sinusoid, fourier, and
// periodic_table (linear interpolation of `samples`, wrapping from the last sample to the first at
// t = period).
double EvaluateTemporal(const TemporalFunction& f, double time, const std::vector<TemporalSample>* samples = nullptr);
// MaterializeBoundaryWaveforms (include/TemporalFunction.hpp:145-171): periodic_table files are read
// relative to case_directory (absolute paths rejected).
SimulationConfig MaterializeWaveforms(const SimulationConfig& config, const std::string& case_directory,
	double time);

// ReadLabeledHexMesh (solvers/cpu/include/BoundarySupport.hpp:25-73).
struct LabeledHexMesh {
	std::vector<std::array<int32_t, 8>> cells;
	std::vector<int> labels;
};
LabeledHexMesh ReadLabeledHexMesh(const std::string& path, int64_t nodes, int64_t elements);
// ReadVelocity (solvers/cpu/include/CaseInput.hpp:72-83).
std::vector<std::array<double, 3>> ReadVelocity(const std::string& path, int64_t nodes);
// WallTraceBasis (BoundarySupport.hpp:82-150): bases with a nonzero trace on a wall face.
std::set<int32_t> WallTraceBasis(const HostMesh& mesh, const LabeledHexMesh& labeled);

struct ResolvedBoundaries {
	std::vector<int32_t> velocity_mask, pressure_mask;
	std::vector<double> velocity;   // 3 per node
	std::vector<double> pressure;   // 1 per node
	size_t velocity_nodes = 0, pressure_nodes = 0;
};
// ResolveFlowBoundaries (GenericCaseInput.hpp:174-259).
ResolvedBoundaries ResolveFlowBoundaries(const SimulationConfig& config, const FlowSystem& system,
	const std::vector<int>& labels, const std::vector<std::array<double, 3>>& reference_velocity);
// ExtractPressureTractions (include/PressureTraction.hpp:11-30).
std::map<int, double> ExtractPressureTractions(const SimulationConfig& config, const FlowSystem& system);

// 0D outlet models (include/OutletModel.hpp:15-174).
struct OutletModel {
	int label = -1;
	std::string kind;   // resistance | windkessel_rc | windkessel_rcr
	double resistance = 0.0, proximal = 0.0, distal = 0.0, capacitance = 0.0, reference_pressure = 0.0;
	double capacitor_pressure = 0.0, flow = 0.0, pressure = 0.0;
};
std::vector<OutletModel> InitializeOutletModels(const SimulationConfig& config, const FlowSystem& system);
// EvaluateOutletModel: returns {pressure, capacitor pressure}.
std::array<double, 2> EvaluateOutletModel(const OutletModel& model, double flow, double dt);
// MaterializeOutletPressures (OutletModel.hpp:152-170).
SimulationConfig MaterializeOutletPressures(const SimulationConfig& config, const std::vector<OutletModel>& models);

// ---- legacy two-species transport case (the `transport` command) ----------

// iga::TransportParameters (solvers/cpu/include/CaseInput.hpp:19-33).
struct TransportParameters {
	double diffusion = 0.0, vplus = 0.0, vminus = 0.0, kplus = 0.0, kminus = 0.0;
	double detach_plus = 0.0, detach_minus = 0.0, dt = 0.0;
	int steps = 0;
	double n0_bc = 0.0, nplus_bc = 0.0, nminus_bc = 0.0, artificial_diffusion = 0.0;
};
// ReadTransportParameters (CaseInput.hpp:85-118): whitespace-separated `key value` pairs of
// simulation_parameter.txt; D vplus vminus kplus kminus k'plus k'minus dt nstep N0bc Nplusbc
// Nminusbc required, artificial_diffusion (or artificial_diffusion_weight) optional.
TransportParameters ReadTransportParameters(const std::string& path);

// case_config.json schema 1 (include/CaseConfig.hpp:29-48, 280-387).
struct CaseBoundaryRule {
	int label = -1;
	std::string name, type = "interior";   // interior | wall | inlet | outlet
	bool has_velocity = false, has_velocity_scale = false, has_pressure = false, has_transport = false;
	std::array<double, 3> velocity{{0.0, 0.0, 0.0}};
	double velocity_scale = 1.0, pressure = 0.0, n0 = 0.0, nplus = 0.0;
};
struct CaseConfiguration {
	bool present = false;
	bool inherit_legacy = true;
	std::vector<CaseBoundaryRule> boundaries;
};
// ReadCaseConfiguration (CaseConfig.hpp:373-387): an absent file is an empty configuration.
CaseConfiguration ReadCaseConfiguration(const std::string& path);
CaseConfiguration ParseCaseConfiguration(const std::string& text);

// ResolveBoundaryConditions (CaseInput.hpp:162-258): legacy labels (0 wall, 1 inlet, >= 2 outlet)
// unless the configuration replaces them, then the configured rules label by label.
struct LegacyBoundaries {
	std::vector<int32_t> velocity_mask, pressure_mask, transport_mask;
	std::vector<double> velocity, pressure, n0, nplus;   // velocity 3 per node
	size_t velocity_nodes = 0, pressure_nodes = 0, transport_nodes = 0;
};
LegacyBoundaries ResolveLegacyBoundaries(const CaseConfiguration& configuration, const std::vector<int>& labels,
	const std::vector<std::array<double, 3>>& reference_velocity, const TransportParameters& parameters);

} // namespace tfiga
