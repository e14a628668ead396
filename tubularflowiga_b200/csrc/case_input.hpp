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
// EvaluateTemporalFunction (include/TemporalFunction.hpp:97-143), analytic kinds.
double EvaluateTemporal(const TemporalFunction& f, double time);
// MaterializeBoundaryWaveforms (include/TemporalFunction.hpp:145-171).
SimulationConfig MaterializeWaveforms(const SimulationConfig& config, double time);

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

} // namespace tfiga
