// Case input and host boundary physics (see case_input.hpp).
#include "case_input.hpp"

#include <filesystem>
#include "json.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace tfiga {

namespace {

std::string ReadText(const std::string& path)
{
	std::ifstream in(path);
	if (!in) Fail(-3, "cannot open "+path);
	std::stringstream ss;
	ss << in.rdbuf();
	return ss.str();
}

double OptionalNumber(const json::Value& object, const char* key, double fallback, const std::string& context)
{
	const auto* v = object.Find(key);
	return v ? v->Number(context+"."+key) : fallback;
}

// The reference's generic JSON validation helpers (include/CaseConfig.hpp:230-270), defined with
// the case_config.json reader below; its simulation_config.json parser reuses them, messages included.
void KnownKeys(const json::Value& object, std::initializer_list<const char*> allowed, const std::string& context);
int CaseInteger(const json::Value& v, const std::string& context);
const std::string& CaseString(const json::Value& v, const std::string& context);

[[noreturn]] void SimulationFail(const std::string& message) { Fail(-4, "simulation_config.json: "+message); }

double CaseNumber(const json::Value& v, const std::string& context);
const json::Value& CaseObject(const json::Value& v, const std::string& context);

const json::Value& Required(const json::Value& object, const char* key, const std::string& context)
{
	const auto* v = object.Find(key);
	if (!v) SimulationFail(context+" requires '"+key+"'");
	return *v;
}

const std::vector<json::Value>& CaseArray(const json::Value& v, const std::string& context)
{
	if (v.kind != json::Value::Kind::Array) Fail(-4, "case_config.json: "+context+" must be an array");
	return v.items;
}

std::vector<double> ValueVector(const json::Value& v, const std::string& context)
{
	if (v.kind == json::Value::Kind::Number) return {CaseNumber(v, context)};
	std::vector<double> out;
	const auto& items = CaseArray(v, context);
	for (size_t i = 0; i < items.size(); ++i) out.push_back(CaseNumber(items[i], context+"["+std::to_string(i)+"]"));
	return out;
}

// The checks of ParseSimulationConfiguration (include/SimulationConfig.hpp:263-600) that concern
// the flow path, in the reference's order and with its messages (its generic helpers name
// case_config.json): root keys and schema 2/3/4 rules; fields; time; temporal functions; equation
// systems (names, kinds, unknowns, Navier-Stokes physics and time integration); boundaries and their
// conditions (known keys, fields, kinds, value / profile, outlet-model parameters, waveforms).  Not
// repeated: the contents of geometry, mesh, coupling, perfusate, velocity_sources, physiology and
// the terms and stabilization of transport systems.
void ValidateSimulationRoot(const json::Value& root)
{
	CaseObject(root, "root");
	KnownKeys(root, {"schema_version", "dimension", "geometry", "mesh", "fields", "equation_systems", "boundaries",
		"time", "temporal_functions", "velocity_sources", "physiology", "simulation_scope", "perfusate",
		"external_circuit", "coupling"}, "root");
	const int schema = CaseInteger(Required(root, "schema_version", "root"), "schema_version");
	const auto* dimension = root.Find("dimension");
	if (schema == 2) {
		if (dimension || root.Find("geometry") || root.Find("mesh"))
			SimulationFail("schema_version 2 does not accept dimension, geometry, or mesh");
	} else if (schema == 3) {
		if (!dimension || CaseString(*dimension, "dimension") != "3d")
			SimulationFail("schema_version 3 3d configuration requires dimension '3d'");
		if (root.Find("geometry") || root.Find("mesh"))
			SimulationFail("schema_version 3 3d configuration does not accept geometry or mesh");
	} else if (schema == 4) {
		if (!dimension || CaseString(*dimension, "dimension") != "3d")
			SimulationFail("schema_version 4 requires dimension '3d'");
		Required(root, "geometry", "root");
		Required(root, "mesh", "root");
	} else {
		SimulationFail("supported schema versions are 2, 3, and 4");
	}

	std::set<std::string> fields;
	const auto& field_list = CaseArray(Required(root, "fields", "root"), "fields");
	for (size_t i = 0; i < field_list.size(); ++i) {
		const std::string context = "fields["+std::to_string(i)+"]";
		const auto& object = CaseObject(field_list[i], context);
		KnownKeys(object, {"name", "kind", "initial_value"}, context);
		const std::string name = CaseString(Required(object, "name", context), context+".name");
		const std::string kind = CaseString(Required(object, "kind", context), context+".kind");
		if (kind != "scalar" && kind != "vector3" && kind != "pressure")
			SimulationFail("unsupported field kind '"+kind+"'");
		if (const auto* v = object.Find("initial_value")) CaseNumber(*v, context+".initial_value");
		if (name.empty() || !fields.insert(name).second) SimulationFail("field names must be non-empty and unique");
	}
	if (fields.empty()) SimulationFail("fields cannot be empty");

	const auto& time = CaseObject(Required(root, "time", "root"), "time");
	KnownKeys(time, {"dt", "steps"}, "time");
	const double dt = CaseNumber(Required(time, "dt", "time"), "time.dt");
	CaseInteger(Required(time, "steps", "time"), "time.steps");
	if (!(dt > 0.0)) SimulationFail("time.dt must be positive");

	std::set<std::string> temporal;
	if (const auto* list = root.Find("temporal_functions")) {
		const auto& functions = CaseArray(*list, "temporal_functions");
		for (size_t i = 0; i < functions.size(); ++i) {
			const std::string context = "temporal_functions["+std::to_string(i)+"]";
			const auto& object = CaseObject(functions[i], context);
			KnownKeys(object, {"name", "kind", "units", "value", "mean", "amplitude", "period", "phase", "file",
				"interpolation", "cosine", "sine"}, context);
			const std::string name = CaseString(Required(object, "name", context), context+".name");
			const std::string kind = CaseString(Required(object, "kind", context), context+".kind");
			if (kind != "constant" && kind != "sinusoid" && kind != "periodic_table" && kind != "fourier")
				SimulationFail("unsupported temporal function kind '"+kind+"'");
			const std::string units = CaseString(Required(object, "units", context), context+".units");
			if (name.empty() || !temporal.insert(name).second)
				SimulationFail("temporal function names must be non-empty and unique");
			if (units.empty()) SimulationFail("temporal function units cannot be empty");
			for (const char* key : {"value", "mean", "amplitude", "period", "phase"})
				if (const auto* v = object.Find(key)) CaseNumber(*v, context+"."+key);
			const double period = object.Find("period") ? object.Find("period")->number : 0.0;
			std::string file, interpolation;
			if (const auto* v = object.Find("file")) file = CaseString(*v, context+".file");
			if (const auto* v = object.Find("interpolation")) interpolation = CaseString(*v, context+".interpolation");
			std::vector<double> cosine, sine;
			if (const auto* v = object.Find("cosine")) cosine = ValueVector(*v, context+".cosine");
			if (const auto* v = object.Find("sine")) sine = ValueVector(*v, context+".sine");
			if (kind == "constant" && !object.Find("value")) SimulationFail("constant temporal function requires value");
			if (kind == "sinusoid" && (!object.Find("mean") || !object.Find("amplitude") || !(period > 0.0)))
				SimulationFail("sinusoid requires mean, amplitude, and positive period");
			if (kind == "periodic_table" && (file.empty() || !(period > 0.0) || interpolation != "linear"))
				SimulationFail("periodic_table requires file, positive period, and linear interpolation");
			if (kind == "fourier" && (!(period > 0.0) || cosine.size() != sine.size() || cosine.empty()))
				SimulationFail("fourier requires positive period and equal non-empty cosine/sine arrays");
		}
	}

	const auto& systems = CaseArray(Required(root, "equation_systems", "root"), "equation_systems");
	std::set<std::string> system_names;
	for (size_t i = 0; i < systems.size(); ++i) {
		const std::string context = "equation_systems["+std::to_string(i)+"]";
		const auto& object = CaseObject(systems[i], context);
		KnownKeys(object, {"name", "kind", "unknowns", "terms", "stabilization", "viscosity", "density",
			"time_integration"}, context);
		const std::string name = CaseString(Required(object, "name", context), context+".name");
		const std::string kind = CaseString(Required(object, "kind", context), context+".kind");
		if (kind != "linear_transport" && kind != "navier_stokes")
			SimulationFail("unsupported equation-system kind '"+kind+"'");
		if (name.empty() || !system_names.insert(name).second)
			SimulationFail("equation-system names must be non-empty and unique");
		const auto& unknowns = CaseArray(Required(object, "unknowns", context), context+".unknowns");
		std::set<std::string> local;
		for (size_t j = 0; j < unknowns.size(); ++j) {
			const std::string u = CaseString(unknowns[j], context+".unknowns["+std::to_string(j)+"]");
			if (!fields.count(u)) SimulationFail("unknown field '"+u+"'");
			if (!local.insert(u).second) SimulationFail("duplicate system unknown '"+u+"'");
		}
		if (local.empty()) SimulationFail("system unknowns cannot be empty");
		double viscosity = 0.0, density = 1.0;
		std::string integration = "steady";
		if (const auto* v = object.Find("viscosity")) viscosity = CaseNumber(*v, context+".viscosity");
		if (const auto* v = object.Find("density")) density = CaseNumber(*v, context+".density");
		if (const auto* v = object.Find("time_integration")) integration = CaseString(*v, context+".time_integration");
		if (kind == "navier_stokes") {
			if (!(viscosity > 0.0)) SimulationFail("navier_stokes viscosity must be positive");
			if (!(density > 0.0)) SimulationFail("navier_stokes density must be positive");
			if (integration != "steady" && integration != "backward_euler")
				SimulationFail("navier_stokes time_integration must be 'steady' or 'backward_euler'");
		} else if (object.Find("density")) {
			SimulationFail("density applies only to navier_stokes");
		}
		if (kind == "linear_transport") {
			// the system-level checks of a transport system (its terms' contents are not repeated here)
			if (!object.Find("time_integration")) integration = "backward_euler";
			if (integration != "backward_euler" && integration != "bdf2")
				SimulationFail("linear_transport time_integration must be 'backward_euler' or 'bdf2'");
			const auto* terms = object.Find("terms");
			if (terms == nullptr || CaseArray(*terms, context+".terms").empty())
				SimulationFail("linear_transport requires terms");
		}
	}
	if (systems.empty()) SimulationFail("equation_systems cannot be empty");

	const auto& boundaries = CaseArray(Required(root, "boundaries", "root"), "boundaries");
	std::set<int> labels;
	for (size_t i = 0; i < boundaries.size(); ++i) {
		const std::string context = "boundaries["+std::to_string(i)+"]";
		const auto& object = CaseObject(boundaries[i], context);
		KnownKeys(object, {"label", "name", "conditions"}, context);
		const int label = CaseInteger(Required(object, "label", context), context+".label");
		CaseString(Required(object, "name", context), context+".name");
		if (!labels.insert(label).second) SimulationFail("duplicate boundary label");
		const auto& conditions = CaseArray(Required(object, "conditions", context), context+".conditions");
		std::set<std::string> conditioned;
		for (size_t j = 0; j < conditions.size(); ++j) {
			const std::string c = context+".conditions["+std::to_string(j)+"]";
			const auto& cond = CaseObject(conditions[j], c);
			KnownKeys(cond, {"field", "type", "value", "coefficient", "exterior_value", "profile", "scale", "waveform",
				"resistance", "proximal_resistance", "distal_resistance", "capacitance", "reference_pressure",
				"initial_pressure", "pressure_gauge", "dirichlet_dofs"}, c);
			const std::string field = CaseString(Required(cond, "field", c), c+".field");
			const std::string type = CaseString(Required(cond, "type", c), c+".type");
			if (type != "dirichlet" && type != "no_flux" && type != "flux" && type != "robin"
				&& type != "advective_outflow" && type != "pressure_traction" && type != "resistance"
				&& type != "windkessel_rc" && type != "windkessel_rcr")
				SimulationFail("unsupported boundary condition '"+type+"'");
			if (!fields.count(field) || !conditioned.insert(field).second)
				SimulationFail("boundary fields must exist and be unique per boundary");
			std::vector<double> value;
			if (const auto* v = cond.Find("value")) value = ValueVector(*v, c+".value");
			double coefficient = 0.0, resistance = 0.0, proximal = 0.0, distal = 0.0, capacitance = 0.0;
			if (const auto* v = cond.Find("coefficient")) coefficient = CaseNumber(*v, c+".coefficient");
			if (const auto* v = cond.Find("exterior_value")) CaseNumber(*v, c+".exterior_value");
			std::string dofs = "face_support";
			if (const auto* v = cond.Find("dirichlet_dofs")) dofs = CaseString(*v, c+".dirichlet_dofs");
			if (dofs != "face_support" && dofs != "node_label")
				SimulationFail("dirichlet_dofs must be 'face_support' or 'node_label'");
			std::string profile, waveform;
			if (const auto* v = cond.Find("profile")) profile = CaseString(*v, c+".profile");
			if (const auto* v = cond.Find("scale")) CaseNumber(*v, c+".scale");
			if (const auto* v = cond.Find("waveform")) waveform = CaseString(*v, c+".waveform");
			if (const auto* v = cond.Find("resistance")) resistance = CaseNumber(*v, c+".resistance");
			if (const auto* v = cond.Find("proximal_resistance")) proximal = CaseNumber(*v, c+".proximal_resistance");
			if (const auto* v = cond.Find("distal_resistance")) distal = CaseNumber(*v, c+".distal_resistance");
			if (const auto* v = cond.Find("capacitance")) capacitance = CaseNumber(*v, c+".capacitance");
			if (const auto* v = cond.Find("reference_pressure")) CaseNumber(*v, c+".reference_pressure");
			if (const auto* v = cond.Find("initial_pressure")) CaseNumber(*v, c+".initial_pressure");
			bool gauge = false;
			if (const auto* v = cond.Find("pressure_gauge")) {
				if (v->kind != json::Value::Kind::Bool) Fail(-4, "case_config.json: "+c+".pressure_gauge must be a boolean");
				gauge = v->boolean;
			}
			if (type == "dirichlet" && value.empty() && profile.empty())
				SimulationFail("dirichlet requires value or profile");
			if (!value.empty() && !profile.empty()) SimulationFail("boundary condition cannot set both value and profile");
			if (type == "flux" && value.size() != 1) SimulationFail("flux requires one value");
			if (type == "pressure_traction" && value.size() != 1) SimulationFail("pressure_traction requires one value");
			if (gauge && (type != "pressure_traction" || value.size() != 1))
				SimulationFail("pressure_gauge requires pressure_traction with one value");
			if (type == "robin" && coefficient == 0.0) SimulationFail("robin requires nonzero coefficient");
			if (type == "resistance" && !(resistance > 0.0))
				SimulationFail("resistance outlet requires positive resistance");
			if (type == "windkessel_rc" && (!(resistance > 0.0) || !(capacitance > 0.0)))
				SimulationFail("windkessel_rc requires positive resistance and capacitance");
			if (type == "windkessel_rcr" && (proximal < 0.0 || !(distal > 0.0) || !(capacitance > 0.0)))
				SimulationFail("windkessel_rcr requires nonnegative proximal resistance and positive distal resistance "
					"and capacitance");
			if (!waveform.empty() && ((type != "dirichlet" && type != "pressure_traction") || !temporal.count(waveform)))
				SimulationFail("waveform must name a temporal function on a Dirichlet or pressure_traction condition");
		}
	}
}

std::vector<double> Numbers(const json::Value& v, const std::string& context)
{
	if (v.kind == json::Value::Kind::Number) return {v.number};
	std::vector<double> out;
	for (const auto& item : v.Array(context)) out.push_back(item.Number(context));
	return out;
}

} // namespace

SimulationConfig ReadSimulationConfig(const std::string& path)
{
	const json::Value root = json::Parse(ReadText(path));
	if (!root.IsObject()) Fail(-4, "simulation_config.json root must be an object");
	ValidateSimulationRoot(root);
	SimulationConfig config;
	const auto& time = root.At("time", "root");
	config.dt = time.At("dt", "time").Number("time.dt");
	config.steps = time.At("steps", "time").Integer("time.steps");
	if (const auto* temporal = root.Find("temporal_functions")) {
		for (const auto& item : temporal->Array("temporal_functions")) {
			TemporalFunction f;
			f.name = item.At("name", "temporal function").String("temporal function.name");
			f.kind = item.At("kind", "temporal function").String("temporal function.kind");
			f.value = OptionalNumber(item, "value", 0.0, "temporal function");
			f.mean = OptionalNumber(item, "mean", 0.0, "temporal function");
			f.amplitude = OptionalNumber(item, "amplitude", 0.0, "temporal function");
			f.period = OptionalNumber(item, "period", 0.0, "temporal function");
			f.phase = OptionalNumber(item, "phase", 0.0, "temporal function");
			if (const auto* c = item.Find("cosine")) f.cosine = Numbers(*c, "temporal function.cosine");
			if (const auto* s = item.Find("sine")) f.sine = Numbers(*s, "temporal function.sine");
			if (const auto* file = item.Find("file")) f.file = file->String("temporal function.file");
			if (f.kind != "constant" && f.kind != "sinusoid" && f.kind != "fourier" && f.kind != "periodic_table")
				Fail(-4, "unknown temporal function kind '"+f.kind+"'");
			if (f.kind != "constant" && !(f.period > 0.0))
				Fail(-4, "temporal function '"+f.name+"' needs a positive period");
			if (f.cosine.size() != f.sine.size())
				Fail(-4, "fourier cosine and sine arrays must have the same length");
			config.temporal.push_back(f);
		}
	}
	for (const auto& item : root.At("equation_systems", "root").Array("equation_systems")) {
		FlowSystem s;
		s.name = item.At("name", "equation system").String("equation system.name");
		s.kind = item.At("kind", "equation system").String("equation system.kind");
		if (const auto* unknowns = item.Find("unknowns"))
			for (const auto& u : unknowns->Array("unknowns")) s.unknowns.push_back(u.String("unknown"));
		s.viscosity = OptionalNumber(item, "viscosity", 0.0, "equation system");
		s.density = OptionalNumber(item, "density", 1.0, "equation system");
		if (const auto* ti = item.Find("time_integration")) s.time_integration = ti->String("time_integration");
		if (s.kind == "navier_stokes" && s.time_integration != "steady" && s.time_integration != "backward_euler")
			Fail(-4, "navier_stokes time_integration must be steady or backward_euler");
		config.systems.push_back(s);
	}
	for (const auto& item : root.At("boundaries", "root").Array("boundaries")) {
		Boundary b;
		b.label = item.At("label", "boundary").Integer("boundary.label");
		if (const auto* name = item.Find("name")) b.name = name->String("boundary.name");
		for (const auto& c : item.At("conditions", "boundary").Array("boundary.conditions")) {
			Condition k;
			const std::string ctx = "boundary "+std::to_string(b.label)+" condition";
			k.field = c.At("field", ctx).String(ctx+".field");
			k.type = c.At("type", ctx).String(ctx+".type");
			if (const auto* v = c.Find("value")) k.value = Numbers(*v, ctx+".value");
			if (const auto* p = c.Find("profile")) k.profile = p->String(ctx+".profile");
			k.scale = OptionalNumber(c, "scale", 1.0, ctx);
			if (const auto* w = c.Find("waveform")) k.waveform = w->String(ctx+".waveform");
			k.resistance = OptionalNumber(c, "resistance", 0.0, ctx);
			k.proximal_resistance = OptionalNumber(c, "proximal_resistance", 0.0, ctx);
			k.distal_resistance = OptionalNumber(c, "distal_resistance", 0.0, ctx);
			k.capacitance = OptionalNumber(c, "capacitance", 0.0, ctx);
			k.reference_pressure = OptionalNumber(c, "reference_pressure", 0.0, ctx);
			k.initial_pressure = OptionalNumber(c, "initial_pressure", 0.0, ctx);
			if (const auto* g = c.Find("pressure_gauge")) k.pressure_gauge = g->kind == json::Value::Kind::Bool && g->boolean;
			b.conditions.push_back(k);
		}
		config.boundaries.push_back(b);
	}
	return config;
}

const FlowSystem& FindNavierStokesSystem(const SimulationConfig& config, const std::string& name)
{
	for (const auto& s : config.systems) {
		if (name.empty() && s.kind == "navier_stokes") return s;
		if (!name.empty() && s.name == name) {
			if (s.kind != "navier_stokes") Fail(-4, "equation system '"+name+"' is not navier_stokes");
			return s;
		}
	}
	if (name.empty()) Fail(-4, "simulation configuration has no navier_stokes equation system");
	Fail(-4, "simulation configuration has no navier_stokes system named '"+name+"'");
}

namespace {

std::string TrimTemporal(const std::string& text)
{
	const auto first = text.find_first_not_of(" \t\r");
	if (first == std::string::npos) return {};
	const auto last = text.find_last_not_of(" \t\r");
	return text.substr(first, last-first+1);
}

double TemporalNumber(const std::string& text, const std::string& context)
{
	const std::string token = TrimTemporal(text);
	size_t used = 0;
	double value = 0.0;
	try {
		value = std::stod(token, &used);
	} catch (const std::exception&) {
		Fail(-4, context+" contains a non-numeric value");
	}
	if (used != token.size() || !std::isfinite(value)) Fail(-4, context+" contains a non-finite or malformed value");
	return value;
}

} // namespace

std::vector<TemporalSample> ParseTemporalCsv(const std::string& text, double period, const std::string& context)
{
	if (!(period > 0.0)) Fail(-4, context+" requires a positive period");
	std::vector<TemporalSample> samples;
	std::istringstream input(text);
	std::string line;
	size_t number = 0;
	while (std::getline(input, line)) {
		++number;
		line = TrimTemporal(line);
		if (line.empty() || line.front() == '#') continue;
		const auto comma = line.find(',');
		if (comma == std::string::npos || line.find(',', comma+1) != std::string::npos)
			Fail(-4, context+" line "+std::to_string(number)+" must contain exactly time,value");
		const std::string first = TrimTemporal(line.substr(0, comma)), second = TrimTemporal(line.substr(comma+1));
		if (samples.empty() && first == "time" && second == "value") continue;
		const std::string where = context+" line "+std::to_string(number);
		const double time = TemporalNumber(first, where), value = TemporalNumber(second, where);
		if (time < 0.0 || time >= period) Fail(-4, context+" sample times must be in [0, period)");
		if (!samples.empty() && !(time > samples.back().time))
			Fail(-4, context+" sample times must be strictly increasing");
		samples.push_back({time, value});
	}
	if (samples.size() < 2 || samples.front().time != 0.0)
		Fail(-4, context+" requires at least two samples beginning at time zero");
	return samples;
}

std::vector<TemporalSample> ReadTemporalCsv(const std::string& path, double period)
{
	std::ifstream in(path, std::ios::binary);
	if (!in) Fail(-3, "cannot open temporal CSV: "+path);
	std::ostringstream text;
	text << in.rdbuf();
	return ParseTemporalCsv(text.str(), period, path);
}

double EvaluateTemporal(const TemporalFunction& f, double time, const std::vector<TemporalSample>* samples)
{
	const double pi = 3.141592653589793238462643383279502884;
	if (f.kind == "constant") return f.value;
	if (!(f.period > 0.0)) Fail(-4, "temporal function period must be positive");
	double wrapped = std::fmod(time, f.period);
	if (wrapped < 0.0) wrapped += f.period;
	const double theta = 2.0*pi*wrapped/f.period+f.phase;
	if (f.kind == "sinusoid") return f.mean+f.amplitude*std::sin(theta);
	if (f.kind == "fourier") {
		double v = f.mean;
		for (size_t h = 0; h < f.cosine.size(); ++h) {
			const double angle = (double)(h+1)*theta;
			v += f.cosine[h]*std::cos(angle)+f.sine[h]*std::sin(angle);
		}
		return v;
	}
	if (samples == nullptr) Fail(-4, "periodic_table evaluation requires loaded samples");
	if (samples->size() < 2 || samples->front().time != 0.0) Fail(-4, "periodic_table samples are invalid");
	// the first sample after `wrapped`; past the last sample the segment closes on the first at t = period
	const auto upper = std::upper_bound(samples->begin(), samples->end(), wrapped,
		[](double value, const TemporalSample& sample) { return value < sample.time; });
	TemporalSample lower, next;
	if (upper == samples->end()) {
		lower = samples->back();
		next = {f.period, samples->front().value};
	} else {
		if (upper == samples->begin()) Fail(-4, "periodic_table samples must begin at zero");
		lower = *(upper-1);
		next = *upper;
	}
	const double fraction = (wrapped-lower.time)/(next.time-lower.time);
	return lower.value+fraction*(next.value-lower.value);
}

SimulationConfig MaterializeWaveforms(const SimulationConfig& config, const std::string& case_directory, double time)
{
	SimulationConfig out = config;
	for (auto& b : out.boundaries)
		for (auto& c : b.conditions) {
			if (c.waveform.empty()) continue;
			const auto it = std::find_if(config.temporal.begin(), config.temporal.end(),
				[&](const TemporalFunction& f) { return f.name == c.waveform; });
			if (it == config.temporal.end()) Fail(-4, "unknown temporal function '"+c.waveform+"'");
			std::vector<TemporalSample> samples;
			const std::vector<TemporalSample>* loaded = nullptr;
			if (it->kind == "periodic_table") {
				const std::filesystem::path relative(it->file);
				if (relative.is_absolute()) Fail(-4, "temporal CSV path must be relative to the case directory");
				samples = ReadTemporalCsv((std::filesystem::path(case_directory)/relative).string(), it->period);
				loaded = &samples;
			}
			const double factor = EvaluateTemporal(*it, time, loaded);
			if (c.profile.empty()) for (double& v : c.value) v *= factor;
			else c.scale *= factor;
			c.waveform.clear();
		}
	return out;
}

LabeledHexMesh ReadLabeledHexMesh(const std::string& path, int64_t nodes, int64_t elements)
{
	std::ifstream in(path);
	if (!in) Fail(-3, "cannot open mesh: "+path);
	std::string token;
	int64_t points = 0;
	while (in >> token) if (token == "POINTS") {
		std::string type;
		if (!(in >> points >> type)) Fail(-4, "invalid POINTS record");
		break;
	}
	if (points != nodes) Fail(-4, "VTK point count does not match database nodes");
	for (int64_t k = 0; k < 3*points; ++k) {
		double ignored;
		if (!(in >> ignored)) Fail(-4, "VTK POINTS record is truncated");
	}
	int64_t cells = 0, values = 0;
	while (in >> token) if (token == "CELLS") {
		if (!(in >> cells >> values)) Fail(-4, "invalid CELLS record");
		break;
	}
	if (cells != elements) Fail(-4, "VTK cell count does not match database elements");
	LabeledHexMesh mesh;
	mesh.cells.resize(cells);
	for (auto& cell : mesh.cells) {
		int count = 0;
		if (!(in >> count) || count != 8) Fail(-4, "only eight-node VTK hexahedra are supported");
		for (auto& node : cell)
			if (!(in >> node) || node < 0 || node >= points) Fail(-4, "invalid hexahedron connectivity");
	}
	int64_t point_data = 0;
	while (in >> token) if (token == "POINT_DATA") {
		if (!(in >> point_data)) Fail(-4, "invalid POINT_DATA record");
		break;
	}
	if (point_data != points) Fail(-4, "VTK POINT_DATA count does not match database nodes");
	while (in >> token) if (token == "LOOKUP_TABLE") { in >> token; break; }
	if (!in) Fail(-4, "VTK point labels were not found");
	mesh.labels.resize(points);
	for (auto& label : mesh.labels) {
		double v = 0.0;
		if (!(in >> v)) Fail(-4, "VTK point-label array is truncated");
		label = (int)v;
		if (v != (double)label) Fail(-4, "VTK point label is not integral");
	}
	return mesh;
}

std::vector<std::array<double, 3>> ReadVelocity(const std::string& path, int64_t nodes)
{
	std::ifstream in(path);
	if (!in) Fail(-3, "cannot open velocity field: "+path);
	std::vector<std::array<double, 3>> v(nodes);
	for (auto& x : v)
		if (!(in >> x[0] >> x[1] >> x[2])) Fail(-4, "velocity field is truncated");
	std::string extra;
	if (in >> extra) Fail(-4, "velocity field contains extra records");
	return v;
}

std::set<int32_t> WallTraceBasis(const HostMesh& mesh, const LabeledHexMesh& labeled)
{
	// External faces of the control hex mesh (faces used once), with the local
	// face numbering of the element faces (BoundarySupport.hpp:84-87).
	static const int corners[6][4] = {{0, 3, 2, 1}, {0, 1, 5, 4}, {1, 2, 6, 5},
		{2, 3, 7, 6}, {0, 4, 7, 3}, {4, 5, 6, 7}};
	std::map<std::array<int32_t, 4>, std::array<int64_t, 3>> faces;   // key -> {element, face, uses}
	for (int64_t e = 0; e < (int64_t)labeled.cells.size(); ++e)
		for (int f = 0; f < 6; ++f) {
			std::array<int32_t, 4> key;
			for (int c = 0; c < 4; ++c) key[c] = labeled.cells[e][corners[f][c]];
			std::sort(key.begin(), key.end());
			auto& entry = faces[key];
			if (entry[2] == 0) { entry[0] = e; entry[1] = f; }
			if (++entry[2] > 2) Fail(-4, "non-manifold control-mesh face");
		}
	std::set<int32_t> result;
	for (const auto& item : faces) {
		if (item.second[2] != 1) continue;
		const int64_t e = item.second[0];
		const int f = (int)item.second[1];
		bool wall = true;
		for (int c = 0; c < 4 && wall; ++c) wall = labeled.labels.at(labeled.cells[e][corners[f][c]]) == 0;
		if (!wall) continue;
		// Bezier columns on the face (FaceBezierColumns, :117-132).
		std::vector<int> columns;
		for (int k = 0; k < 4; ++k)
			for (int j = 0; j < 4; ++j)
				for (int i = 0; i < 4; ++i)
					if ((f == 0 && k == 0) || (f == 1 && j == 0) || (f == 2 && i == 3) || (f == 3 && j == 3)
						|| (f == 4 && i == 0) || (f == 5 && k == 3))
						columns.push_back(i+4*j+16*k);
		for (int32_t a = mesh.element_offsets[e]; a < mesh.element_offsets[e+1]; ++a)
			for (int32_t k = mesh.extraction_offsets[a]; k < mesh.extraction_offsets[a+1]; ++k)
				if (mesh.extraction_values[k] != 0.0
					&& std::find(columns.begin(), columns.end(), (int)mesh.extraction_columns[k]) != columns.end()) {
					result.insert(mesh.connectivity[a]);
					break;
				}
	}
	return result;
}

ResolvedBoundaries ResolveFlowBoundaries(const SimulationConfig& config, const FlowSystem& system,
	const std::vector<int>& labels, const std::vector<std::array<double, 3>>& reference_velocity)
{
	if (system.unknowns.size() != 2) Fail(-4, "navier_stokes requires [velocity, pressure] unknowns");
	const auto& vname = system.unknowns[0];
	const auto& pname = system.unknowns[1];
	const size_t n = labels.size();
	if (reference_velocity.size() != n) Fail(-4, "velocity profile and boundary labels have different node counts");
	ResolvedBoundaries r;
	r.velocity_mask.assign(n, 0);
	r.pressure_mask.assign(n, 0);
	r.velocity.assign(3*n, 0.0);
	r.pressure.assign(n, 0.0);
	std::set<int> mesh_labels, configured;
	for (int l : labels) if (l >= 0) mesh_labels.insert(l);
	bool traction = false;
	for (const auto& b : config.boundaries) {
		if (!mesh_labels.count(b.label))
			Fail(-4, "simulation_config.json boundary label "+std::to_string(b.label)
				+" is not present in controlmesh.vtk");
		configured.insert(b.label);
		for (const auto& c : b.conditions) {
			if (c.field != vname && c.field != pname) continue;
			if (!c.waveform.empty()) Fail(-7, "time-dependent Navier-Stokes boundary execution is not implemented");
			if (c.type == "pressure_traction") {
				if (c.field != pname || c.value.size() != 1)
					Fail(-4, "pressure_traction requires the Navier-Stokes pressure field");
				if (c.pressure_gauge)
					Fail(-4, "pressure_traction already fixes the pressure reference; remove pressure_gauge "
						"to preserve every continuity equation");
				traction = true;
				continue;
			}
			if (c.type != "dirichlet")
				Fail(-4, "navier_stokes boundary field '"+c.field+"' currently supports only dirichlet conditions");
			if (c.field == vname) {
				if (c.profile.empty() && c.value.size() != 3)
					Fail(-4, "velocity Dirichlet condition requires three values or a profile");
				if (!c.profile.empty() && c.profile != "initial_velocityfield.txt")
					Fail(-4, "unsupported velocity profile '"+c.profile+"'");
				for (size_t i = 0; i < n; ++i)
					if (labels[i] == b.label) {
						r.velocity_mask[i] = 1;
						for (int d = 0; d < 3; ++d)
							r.velocity[3*i+d] = c.profile.empty() ? c.value[d] : c.scale*reference_velocity[i][d];
					}
			} else {
				if (c.value.size() != 1) Fail(-4, "pressure Dirichlet condition requires one value");
				for (size_t i = 0; i < n; ++i)
					if (labels[i] == b.label) { r.pressure_mask[i] = 1; r.pressure[i] = c.value[0]; }
			}
		}
	}
	for (int l : mesh_labels)
		if (!configured.count(l))
			Fail(-4, "mesh boundary label "+std::to_string(l)+" has no simulation_config.json boundary definition");
	r.velocity_nodes = (size_t)std::count(r.velocity_mask.begin(), r.velocity_mask.end(), 1);
	r.pressure_nodes = (size_t)std::count(r.pressure_mask.begin(), r.pressure_mask.end(), 1);
	if (r.velocity_nodes == 0 || (r.pressure_nodes == 0 && !traction))
		Fail(-4, "navier_stokes requires velocity Dirichlet and pressure gauge/traction boundaries");
	return r;
}

std::map<int, double> ExtractPressureTractions(const SimulationConfig& config, const FlowSystem& system)
{
	if (system.kind != "navier_stokes" || system.unknowns.size() != 2)
		Fail(-4, "pressure traction requires a Navier-Stokes system");
	const auto& pname = system.unknowns[1];
	std::map<int, double> out;
	for (const auto& b : config.boundaries)
		for (const auto& c : b.conditions) {
			if (c.type != "pressure_traction") continue;
			if (c.field != pname || c.value.size() != 1)
				Fail(-4, "pressure_traction must provide one value for the pressure field");
			if (!out.emplace(b.label, c.value[0]).second) Fail(-4, "duplicate pressure traction boundary label");
		}
	return out;
}

std::vector<OutletModel> InitializeOutletModels(const SimulationConfig& config, const FlowSystem& system)
{
	if (system.kind != "navier_stokes" || system.unknowns.size() != 2)
		Fail(-4, "outlet models require a Navier-Stokes velocity-pressure system");
	const auto& pname = system.unknowns[1];
	std::vector<OutletModel> models;
	for (const auto& b : config.boundaries)
		for (const auto& c : b.conditions) {
			if (c.field != pname || (c.type != "resistance" && c.type != "windkessel_rc" && c.type != "windkessel_rcr"))
				continue;
			OutletModel m;
			m.label = b.label;
			m.kind = c.type;
			m.resistance = c.resistance;
			m.proximal = c.proximal_resistance;
			m.distal = c.distal_resistance;
			m.capacitance = c.capacitance;
			m.reference_pressure = c.reference_pressure;
			m.capacitor_pressure = c.initial_pressure;
			m.pressure = c.type == "resistance" ? c.reference_pressure : c.initial_pressure;
			models.push_back(m);
		}
	return models;
}

std::array<double, 2> EvaluateOutletModel(const OutletModel& m, double flow, double dt)
{
	if (!std::isfinite(flow)) Fail(-6, "outlet flow must be finite");
	if (m.kind == "resistance") return {m.reference_pressure+m.resistance*flow, m.capacitor_pressure};
	if (!(dt > 0.0)) Fail(-4, "RC/RCR outlets require positive transient dt");
	const double r = m.kind == "windkessel_rc" ? m.resistance : m.distal;
	const double pc = (m.capacitance*m.capacitor_pressure/dt+flow+m.reference_pressure/r)/(m.capacitance/dt+1.0/r);
	return {pc+(m.kind == "windkessel_rcr" ? m.proximal*flow : 0.0), pc};
}

SimulationConfig MaterializeOutletPressures(const SimulationConfig& config, const std::vector<OutletModel>& models)
{
	SimulationConfig out = config;
	std::map<int, double> pressures;
	for (const auto& m : models) pressures.emplace(m.label, m.pressure);
	for (auto& b : out.boundaries) {
		const auto it = pressures.find(b.label);
		if (it == pressures.end()) continue;
		for (auto& c : b.conditions)
			if (c.type == "resistance" || c.type == "windkessel_rc" || c.type == "windkessel_rcr") {
				c.type = "pressure_traction";
				c.value = {it->second};
			}
	}
	return out;
}

// ---- legacy two-species transport case ------------------------------------

TransportParameters ReadTransportParameters(const std::string& path)
{
	std::ifstream in(path);
	if (!in) Fail(-3, "cannot open simulation parameters: "+path);
	std::map<std::string, double> values;
	std::string key;
	double value = 0.0;
	while (in >> key >> value) values[key] = value;
	auto required = [&](const char* name) {
		const auto it = values.find(name);
		if (it == values.end()) Fail(-4, std::string("missing transport parameter: ")+name);
		return it->second;
	};
	TransportParameters p;
	p.diffusion = required("D");
	p.vplus = required("vplus");
	p.vminus = required("vminus");
	p.kplus = required("kplus");
	p.kminus = required("kminus");
	p.detach_plus = required("k'plus");
	p.detach_minus = required("k'minus");
	p.dt = required("dt");
	p.steps = (int)required("nstep");
	p.n0_bc = required("N0bc");
	p.nplus_bc = required("Nplusbc");
	p.nminus_bc = required("Nminusbc");
	auto artificial = values.find("artificial_diffusion");
	if (artificial == values.end()) artificial = values.find("artificial_diffusion_weight");
	if (artificial != values.end()) p.artificial_diffusion = artificial->second;
	if (p.dt <= 0.0 || p.steps < 0) Fail(-4, "dt and nstep must be positive");
	return p;
}

namespace {

[[noreturn]] void CaseFail(const std::string& message) { Fail(-4, "case_config.json: "+message); }

void KnownKeys(const json::Value& object, std::initializer_list<const char*> allowed, const std::string& context)
{
	// the reference walks its keys in sorted order (a std::map), so the first unknown key it reports is
	// the smallest one
	const std::string* first = nullptr;
	for (const auto& m : object.members) {
		bool ok = false;
		for (const char* a : allowed) ok = ok || m.first == a;
		if (!ok && (first == nullptr || m.first < *first)) first = &m.first;
	}
	if (first) CaseFail("unknown "+context+" key '"+*first+"'");
}

const json::Value& CaseObject(const json::Value& v, const std::string& context)
{
	if (!v.IsObject()) CaseFail(context+" must be an object");
	return v;
}

double CaseNumber(const json::Value& v, const std::string& context)
{
	if (v.kind != json::Value::Kind::Number || !std::isfinite(v.number)) CaseFail(context+" must be a finite number");
	return v.number;
}

int CaseInteger(const json::Value& v, const std::string& context)
{
	const double n = CaseNumber(v, context);
	if (std::floor(n) != n || n < 0.0 || n > 2147483647.0) CaseFail(context+" must be a non-negative integer");
	return (int)n;
}

const std::string& CaseString(const json::Value& v, const std::string& context)
{
	if (v.kind != json::Value::Kind::String) CaseFail(context+" must be a string");
	return v.text;
}

CaseBoundaryRule ParseRule(const json::Value& value, size_t index)
{
	const std::string context = "boundaries.conditions["+std::to_string(index)+"]";
	const auto& object = CaseObject(value, context);
	KnownKeys(object, {"label", "name", "type", "velocity", "velocity_scale", "pressure", "transport"}, context);
	const auto* label = object.Find("label");
	const auto* type = object.Find("type");
	if (!label || !type) CaseFail(context+" requires label and type");
	CaseBoundaryRule rule;
	rule.label = CaseInteger(*label, context+".label");
	rule.type = CaseString(*type, context+".type");
	if (rule.type != "interior" && rule.type != "wall" && rule.type != "inlet" && rule.type != "outlet")
		CaseFail("unsupported boundary type '"+rule.type+"'");
	if (const auto* name = object.Find("name")) rule.name = CaseString(*name, context+".name");
	if (const auto* scale = object.Find("velocity_scale")) {
		rule.has_velocity_scale = true;
		rule.velocity_scale = CaseNumber(*scale, context+".velocity_scale");
	}
	if (const auto* velocity = object.Find("velocity")) {
		if (velocity->kind != json::Value::Kind::Array) CaseFail(context+".velocity must be an array");
		if (velocity->items.size() != 3) CaseFail(context+".velocity must have three entries");
		rule.has_velocity = true;
		for (int i = 0; i < 3; ++i)
			rule.velocity[i] = CaseNumber(velocity->items[i], context+".velocity["+std::to_string(i)+"]");
	}
	if (const auto* pressure = object.Find("pressure")) {
		rule.has_pressure = true;
		rule.pressure = CaseNumber(*pressure, context+".pressure");
	}
	if (const auto* transport = object.Find("transport")) {
		CaseObject(*transport, context+".transport");
		KnownKeys(*transport, {"N0", "Nplus"}, context+".transport");
		const auto* n0 = transport->Find("N0");
		const auto* nplus = transport->Find("Nplus");
		if (!n0 || !nplus) CaseFail(context+".transport requires N0 and Nplus");
		rule.has_transport = true;
		rule.n0 = CaseNumber(*n0, context+".transport.N0");
		rule.nplus = CaseNumber(*nplus, context+".transport.Nplus");
	}
	if (rule.has_velocity && rule.has_velocity_scale) CaseFail(context+" cannot set both velocity and velocity_scale");
	if (rule.type == "interior") {
		if (rule.has_velocity || rule.has_velocity_scale || rule.has_pressure || rule.has_transport)
			CaseFail("interior boundary rules cannot set values");
	} else if (rule.type == "wall") {
		if (rule.has_velocity_scale || rule.has_pressure || rule.has_transport)
			CaseFail("wall rules only support an optional velocity");
	} else if (rule.type == "inlet") {
		if (rule.has_pressure) CaseFail("inlet rules cannot set pressure");
	} else if (rule.has_velocity || rule.has_velocity_scale || rule.has_transport) {
		CaseFail("outlet rules only support an optional pressure");
	}
	return rule;
}

} // namespace

CaseConfiguration ParseCaseConfiguration(const std::string& text)
{
	json::Value root;
	try {
		root = json::Parse(text);
	} catch (const Error&) {
		throw;
	} catch (const std::exception& error) {
		CaseFail(error.what());
	}
	CaseObject(root, "root");
	KnownKeys(root, {"schema_version", "boundaries"}, "root");
	if (const auto* version = root.Find("schema_version"))
		if (CaseInteger(*version, "schema_version") != 1) CaseFail("only schema_version 1 is supported");
	const auto* boundaries = root.Find("boundaries");
	if (!boundaries) CaseFail("missing boundaries object");
	CaseObject(*boundaries, "boundaries");
	KnownKeys(*boundaries, {"inherit_legacy", "conditions"}, "boundaries");
	CaseConfiguration configuration;
	configuration.present = true;
	if (const auto* inherit = boundaries->Find("inherit_legacy")) {
		if (inherit->kind != json::Value::Kind::Bool) CaseFail("boundaries.inherit_legacy must be a boolean");
		configuration.inherit_legacy = inherit->boolean;
	}
	const auto* conditions = boundaries->Find("conditions");
	if (!conditions) CaseFail("boundaries.conditions is required");
	if (conditions->kind != json::Value::Kind::Array) CaseFail("boundaries.conditions must be an array");
	std::set<int> labels;
	for (size_t i = 0; i < conditions->items.size(); ++i) {
		CaseBoundaryRule rule = ParseRule(conditions->items[i], i);
		if (!labels.insert(rule.label).second) CaseFail("duplicate boundary label "+std::to_string(rule.label));
		configuration.boundaries.push_back(std::move(rule));
	}
	return configuration;
}

CaseConfiguration ReadCaseConfiguration(const std::string& path)
{
	std::ifstream in(path);
	if (!in) return {};
	std::stringstream ss;
	ss << in.rdbuf();
	return ParseCaseConfiguration(ss.str());
}

LegacyBoundaries ResolveLegacyBoundaries(const CaseConfiguration& configuration, const std::vector<int>& labels,
	const std::vector<std::array<double, 3>>& reference_velocity, const TransportParameters& parameters)
{
	if (labels.size() != reference_velocity.size())
		Fail(-4, "boundary labels and velocity field have different node counts");
	const size_t nodes = labels.size();
	LegacyBoundaries r;
	r.velocity_mask.assign(nodes, 0);
	r.pressure_mask.assign(nodes, 0);
	r.transport_mask.assign(nodes, 0);
	r.velocity.assign(3*nodes, 0.0);
	r.pressure.assign(nodes, 0.0);
	r.n0.assign(nodes, 0.0);
	r.nplus.assign(nodes, 0.0);
	auto clear = [&](size_t node) {
		r.velocity_mask[node] = r.pressure_mask[node] = r.transport_mask[node] = 0;
		for (int d = 0; d < 3; ++d) r.velocity[3*node+d] = 0.0;
		r.pressure[node] = r.n0[node] = r.nplus[node] = 0.0;
	};
	if (!configuration.present || configuration.inherit_legacy)
		for (size_t node = 0; node < nodes; ++node) {
			if (labels[node] == 0) {
				r.velocity_mask[node] = 1;
			} else if (labels[node] == 1) {
				r.velocity_mask[node] = 1;
				for (int d = 0; d < 3; ++d) r.velocity[3*node+d] = parameters.vplus*reference_velocity[node][d];
				r.transport_mask[node] = 1;
				r.n0[node] = parameters.n0_bc;
				r.nplus[node] = parameters.nplus_bc;
			} else if (labels[node] >= 2) {
				r.pressure_mask[node] = 1;
			}
		}
	std::set<int> configured;
	for (const auto& rule : configuration.boundaries) {
		configured.insert(rule.label);
		bool found = false;
		for (size_t node = 0; node < nodes; ++node) {
			if (labels[node] != rule.label) continue;
			found = true;
			clear(node);
			if (rule.type == "wall") {
				r.velocity_mask[node] = 1;
				if (rule.has_velocity) for (int d = 0; d < 3; ++d) r.velocity[3*node+d] = rule.velocity[d];
			} else if (rule.type == "inlet") {
				r.velocity_mask[node] = 1;
				if (rule.has_velocity) {
					for (int d = 0; d < 3; ++d) r.velocity[3*node+d] = rule.velocity[d];
				} else {
					const double scale = rule.has_velocity_scale ? rule.velocity_scale : parameters.vplus;
					for (int d = 0; d < 3; ++d) r.velocity[3*node+d] = scale*reference_velocity[node][d];
				}
				r.transport_mask[node] = 1;
				r.n0[node] = rule.has_transport ? rule.n0 : parameters.n0_bc;
				r.nplus[node] = rule.has_transport ? rule.nplus : parameters.nplus_bc;
			} else if (rule.type == "outlet") {
				r.pressure_mask[node] = 1;
				r.pressure[node] = rule.has_pressure ? rule.pressure : 0.0;
			}
		}
		if (!found)
			Fail(-4, "case_config.json boundary label "+std::to_string(rule.label)+" is not present in controlmesh.vtk");
	}
	if (configuration.present && !configuration.inherit_legacy)
		for (int label : labels)
			if (label >= 0 && !configured.count(label))
				Fail(-4, "mesh boundary label "+std::to_string(label)
					+" has no case_config.json rule while inherit_legacy is false");
	for (size_t node = 0; node < nodes; ++node) {
		r.velocity_nodes += r.velocity_mask[node] == 1;
		r.pressure_nodes += r.pressure_mask[node] == 1;
		r.transport_nodes += r.transport_mask[node] == 1;
	}
	if (r.velocity_nodes == 0) Fail(-4, "case has no velocity boundary nodes");
	if (r.pressure_nodes == 0) Fail(-4, "case has no pressure boundary nodes");
	return r;
}

} // namespace tfiga
