// Host mesh I/O and the device-resident mesh.
#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>

namespace tfiga {

namespace {

constexpr char kMagic[8] = {'N', 'T', 'I', 'G', 'A', 'D', 'B', '2'};

template <class T>
void ReadValue(std::istream& in, T& value)
{
	in.read(reinterpret_cast<char*>(&value), sizeof(T));
	if (!in) Fail(-4, "binary database is truncated");
}

} // namespace

void HostMesh::Validate() const
{
	const int64_t E = elements();
	if (nodes <= 0 || E <= 0) Fail(-1, "mesh needs at least one node and one element");
	if (nodes > std::numeric_limits<int32_t>::max()/4) Fail(-7, "node count exceeds the int32 field index range");
	if ((int64_t)connectivity.size() != element_offsets.back()) Fail(-1, "connectivity size mismatch");
	if ((int64_t)extraction_offsets.size() != element_offsets.back()+1) Fail(-1, "extraction offsets size mismatch");
	if ((int64_t)extraction_columns.size() != extraction_offsets.back()
		|| extraction_values.size() != extraction_columns.size())
		Fail(-1, "extraction arrays size mismatch");
	if ((int64_t)bezier_points.size() != E*192) Fail(-1, "bezier point array size mismatch");
	if ((int64_t)boundary_labels.size() != E*6) Fail(-1, "boundary label array size mismatch");
	for (int64_t e = 0; e < E; ++e)
		if (element_offsets[e+1] <= element_offsets[e]) Fail(-4, "element without basis functions");
	for (int32_t node : connectivity)
		if (node < 0 || node >= nodes) Fail(-4, "connectivity references an invalid node");
	for (uint8_t c : extraction_columns)
		if (c >= 64) Fail(-4, "invalid extraction column");
}

HostMesh ReadNtiga(const std::string& path)
{
	std::ifstream in(path, std::ios::binary);
	if (!in) Fail(-3, "cannot open database: "+path);
	char magic[8];
	in.read(magic, 8);
	uint32_t version = 0, ranks = 0, bezier = 0, reserved = 0;
	uint64_t elements = 0, nodes = 0, rank_index = 0;
	ReadValue(in, version); ReadValue(in, ranks); ReadValue(in, elements); ReadValue(in, nodes);
	ReadValue(in, bezier); ReadValue(in, reserved); ReadValue(in, rank_index);
	if (std::memcmp(magic, kMagic, 8) != 0) Fail(-4, "not a supported .ntiga database");
	if (version != 3 && version != 4 && version != 5) Fail(-4, "unsupported database version");
	if (version >= 5) {
		double transform[5];
		for (double& v : transform) ReadValue(in, v);
		if (!(transform[3] > 0.0) || !(transform[4] > 0.0)) Fail(-4, "invalid database geometry transform");
	}
	if (bezier != 64) Fail(-4, "unsupported Bezier point count");
	if (nodes == 0 || rank_index == 0) Fail(-4, "invalid database ownership index");
	if (elements > (uint64_t)std::numeric_limits<int32_t>::max()) Fail(-7, "too many elements");
	std::vector<uint64_t> offsets(elements+1);
	in.read(reinterpret_cast<char*>(offsets.data()), (std::streamsize)(offsets.size()*sizeof(uint64_t)));
	if (!in || offsets.front() >= offsets.back()) Fail(-4, "invalid database offsets");
	HostMesh mesh;
	mesh.nodes = (int64_t)nodes;
	mesh.bezier_points.resize(elements*192);
	mesh.boundary_labels.assign(elements*6, -1);
	std::vector<char> record;
	for (uint64_t e = 0; e < elements; ++e) {
		in.clear();
		in.seekg((std::streamoff)offsets[e]);
		uint64_t id = 0; int32_t type = 0, owner = 0; uint32_t nen = 0;
		ReadValue(in, id); ReadValue(in, type); ReadValue(in, owner); ReadValue(in, nen);
		if (version >= 4)
			in.read(reinterpret_cast<char*>(mesh.boundary_labels.data()+6*e), 6*sizeof(int32_t));
		if (nen == 0 || nen > 4096) Fail(-4, "invalid element basis count");
		mesh.max_basis = std::max<int32_t>(mesh.max_basis, (int32_t)nen);
		const size_t start = mesh.connectivity.size();
		mesh.connectivity.resize(start+nen);
		in.read(reinterpret_cast<char*>(mesh.connectivity.data()+start), (std::streamsize)(nen*sizeof(int32_t)));
		for (uint32_t a = 0; a < nen; ++a) {
			uint8_t nonzeros = 0;
			ReadValue(in, nonzeros);
			for (uint8_t j = 0; j < nonzeros; ++j) {
				uint8_t column = 0; double value = 0.0;
				ReadValue(in, column); ReadValue(in, value);
				if (column >= 64) Fail(-4, "invalid extraction column");
				if (value == 0.0) continue;
				mesh.extraction_columns.push_back(column);
				mesh.extraction_values.push_back(value);
			}
			mesh.extraction_offsets.push_back((int32_t)mesh.extraction_values.size());
		}
		in.read(reinterpret_cast<char*>(mesh.bezier_points.data()+192*e), 192*sizeof(double));
		if (!in) Fail(-4, "element record is truncated");
		mesh.element_offsets.push_back((int32_t)mesh.connectivity.size());
	}
	mesh.Validate();
	return mesh;
}

HostPattern BuildPattern(const HostMesh& mesh)
{
	const int64_t n = mesh.nodes, E = mesh.elements();
	// node -> incident elements
	std::vector<int64_t> start(n+1, 0);
	for (int32_t node : mesh.connectivity) ++start[node+1];
	for (int64_t i = 0; i < n; ++i) start[i+1] += start[i];
	std::vector<int32_t> incident(start[n]);
	std::vector<int64_t> fill(start.begin(), start.end()-1);
	for (int64_t e = 0; e < E; ++e)
		for (int32_t k = mesh.element_offsets[e]; k < mesh.element_offsets[e+1]; ++k)
			incident[fill[mesh.connectivity[k]]++] = (int32_t)e;
	HostPattern p;
	p.row_offsets.resize(n+1);
	p.diagonal.assign(n, -1);
	std::vector<int32_t> stamp(n, -1), row;
	int64_t total = 0;
	p.row_offsets[0] = 0;
	for (int64_t node = 0; node < n; ++node) {
		row.clear();
		for (int64_t k = start[node]; k < start[node+1]; ++k) {
			const int32_t e = incident[k];
			for (int32_t j = mesh.element_offsets[e]; j < mesh.element_offsets[e+1]; ++j) {
				const int32_t c = mesh.connectivity[j];
				if (stamp[c] != (int32_t)node) { stamp[c] = (int32_t)node; row.push_back(c); }
			}
		}
		std::sort(row.begin(), row.end());
		const auto it = std::lower_bound(row.begin(), row.end(), (int32_t)node);
		if (it == row.end() || *it != node) Fail(-4, "block pattern is missing a diagonal entry");
		p.diagonal[node] = (int32_t)(total+(it-row.begin()));
		p.columns.insert(p.columns.end(), row.begin(), row.end());
		total += (int64_t)row.size();
		if (total > std::numeric_limits<int32_t>::max()) Fail(-7, "block CSR has more than INT_MAX blocks");
		p.row_offsets[node+1] = (int32_t)total;
		p.max_row = std::max<int32_t>(p.max_row, (int32_t)row.size());
	}
	return p;
}

int64_t MoveLargeElementsLast(HostMesh& m)
{
	const int64_t E = m.elements();
	std::vector<int64_t> order;
	order.reserve((size_t)E);
	for (int64_t e = 0; e < E; ++e)
		if (m.element_offsets[e+1]-m.element_offsets[e] <= kMaxBasis) order.push_back(e);
	const int64_t regular = (int64_t)order.size();
	if (regular == E) return E;
	for (int64_t e = 0; e < E; ++e)
		if (m.element_offsets[e+1]-m.element_offsets[e] > kMaxBasis) order.push_back(e);
	HostMesh out;
	out.nodes = m.nodes;
	out.max_basis = m.max_basis;
	out.connectivity.reserve(m.connectivity.size());
	out.extraction_offsets.reserve(m.extraction_offsets.size());
	out.extraction_columns.reserve(m.extraction_columns.size());
	out.extraction_values.reserve(m.extraction_values.size());
	out.bezier_points.reserve(m.bezier_points.size());
	out.boundary_labels.reserve(m.boundary_labels.size());
	for (const int64_t e : order) {
		for (int32_t k = m.element_offsets[e]; k < m.element_offsets[e+1]; ++k) {
			out.connectivity.push_back(m.connectivity[k]);
			const int32_t lo = m.extraction_offsets[k], hi = m.extraction_offsets[k+1];
			out.extraction_columns.insert(out.extraction_columns.end(), m.extraction_columns.begin()+lo,
				m.extraction_columns.begin()+hi);
			out.extraction_values.insert(out.extraction_values.end(), m.extraction_values.begin()+lo,
				m.extraction_values.begin()+hi);
			out.extraction_offsets.push_back((int32_t)out.extraction_values.size());
		}
		out.element_offsets.push_back((int32_t)out.connectivity.size());
		out.bezier_points.insert(out.bezier_points.end(), m.bezier_points.begin()+192*e,
			m.bezier_points.begin()+192*(e+1));
		out.boundary_labels.insert(out.boundary_labels.end(), m.boundary_labels.begin()+6*e,
			m.boundary_labels.begin()+6*(e+1));
	}
	m = std::move(out);
	return regular;
}

Mesh::Mesh(HostMesh host) : host_(std::move(host))
{
	RequireDevice();
	host_.Validate();
	if (host_.max_basis > kMaxBasisLarge)
		Fail(-7, "CUDA kernels support at most 80 basis functions per element (max_basis="
			+std::to_string(host_.max_basis)+")");
	regular_elements_ = MoveLargeElementsLast(host_);
	face_stride_ = host_.max_basis > kMaxBasis ? kMaxBasisLarge : kMaxBasis;
	pattern_ = BuildPattern(host_);
	CudaCheck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "mesh stream");
	const int64_t E = host_.elements();
	auto up = [&](auto& dev, const auto& vec) {
		dev.Allocate(vec.size());
		dev.Upload(vec.data(), vec.size(), stream_);
	};
	up(element_offsets_, host_.element_offsets);
	up(connectivity_, host_.connectivity);
	up(extraction_offsets_, host_.extraction_offsets);
	up(extraction_columns_, host_.extraction_columns);
	up(extraction_values_, host_.extraction_values);
	up(bezier_points_, host_.bezier_points);
	up(row_offsets_, pattern_.row_offsets);
	up(columns_, pattern_.columns);
	up(diagonal_, pattern_.diagonal);
	view_ = {(int)host_.nodes, (int)E, element_offsets_.get(), connectivity_.get(), extraction_offsets_.get(),
		extraction_columns_.get(), extraction_values_.get(), bezier_points_.get()};
	pattern_view_ = {(int)host_.nodes, (long long)pattern_.columns.size(), row_offsets_.get(), columns_.get(),
		diagonal_.get()};
	regular_view_ = view_;
	regular_view_.elements = (int)regular_elements_;
	const int64_t large = E-regular_elements_;
	phi_.Allocate((size_t)regular_elements_*kFeatures*kQuad*kMaxBasis);
	qdata_.Allocate((size_t)E*kQuad*kQData);
	LaunchBuildBasis(regular_view_, phi_.get(), qdata_.get(), stream_);
	element_blocks_.Allocate((size_t)regular_elements_*kMaxBasis*kMaxBasis);
	LaunchElementBlocks(regular_view_, pattern_view_, element_blocks_.get(), stream_);
	if (large > 0) {
		phi_large_.Allocate((size_t)large*kFeatures*kQuad*kMaxBasisLarge);
		LaunchBuildBasisLarge(view_, (int)regular_elements_, (int)large, phi_large_.get(), qdata_.get(), stream_);
		element_blocks_large_.Allocate((size_t)large*kMaxBasisLarge*kMaxBasisLarge);
		LaunchElementBlocksLarge(view_, pattern_view_, (int)regular_elements_, (int)large,
			element_blocks_large_.get(), stream_);
	}
	// Labelled boundary faces in element order.
	std::vector<int32_t> fe, fi;
	for (int64_t e = 0; e < E; ++e)
		for (int f = 0; f < 6; ++f) {
			const int32_t label = host_.boundary_labels[6*e+f];
			if (label < 0) continue;
			faces_.push_back({(int32_t)e, f, label});
			fe.push_back((int32_t)e);
			fi.push_back(f);
		}
	if (!faces_.empty()) {
		up(face_element_, fe);
		up(face_index_, fi);
		face_coef_.Allocate(faces_.size()*face_stride_*3);
		LaunchFaceCoefficients(view_, (int)faces_.size(), face_element_.get(), face_index_.get(), face_coef_.get(),
			face_stride_, stream_);
	}
	std::vector<double> qd((size_t)E*kQuad*kQData);
	qdata_.Download(qd.data(), qd.size(), stream_);
	CudaCheck(cudaStreamSynchronize(stream_), "mesh setup");
	min_detj_ = std::numeric_limits<double>::infinity();
	for (size_t k = 0; k < (size_t)E*kQuad; ++k) {
		const double det = qd[k*kQData+9];
		min_detj_ = std::min(min_detj_, det);
		if (!std::isfinite(det) || det <= 0.0 || qd[k*kQData] == 0.0) ++bad_samples_;
	}
	device_bytes_ = (int64_t)(element_offsets_.bytes()+connectivity_.bytes()+extraction_offsets_.bytes()
		+extraction_columns_.bytes()+extraction_values_.bytes()+bezier_points_.bytes()+row_offsets_.bytes()
		+columns_.bytes()+diagonal_.bytes()+phi_.bytes()+qdata_.bytes()+element_blocks_.bytes()
		+face_element_.bytes()+face_index_.bytes()+face_coef_.bytes()+phi_large_.bytes()
		+element_blocks_large_.bytes());
}

const float* Mesh::phi32()
{
	if (phi32_.get() == nullptr) {
		const size_t count = (size_t)regular_elements_*kFeatures*kQuad*kMaxBasis;
		phi32_.Allocate(count);
		LaunchToFloatPointPairs((long long)regular_elements_*kFeatures, phi_.get(), phi32_.get(), stream_);
		CudaCheck(cudaStreamSynchronize(stream_), "FP32 basis tables");
		device_bytes_ += (int64_t)phi32_.bytes();
	}
	return phi32_.get();
}

void Mesh::ReleasePhi32()
{
	if (phi32_.get() == nullptr) return;
	device_bytes_ -= (int64_t)phi32_.bytes();
	phi32_.Release();
}

Mesh::~Mesh()
{
	if (stream_) cudaStreamDestroy(stream_);
}

} // namespace tfiga
