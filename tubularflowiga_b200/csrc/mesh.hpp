// Host mesh (FlatMesh layout), .ntiga reader, block pattern, and the
// device-resident mesh with its per-element basis tables.
#pragma once

#include "common.hpp"
#include "kernels.cuh"

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace tfiga {

// Flattened mesh: solvers/cuda/include/DeviceMesh.hpp:16-57.
struct HostMesh {
	int64_t nodes = 0;
	std::vector<int32_t> element_offsets{0};
	std::vector<int32_t> connectivity;
	std::vector<int32_t> extraction_offsets{0};
	std::vector<uint8_t> extraction_columns;
	std::vector<double> extraction_values;
	std::vector<double> bezier_points;
	std::vector<int32_t> boundary_labels;      // 6 per element
	int32_t max_basis = 0;
	int64_t elements() const { return (int64_t)element_offsets.size()-1; }
	void Validate() const;
};

// Reads a v3/v4/v5 .ntiga database (iga::Database, IgaDatabase.hpp:64-161).
HostMesh ReadNtiga(const std::string& path);

// Node-graph block CSR (BlockPattern, BlockCsr.hpp:15-55).
struct HostPattern {
	std::vector<int32_t> row_offsets;
	std::vector<int32_t> columns;
	std::vector<int32_t> diagonal;
	int32_t max_row = 0;
};
HostPattern BuildPattern(const HostMesh& mesh);

// A labelled boundary face: element, local face (0..5), label.
struct BoundaryFace {
	int32_t element;
	int32_t face;
	int32_t label;
};

// Stable partition of the elements: those with at most 64 basis functions first, the others (up to
// 80) last, each group in its original order.  Returns the number of elements in the first group.
int64_t MoveLargeElementsLast(HostMesh& mesh);

// Device mesh.  Elements with 65..80 basis functions (from the reference spline extraction's
// extraordinary vertices) are moved behind the others at construction: the fast kernels run over
// regular_view() (the first regular_elements(), 64-wide tables phi / element_blocks), the
// large-element kernels over [large_first(), large_first() + large_count()) with 80-wide tables.
// Meshes without such elements keep their element order.
class Mesh {
public:
	explicit Mesh(HostMesh host);
	~Mesh();
	Mesh(const Mesh&) = delete;
	Mesh& operator=(const Mesh&) = delete;

	const HostMesh& host() const { return host_; }
	const HostPattern& pattern() const { return pattern_; }
	DeviceMeshView view() const { return view_; }
	DeviceMeshView regular_view() const { return regular_view_; }
	int64_t regular_elements() const { return regular_elements_; }
	int large_first() const { return (int)regular_elements_; }
	int large_count() const { return (int)(host_.elements()-regular_elements_); }
	const double* phi_large() const { return phi_large_.get(); }
	const int32_t* element_blocks_large() const { return element_blocks_large_.get(); }
	int face_stride() const { return face_stride_; }
	DevicePatternView pattern_view() const { return pattern_view_; }
	const double* phi() const { return phi_.get(); }
	// FP32 copy of the basis tables (operand staging of the tensor-core tangent), made on first use.
	const float* phi32();
	void ReleasePhi32();
	const double* qdata() const { return qdata_.get(); }
	const int32_t* element_blocks() const { return element_blocks_.get(); }
	const std::vector<BoundaryFace>& faces() const { return faces_; }
	const int32_t* face_element() const { return face_element_.get(); }
	const double* face_coef() const { return face_coef_.get(); }
	double min_detj() const { return min_detj_; }
	int64_t bad_samples() const { return bad_samples_; }
	int64_t device_bytes() const { return device_bytes_; }
	cudaStream_t stream() const { return stream_; }
	int64_t nodes() const { return host_.nodes; }

private:
	HostMesh host_;
	HostPattern pattern_;
	cudaStream_t stream_ = nullptr;
	DeviceArray<int32_t> element_offsets_, connectivity_, extraction_offsets_, row_offsets_, columns_, diagonal_,
		element_blocks_, face_element_, face_index_;
	DeviceArray<uint8_t> extraction_columns_;
	DeviceArray<double> extraction_values_, bezier_points_, phi_, qdata_, face_coef_, phi_large_;
	DeviceArray<int32_t> element_blocks_large_;
	DeviceArray<float> phi32_;
	DeviceMeshView view_, regular_view_;
	int64_t regular_elements_ = 0;
	int face_stride_ = kMaxBasis;
	DevicePatternView pattern_view_;
	std::vector<BoundaryFace> faces_;
	double min_detj_ = 0.0;
	int64_t bad_samples_ = 0;
	int64_t device_bytes_ = 0;
};

} // namespace tfiga
