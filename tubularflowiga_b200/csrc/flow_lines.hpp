// Flow-line preconditioner of the 2x2 transport system (an alternative to the reference's
// block-Jacobi): nodes are chained along the advection direction read from the matrix itself,
// and every chain's 2x2-block system is factored once (L is constant over the steps) and
// solved exactly inside the GMRES.
//
// Lines: node i links to the pattern neighbour j with the largest a_ij = L++_ji - L++_ij > 0,
// the antisymmetric part of the advected species' block (positive towards downstream); a node
// keeps only its strongest upstream link; chains start at nodes without an upstream link (then
// any closed loop becomes one line).  Factors: banded 2x2-block LU without pivoting; the band
// width of a line is the largest position difference of two coupled nodes on it; block (p, q)
// sits at row p, slot q - p + w, 4 doubles; after factoring the strict lower band holds L
// (unit diagonal), the strict upper band U, and the diagonal slots U_pp^{-1}.
#pragma once

#include <cstdint>
#include <vector>

namespace tfiga {

struct FlowLineFactors {
	std::vector<int32_t> line_offsets;   // [lines + 1]
	std::vector<int32_t> line_nodes;     // [nodes], chain order
	std::vector<int32_t> band_width;     // [lines]
	std::vector<int64_t> band_offsets;   // [lines], doubles into factors
	std::vector<double> factors;
	int32_t lines() const { return (int32_t)band_width.size(); }
};

// values: 2x2 blocks [blocks * 4] (row-major) on the pattern (row_offsets [nodes + 1], sorted columns).
FlowLineFactors BuildFlowLines(int32_t nodes, const int32_t* row_offsets, const int32_t* columns,
	const double* values);

} // namespace tfiga
