// Host construction of the flow-line preconditioner (once per transport run).
#include "flow_lines.hpp"

#include "common.hpp"

#include <algorithm>
#include <cstdlib>
#include <cstring>

namespace tfiga {
namespace {

// Block index of (row, column) in the sorted block row, or -1.
int64_t FindBlock(const int32_t* row_offsets, const int32_t* columns, int32_t row, int32_t column)
{
	const int32_t* first = columns+row_offsets[row];
	const int32_t* last = columns+row_offsets[row+1];
	const int32_t* it = std::lower_bound(first, last, column);
	return it != last && *it == column ? (int64_t)(it-columns) : -1;
}

void Inverse2(const double* a, double* r)
{
	const double det = a[0]*a[3]-a[1]*a[2];
	if (!(det != 0.0)) Fail(-6, "flow-line factorization met a singular 2x2 pivot");
	r[0] = a[3]/det; r[1] = -a[1]/det; r[2] = -a[2]/det; r[3] = a[0]/det;
}

void Multiply2(const double* a, const double* b, double* r)
{
	r[0] = a[0]*b[0]+a[1]*b[2]; r[1] = a[0]*b[1]+a[1]*b[3];
	r[2] = a[2]*b[0]+a[3]*b[2]; r[3] = a[2]*b[1]+a[3]*b[3];
}

} // namespace

FlowLineFactors BuildFlowLines(int32_t nodes, const int32_t* row_offsets, const int32_t* columns,
	const double* values)
{
	if (nodes <= 0) Fail(-1, "flow lines need nodes");
	std::vector<int32_t> down((size_t)nodes, -1), up((size_t)nodes, -1);
	std::vector<double> down_value((size_t)nodes, 0.0), up_value((size_t)nodes, 0.0);
	for (int32_t i = 0; i < nodes; ++i)
		for (int32_t b = row_offsets[i]; b < row_offsets[i+1]; ++b) {
			const int32_t j = columns[b];
			if (j == i) continue;
			const int64_t t = FindBlock(row_offsets, columns, j, i);
			const double a = (t >= 0 ? values[t*4+3] : 0.0)-values[(size_t)b*4+3];
			if (a > down_value[i]) { down_value[i] = a; down[i] = j; }
		}
	for (int32_t i = 0; i < nodes; ++i) {
		const int32_t j = down[i];
		if (j >= 0 && (up[j] < 0 || down_value[i] > up_value[j])) { up[j] = i; up_value[j] = down_value[i]; }
	}
	for (int32_t i = 0; i < nodes; ++i)
		if (down[i] >= 0 && up[down[i]] != i) down[i] = -1;

	FlowLineFactors f;
	f.line_offsets.push_back(0);
	f.line_nodes.reserve((size_t)nodes);
	std::vector<char> seen((size_t)nodes, 0);
	auto chain = [&](int32_t head) {
		for (int32_t i = head; i >= 0 && !seen[i]; i = down[i]) { seen[i] = 1; f.line_nodes.push_back(i); }
		f.line_offsets.push_back((int32_t)f.line_nodes.size());
	};
	for (int32_t h = 0; h < nodes; ++h)
		if (up[h] < 0 && !seen[h]) chain(h);
	for (int32_t h = 0; h < nodes; ++h)
		if (!seen[h]) chain(h);
	const int32_t lines = (int32_t)f.line_offsets.size()-1;

	std::vector<int32_t> pos((size_t)nodes), line_of((size_t)nodes);
	for (int32_t l = 0; l < lines; ++l)
		for (int32_t k = f.line_offsets[l]; k < f.line_offsets[l+1]; ++k) {
			pos[f.line_nodes[k]] = k-f.line_offsets[l];
			line_of[f.line_nodes[k]] = l;
		}
	f.band_width.assign((size_t)lines, 0);
	f.band_offsets.assign((size_t)lines, 0);
	int64_t total = 0;
	for (int32_t l = 0; l < lines; ++l) {
		int32_t w = 0;
		for (int32_t k = f.line_offsets[l]; k < f.line_offsets[l+1]; ++k) {
			const int32_t i = f.line_nodes[k];
			for (int32_t b = row_offsets[i]; b < row_offsets[i+1]; ++b)
				if (line_of[columns[b]] == l) w = std::max(w, std::abs(pos[columns[b]]-pos[i]));
		}
		f.band_width[l] = w;
		f.band_offsets[l] = total;
		total += 4LL*(f.line_offsets[l+1]-f.line_offsets[l])*(2*w+1);
	}
	f.factors.assign((size_t)total, 0.0);
	for (int32_t l = 0; l < lines; ++l) {
		const int32_t m = f.line_offsets[l+1]-f.line_offsets[l], w = f.band_width[l], s = 2*w+1;
		double* B = f.factors.data()+f.band_offsets[l];
		for (int32_t k = f.line_offsets[l]; k < f.line_offsets[l+1]; ++k) {
			const int32_t i = f.line_nodes[k], p = pos[i];
			for (int32_t b = row_offsets[i]; b < row_offsets[i+1]; ++b)
				if (line_of[columns[b]] == l)
					std::memcpy(B+4*((size_t)p*s+(pos[columns[b]]-p+w)), values+(size_t)b*4, 4*sizeof(double));
		}
		for (int32_t p = 0; p < m; ++p) {
			double dinv[4], lrp[4], t[4];
			Inverse2(B+4*((size_t)p*s+w), dinv);
			for (int32_t r = p+1; r <= p+w && r < m; ++r) {
				double* Arp = B+4*((size_t)r*s+(p-r+w));
				Multiply2(Arp, dinv, lrp);
				std::memcpy(Arp, lrp, sizeof(lrp));
				for (int32_t c = p+1; c <= p+w && c < m; ++c) {
					double* Arc = B+4*((size_t)r*s+(c-r+w));
					Multiply2(lrp, B+4*((size_t)p*s+(c-p+w)), t);
					for (int e = 0; e < 4; ++e) Arc[e] -= t[e];
				}
			}
			std::memcpy(B+4*((size_t)p*s+w), dinv, sizeof(dinv));
		}
	}
	return f;
}

} // namespace tfiga
