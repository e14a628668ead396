// Learned stage of the FGMRES preconditioner: a message-passing network over
// the element face-adjacency graph that maps a residual to a correction,
// z = M_AMG(r) + N(D^{-1} r).  FGMRES accepts any preconditioner that may
// change from one iteration to the next, and it still drives the FP64 true
// residual to the same tolerance, so the network only changes the iteration
// count; the AMG-only solve stays available and is the reference for its
// effect.
//
// Network (hidden width 64, L message-passing layers; the definition is the
// CPU oracle's, oracle/learned_oracle.py):
//   X[e, 4a + c] = s_in[c] x[node(e, a), c]                 gather, E x 256
//   h0 = act(X Win^T + bin)                                 encode
//   h_{l+1} = h_l + act(h_l Ws_l^T + mean_nb(h_l) Wn_l^T + b_l)
//   y = h_L Wout^T + bout                                   decode, E x 256
//   o[node, c] = s_out[c] / deg(node) sum_{(e, a) -> node} y[e, 4a + c]
//   act(v) = max(v, 0.1 v); the linear variant uses act(v) = v and zero biases
// Inference reads BF16 weights and accumulates in FP32; training keeps FP32
// master weights, runs the hand-written backward kernels, reduces the weight
// gradients in a fixed order (deterministic) and takes Adam steps.
// Training pairs are produced by the solver itself: each solved Newton system
// J delta = b gives x = D^{-1} b / |b| with the AMG's residual
// q = (b - J M_AMG(b)) / |b|, and the flexible GMRES gives x = D^{-1} w_j,
// q = w_j - A M_AMG(w_j) from w_j = A z_j on every eighth iteration, which
// covers the vectors the stage is applied to.  The loss is the residual one,
// sum ((A N(x)) - q)^2 weighted per field, whose gradient goes back through
// A^T; the solution-space loss (N(x) against delta - M_AMG) is kept for the
// oracle checks.
#pragma once

#include "common.hpp"
#include "kernels.cuh"

#include <cuda_bf16.h>
#include <vector>

namespace tfiga {

class Mesh;

class LearnedPreconditioner {
public:
	static constexpr int kHidden = 64;
	static constexpr int kInputs = 256;      // 64 local basis functions x 4 fields
	static constexpr int kMaxLayers = 8;
	static constexpr int kPairCapacity = 128;   // ring of training pairs

	// linear: identity activation and biases held at zero, so the stage is a fixed linear operator.
	LearnedPreconditioner(const Mesh& mesh, int layers, unsigned long long seed, cudaStream_t stream,
		bool linear = false);
	bool linear() const { return linear_; }
	int layers() const { return layers_; }
	long long parameter_count() const { return params_; }
	long long elements() const { return elements_; }
	int nodes() const { return nodes_; }
	const std::vector<int32_t>& neighbours() const { return nb_host_; }

	void SetParameters(const float* host);
	void GetParameters(float* host) const;
	// Per-field input / output scales and loss weights.
	void SetScales(const double in[4], const double out[4], const double weights[4]);
	void GetScales(double in[4], double out[4], double weights[4]) const;

	// Inference with the BF16 weights: z (4n, FP64) += N(x); kernels return at once when *stop is set.
	void Apply(const double* x, double* z, const int* stop);
	// FP32 forward; o (4n, FP64) is written.
	void Forward(const double* x, double* o);
	// FP32 forward + backward of the loss against target t; returns the loss, gradient on the device.
	double LossAndGradient(const double* x, const double* target);
	const float* gradient() const { return grad_.get(); }

	// Training data: copies a pair (device vectors of 4n doubles) into the pair store.
	void AddPair(const double* x, const double* target);
	// The pair of one solved Newton system J delta = b, scaled by 1 / |b|: x = D^{-1} b,
	// t = delta - M_AMG(b), q = b - J M_AMG(b).
	void AddSolvedPair(const double* dinv_b, const double* delta, const double* amg_b, const double* b,
		const double* a_amg_b, double b_norm);
	// A flexible-GMRES pair, w = A z exactly: x = D^{-1} w, t = z - M_AMG(w), q = w - A M_AMG(w)
	// (skipped when *stop).
	void AddKrylovPair(const double* dinv_w, const double* z, const double* amg_w, const double* w,
		const double* a_amg_w, const int* stop);
	// Operator of the residual loss (the current Jacobian; FP32 or FP64 values).  With an operator the
	// training loss is sum w_c ((A N(x))_c - q_c)^2 / (4n): the stage is fitted to cancel the residual the
	// AMG leaves, which is what the FGMRES sees; without one it is the solution-space loss against t.
	void SetOperator(const DevicePatternView& pattern, const float* values32, const double* values64);
	bool has_operator() const { return op32_ != nullptr || op64_ != nullptr; }
	double ResidualLossAndGradient(const double* x, const double* q);
	int pair_count() const { return pair_count_; }
	// Size of the pair store (before the first pair; default kPairCapacity).
	void SetCapacity(int capacity);
	int pair_capacity() const { return capacity_; }
	// Scales from the stored pairs (RMS per field; loss weights 1/RMS^2 of the target).
	void FitScales();
	// `steps` Adam steps cycling over the stored pairs; returns the mean loss of the last pass.
	double Train(int steps, double learning_rate);
	// Mean loss over the stored pairs (FP32 forward).
	double EvaluatePairs();
	// Least-squares output gain over the stored pairs, gain = <o, t>_w / <o, o>_w (clamped at 0),
	// folded into the output scales so that the stage can only lower the weighted training loss;
	// returns the gain.
	double FitGain();

	cudaStream_t stream() const { return stream_; }

private:
	void AllocatePairs();
	void ApplyOperator(const double* in, double* out);
	void Backward();
	double PairLoss(int p, bool gradient);
	void Gather(const double* x);
	void ForwardLayers(bool keep);
	void SyncBf16();
	float* param(const char* name, int layer = 0);

	cudaStream_t stream_;
	int layers_, nodes_;
	long long elements_, params_;
	std::vector<int32_t> nb_host_;
	DeviceArray<int32_t> conn_, nb_, node_offsets_, node_entries_;
	DeviceArray<float> theta_, grad_, adam_m_, adam_v_, partial_;
	DeviceArray<__nv_bfloat16> theta16_;
	DeviceArray<float> X_, z0_, y_, dy_, dh_, dprev_, dm_, dz0_, node_do_;
	std::vector<DeviceArray<float>> h_, m_, z_, dz_;
	DeviceArray<double> o_, scales_, loss_partial_, loss_;
	DeviceArray<double> pairs_x_, pairs_t_, pairs_q_;
	DevicePatternView op_;
	const float* op32_ = nullptr;
	const double* op64_ = nullptr;
	DeviceArray<double> ro_, g_, atg_;
	double scale_in_[4] = {1, 1, 1, 1}, scale_out_[4] = {1, 1, 1, 1}, weight_[4] = {1, 1, 1, 1};
	int pair_count_ = 0, capacity_ = 0, next_pair_ = 0, requested_capacity_ = kPairCapacity;
	long long adam_steps_ = 0;
	bool bf16_dirty_ = true;
	bool linear_ = false;
	float slope_ = 0.1f;
};

} // namespace tfiga
