// 0D outlet models coupled inside the Newton loop, on the device.
//
// The reference couples its outlets on the host: after a Newton solve it
// copies the state back, integrates the outlet flows, evaluates each model
// (EvaluateOutletModel, include/OutletModel.hpp:70-90), relaxes the outlet
// pressures (RelaxOutletCoupling, :118-135) and uploads the new pressure
// traction (solvers/cuda/src/iga_cuda.cu:933-951, 1059-1085).  Here the
// update runs between Newton iterations without leaving the device: the face
// flows of the current state are summed per label, one warp evaluates every
// outlet model, applies the relaxed update (after the first Newton iteration of
// the step) while the largest change exceeds 1e-12 + 1e-9 max(1, max |P_eval|),
// and records whether the pressures now in use agree with their evaluation
// within the reference's tolerance 1e-8 + 1e-6 max(1, max |P_eval|) (the outlet
// half of the step's acceptance test); the per-face pressures and the traction
// rhs are then rebuilt from the outlet pressures.  The acceptance decision is
// the outer loop's; the update band is a thousand times narrower, so the
// accepted pressures are within 1e-9 of the fixed point rather than anywhere
// inside the reference's 1e-6 band (runs that differ only in precision then
// agree), while pressures that have settled stop moving and no longer reopen
// the Newton test.
// The host reads the acceptance flag together with the Newton norms it
// downloads anyway.
#include "common.hpp"
#include "kernels.cuh"

#include "../../include/tfiga.h"

namespace tfiga {
namespace {

__device__ __forceinline__ double WarpMax(double v)
{
	for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}

// One warp.  label_flow[slot] are the per-label boundary flows of the current state.
__global__ void __launch_bounds__(32) OutletUpdateKernel(int count, DeviceOutlet* __restrict__ outlets,
	const double* __restrict__ label_flow, double dt, double relaxation, int update, double* __restrict__ accepted,
	int* __restrict__ updates)
{
	const int lane = threadIdx.x;
	double change = 0.0, scale = 1.0;
	for (int i = lane; i < count; i += 32) {
		DeviceOutlet& o = outlets[i];
		const double q = o.slot >= 0 ? label_flow[o.slot] : 0.0;
		double p, pc;
		if (o.kind == TFIGA_OUTLET_RESISTANCE) {
			p = o.reference_pressure+o.resistance*q;
			pc = o.capacitor_pressure;
		} else {
			const double r = o.kind == TFIGA_OUTLET_RC ? o.resistance : o.distal;
			pc = (o.capacitance*o.capacitor_pressure/dt+q+o.reference_pressure/r)/(o.capacitance/dt+1.0/r);
			p = pc+(o.kind == TFIGA_OUTLET_RCR ? o.proximal*q : 0.0);
		}
		o.flow = q;
		o.evaluated = p;
		o.evaluated_capacitor = pc;
		change = fmax(change, fabs(p-o.pressure));
		scale = fmax(scale, fabs(p));
	}
	change = WarpMax(change);
	scale = WarpMax(scale);
	const double tolerance = 1e-8+1e-6*scale;
	const bool relax = update && change > 1e-12+1e-9*scale;
	double post = 0.0;
	for (int i = lane; i < count; i += 32) {
		DeviceOutlet& o = outlets[i];
		if (relax) o.pressure = (1.0-relaxation)*o.pressure+relaxation*o.evaluated;
		post = fmax(post, fabs(o.evaluated-o.pressure));
	}
	post = WarpMax(post);
	if (lane == 0) {
		*accepted = post <= tolerance ? 1.0 : 0.0;
		if (relax) ++*updates;
	}
}

// face_pressure[f] = the pressure of the outlet owning the face's label, else the fixed traction.
__global__ void FacePressureKernel(int faces, const int32_t* __restrict__ face_slot,
	const int32_t* __restrict__ slot_outlet, const double* __restrict__ base, const DeviceOutlet* __restrict__ outlets,
	double* __restrict__ face_pressure)
{
	const int f = blockIdx.x*blockDim.x+threadIdx.x;
	if (f >= faces) return;
	const int o = slot_outlet[face_slot[f]];
	face_pressure[f] = o >= 0 ? outlets[o].pressure : base[f];
}

} // namespace

void LaunchOutletUpdate(int count, DeviceOutlet* outlets, const double* label_flow, double dt, double relaxation,
	bool update, double* accepted, int* updates, cudaStream_t stream)
{
	OutletUpdateKernel<<<1, 32, 0, stream>>>(count, outlets, label_flow, dt, relaxation, update ? 1 : 0, accepted,
		updates);
	LaunchCheck("OutletUpdateKernel");
}

void LaunchFacePressures(int faces, const int32_t* face_slot, const int32_t* slot_outlet, const double* base,
	const DeviceOutlet* outlets, double* face_pressure, cudaStream_t stream)
{
	if (faces == 0) return;
	FacePressureKernel<<<(faces+255)/256, 256, 0, stream>>>(faces, face_slot, slot_outlet, base, outlets,
		face_pressure);
	LaunchCheck("FacePressureKernel");
}

} // namespace tfiga
