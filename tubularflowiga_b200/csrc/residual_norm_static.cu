// tfiga_block_residual_norm_static: ||b - A x||_2 over a 4x4 block-CSR
// matrix, computed without allocating anything.
//
// Every other entry point of this library works through a handle whose
// create call allocates its device buffers.  This one serves callers that
// must not allocate at call time (a host loop that pre-sizes everything, or a
// caller whose memory pool forbids new device allocations after setup): its
// only scratch -- one partial sum of squares per CTA of the first kernel -- is
// the file-scope device array below, whose address is looked up once per
// device with cudaGetSymbolAddress.
//
// Limits and rules, stated in the header as well:
//  * at most kMaxPartials CTAs of 8 block rows, i.e. nodes <= kMaxNodes; a
//    larger system is rejected with TFIGA_E_UNSUPPORTED before any launch;
//  * nothing has to start at zero: every CTA overwrites its own partial slot
//    and the finalize kernel reads exactly the slots written by this call;
//  * the scratch is shared by every call on a device, so two calls whose
//    kernels overlap (different streams, or different host threads) race on
//    it; calls must be ordered on one stream or otherwise serialized;
//  * the first call on each device performs the symbol lookup, so make that
//    first call before any stream capture on that device begins; the address
//    is cached with the unique id of the context it was looked up in, so a
//    call made after cudaDeviceReset (a new primary context) looks it up again
//    instead of using the stale address.
// The two kernels sum in a fixed order, so equal inputs give bitwise equal
// norms.
#include "common.hpp"

#include "../../include/tfiga.h"

#include <cuda.h>

#include <mutex>

namespace tfiga {
void RecordLastError(const char* message);
}

namespace {

constexpr int kRowsPerCta = 8;                          // one warp per block row
constexpr int kMaxPartials = 32768;                     // 256 KiB of FP64 partial sums
constexpr int kMaxNodes = kMaxPartials*kRowsPerCta;     // 262,144 block rows
constexpr int kMaxDevices = 64;
constexpr int kFinalizeThreads = 1024;

static __device__ __align__(256) double g_partials[kMaxPartials];

// Per device: the scratch address and the id of the context it belongs to (0: none yet).
struct ScratchEntry {
	unsigned long long context_id = 0;
	double* address = nullptr;
};
ScratchEntry g_scratch[kMaxDevices];
std::mutex g_scratch_mutex;

__global__ void __launch_bounds__(256) ResidualPartialKernel(int nodes, const int32_t* __restrict__ row_offsets,
	const int32_t* __restrict__ columns, const double* __restrict__ values, const double* __restrict__ x,
	const double* __restrict__ b, double* __restrict__ partials)
{
	__shared__ double warp_sums[kRowsPerCta];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int row = blockIdx.x*kRowsPerCta+warp;
	double sq = 0.0;
	if (row < nodes) {
		// lane = 4*slot + r: row r of blocks slot, slot+8, ... (coalesced 128-byte block loads)
		const int r = lane & 3, slot = lane >> 2;
		double sum = 0.0;
		const int lo = row_offsets[row], hi = row_offsets[row+1];
		for (int k = lo+slot; k < hi; k += 8) {
			const double2* a = reinterpret_cast<const double2*>(values+(size_t)k*16+r*4);
			const double2 a01 = __ldg(a), a23 = __ldg(a+1);
			const double2* xv = reinterpret_cast<const double2*>(x+4*(size_t)columns[k]);
			const double2 x01 = __ldg(xv), x23 = __ldg(xv+1);
			sum = fma(a01.x, x01.x, sum); sum = fma(a01.y, x01.y, sum);
			sum = fma(a23.x, x23.x, sum); sum = fma(a23.y, x23.y, sum);
		}
		sum += __shfl_xor_sync(0xffffffffu, sum, 4);
		sum += __shfl_xor_sync(0xffffffffu, sum, 8);
		sum += __shfl_xor_sync(0xffffffffu, sum, 16);
		const double res = b[4*(size_t)row+r]-sum;
		sq = lane < 4 ? res*res : 0.0;
	}
	sq += __shfl_xor_sync(0xffffffffu, sq, 1);
	sq += __shfl_xor_sync(0xffffffffu, sq, 2);
	if (lane == 0) warp_sums[warp] = sq;
	__syncthreads();
	if (threadIdx.x == 0) {
		double total = 0.0;
		for (int w = 0; w < kRowsPerCta; ++w) total += warp_sums[w];
		partials[blockIdx.x] = total;
	}
}

__global__ void __launch_bounds__(kFinalizeThreads) ResidualFinalizeKernel(int count,
	const double* __restrict__ partials, double* __restrict__ norm)
{
	__shared__ double s[kFinalizeThreads];
	double sum = 0.0;
	for (int i = threadIdx.x; i < count; i += kFinalizeThreads) sum += partials[i];
	s[threadIdx.x] = sum;
	__syncthreads();
	for (int h = kFinalizeThreads/2; h > 0; h >>= 1) {
		if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x+h];
		__syncthreads();
	}
	if (threadIdx.x == 0) *norm = sqrt(s[0]);
}

int Reject(int status, const char* message)
{
	tfiga::RecordLastError(message);
	return status;
}

// Driver entry points for the current context and its process-unique id, taken through the
// runtime so the library needs no link against libcuda.
using CtxGetCurrent = CUresult (*)(CUcontext*);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long*);

bool DriverEntryPoints(CtxGetCurrent* get_current, CtxGetId* get_id)
{
	static CtxGetCurrent current = nullptr;
	static CtxGetId id = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void* f = nullptr;
		cudaDriverEntryPointQueryResult found{};
		if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &found) == cudaSuccess
			&& found == cudaDriverEntryPointSuccess)
			current = reinterpret_cast<CtxGetCurrent>(f);
		f = nullptr;
		if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &found) == cudaSuccess
			&& found == cudaDriverEntryPointSuccess)
			id = reinterpret_cast<CtxGetId>(f);
	});
	*get_current = current;
	*get_id = id;
	return current != nullptr && id != nullptr;
}

// Id of the calling thread's current context, or 0 when none is current (or it is gone).
unsigned long long CurrentContextId(CtxGetCurrent get_current, CtxGetId get_id)
{
	CUcontext context = nullptr;
	unsigned long long id = 0;
	if (get_current(&context) != CUDA_SUCCESS || context == nullptr || get_id(context, &id) != CUDA_SUCCESS) return 0;
	return id;
}

// Address of this device's scratch array, looked up once per device and context: the cached
// address is reused only while the context it was looked up in is still the current one.
int Scratch(double** out)
{
	int device = 0;
	if (cudaGetDevice(&device) != cudaSuccess) return Reject(TFIGA_E_CUDA, "cudaGetDevice failed");
	if (device < 0 || device >= kMaxDevices) return Reject(TFIGA_E_UNSUPPORTED, "device ordinal above 63");
	CtxGetCurrent get_current = nullptr;
	CtxGetId get_id = nullptr;
	if (!DriverEntryPoints(&get_current, &get_id))
		return Reject(TFIGA_E_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId unavailable");
	unsigned long long context_id = CurrentContextId(get_current, get_id);
	std::lock_guard<std::mutex> lock(g_scratch_mutex);
	ScratchEntry& entry = g_scratch[device];
	if (context_id == 0 || entry.context_id != context_id || entry.address == nullptr) {
		// the lookup also makes the runtime (re)create the device's primary context when none is current
		void* address = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&address, g_partials);
		if (e != cudaSuccess || address == nullptr)
			return Reject(TFIGA_E_CUDA, "cudaGetSymbolAddress of the residual-norm scratch failed");
		context_id = CurrentContextId(get_current, get_id);
		if (context_id == 0) return Reject(TFIGA_E_CUDA, "no current CUDA context after the scratch lookup");
		entry.address = static_cast<double*>(address);
		entry.context_id = context_id;
	}
	*out = entry.address;
	return TFIGA_OK;
}

} // namespace

extern "C" int tfiga_block_residual_norm_static(int64_t nodes, const int32_t* row_offsets_device,
	const int32_t* columns_device, const double* values_device, const double* x_device, const double* b_device,
	double* norm_device, void* stream)
{
	if (nodes < 0) return Reject(TFIGA_E_INVALID, "nodes must be non-negative");
	if (nodes > kMaxNodes)
		return Reject(TFIGA_E_UNSUPPORTED, "nodes exceeds the static scratch limit of 262144 block rows");
	if (norm_device == nullptr || (nodes > 0 && (row_offsets_device == nullptr || columns_device == nullptr
		|| values_device == nullptr || x_device == nullptr || b_device == nullptr)))
		return Reject(TFIGA_E_INVALID, "null device pointer");
	double* partials = nullptr;
	const int status = Scratch(&partials);
	if (status != TFIGA_OK) return status;
	const cudaStream_t s = static_cast<cudaStream_t>(stream);
	const int ctas = (int)((nodes+kRowsPerCta-1)/kRowsPerCta);
	if (ctas > 0)
		ResidualPartialKernel<<<ctas, 256, 0, s>>>((int)nodes, row_offsets_device, columns_device, values_device,
			x_device, b_device, partials);
	ResidualFinalizeKernel<<<1, kFinalizeThreads, 0, s>>>(ctas, partials, norm_device);
	const cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) return Reject(TFIGA_E_CUDA, cudaGetErrorString(e));
	return TFIGA_OK;
}
