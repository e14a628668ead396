// Errors, CUDA checks, device requirement and allocation accounting.
#include "common.hpp"
#include "kernels.cuh"

#include <cuda_bf16.h>

#include <atomic>
#include <string>

namespace tfiga {

namespace {
std::atomic<long long> g_live{0};
std::atomic<long long> g_peak{0};
}

void Fail(int status, const std::string& message)
{
	throw Error(status, message);
}

void CudaCheck(cudaError_t error, const char* what)
{
	if (error != cudaSuccess) {
		(void)cudaGetLastError();
		Fail(-2, std::string(what)+": "+cudaGetErrorString(error));
	}
}

void LaunchCheck(const char* kernel)
{
	const cudaError_t error = cudaGetLastError();
	if (error != cudaSuccess) Fail(-2, std::string(kernel)+" launch failed: "+cudaGetErrorString(error));
}

template <class T>
void DeviceArray<T>::Track(long long delta)
{
	const long long now = g_live.fetch_add(delta)+delta;
	long long peak = g_peak.load();
	while (now > peak && !g_peak.compare_exchange_weak(peak, now)) {}
}

template class DeviceArray<double>;
template class DeviceArray<int32_t>;
template class DeviceArray<uint8_t>;
template class DeviceArray<unsigned>;
template class DeviceArray<float>;
template class DeviceArray<int64_t>;
template class DeviceArray<uint16_t>;
template class DeviceArray<__nv_bfloat16>;
template class DeviceArray<DeviceOutlet>;

long long DeviceBytesLive() { return g_live.load(); }
long long DeviceBytesPeak() { return g_peak.load(); }

void RequireDevice()
{
	int count = 0;
	const cudaError_t error = cudaGetDeviceCount(&count);
	if (error != cudaSuccess || count == 0) {
		(void)cudaGetLastError();
		Fail(-2, std::string("no CUDA device available (")+cudaGetErrorString(error)
			+"); this library has no CPU fallback");
	}
	int device = 0;
	CudaCheck(cudaGetDevice(&device), "cudaGetDevice");
	cudaDeviceProp prop{};
	CudaCheck(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
	if (prop.major != 10)
		Fail(-7, "this build targets sm_100a (B200); device "+std::string(prop.name)+" is sm_"
			+std::to_string(prop.major)+std::to_string(prop.minor));
}

Profiler::~Profiler()
{
	for (auto& m : pool_) { cudaEventDestroy(m.start); cudaEventDestroy(m.stop); }
}

void Profiler::Begin(Family family, cudaStream_t stream)
{
	if (!enabled_) return;
	if (used_ == pool_.size()) {
		Mark m{};
		CudaCheck(cudaEventCreate(&m.start), "profile event");
		CudaCheck(cudaEventCreate(&m.stop), "profile event");
		pool_.push_back(m);
	}
	pool_[used_].family = family;
	CudaCheck(cudaEventRecord(pool_[used_].start, stream), "profile record");
	open_ = (int)used_;
}

void Profiler::End(cudaStream_t stream)
{
	if (!enabled_ || open_ < 0) return;
	CudaCheck(cudaEventRecord(pool_[open_].stop, stream), "profile record");
	open_ = -1;
	++used_;
}

void Profiler::Collect()
{
	for (size_t i = 0; i < used_; ++i) {
		CudaCheck(cudaEventSynchronize(pool_[i].stop), "profile sync");
		float ms = 0.0f;
		CudaCheck(cudaEventElapsedTime(&ms, pool_[i].start, pool_[i].stop), "profile elapsed");
		ms_[pool_[i].family] += ms;
		count_[pool_[i].family] += 1;
	}
	used_ = 0;
}

void Profiler::Totals(double* ms, long long* counts, bool reset, double* bytes, double* moved)
{
	Collect();
	for (int f = 0; f < kFamilies; ++f) {
		if (ms) ms[f] = ms_[f];
		if (counts) counts[f] = count_[f];
		if (bytes) bytes[f] = bytes_[f];
		if (moved) moved[f] = moved_[f];
		if (reset) { ms_[f] = 0.0; count_[f] = 0; bytes_[f] = 0.0; moved_[f] = 0.0; }
	}
}

} // namespace tfiga
