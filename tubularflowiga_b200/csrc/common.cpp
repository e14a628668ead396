// Errors, CUDA checks, device requirement and allocation accounting.
#include "common.hpp"

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

} // namespace tfiga
