// Shared host-side infrastructure: errors, device buffers, launch accounting.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace tfiga {

// Errors carry a TFIGA_E_* status through to the C ABI.
struct Error : std::runtime_error {
	int status;
	Error(int s, const std::string& message) : std::runtime_error(message), status(s) {}
};

[[noreturn]] void Fail(int status, const std::string& message);
void CudaCheck(cudaError_t error, const char* what);
// Checks the last launch (the launch configuration) without synchronizing.
void LaunchCheck(const char* kernel);

// RAII device allocation with a byte counter per process.
template <class T>
class DeviceArray {
public:
	DeviceArray() = default;
	explicit DeviceArray(std::size_t count) { Allocate(count); }
	~DeviceArray() { Release(); }
	DeviceArray(const DeviceArray&) = delete;
	DeviceArray& operator=(const DeviceArray&) = delete;
	DeviceArray(DeviceArray&& other) noexcept { *this = std::move(other); }
	DeviceArray& operator=(DeviceArray&& other) noexcept
	{
		if (this != &other) {
			Release();
			data_ = other.data_; count_ = other.count_;
			other.data_ = nullptr; other.count_ = 0;
		}
		return *this;
	}
	void Allocate(std::size_t count)
	{
		Release();
		if (count == 0) return;
		void* pointer = nullptr;
		const cudaError_t error = cudaMalloc(&pointer, count*sizeof(T));
		if (error != cudaSuccess) {
			(void)cudaGetLastError();
			Fail(-8, "device allocation of " + std::to_string(count*sizeof(T)) + " bytes failed: "
				+ cudaGetErrorString(error));
		}
		data_ = static_cast<T*>(pointer);
		count_ = count;
		Track(static_cast<long long>(bytes()));
	}
	void Release()
	{
		if (data_) {
			cudaFree(data_);
			Track(-static_cast<long long>(bytes()));
		}
		data_ = nullptr;
		count_ = 0;
	}
	// Source/destination may be host (pageable or pinned) or device memory (unified addressing).
	void Upload(const T* host, std::size_t count, cudaStream_t stream)
	{
		if (count > count_) Fail(-1, "upload exceeds device array size");
		if (count) CudaCheck(cudaMemcpyAsync(data_, host, count*sizeof(T), cudaMemcpyDefault, stream), "upload");
	}
	void Download(T* host, std::size_t count, cudaStream_t stream) const
	{
		if (count > count_) Fail(-1, "download exceeds device array size");
		if (count) CudaCheck(cudaMemcpyAsync(host, data_, count*sizeof(T), cudaMemcpyDefault, stream), "download");
	}
	void Zero(cudaStream_t stream)
	{
		if (count_) CudaCheck(cudaMemsetAsync(data_, 0, bytes(), stream), "memset");
	}
	T* get() const { return data_; }
	std::size_t size() const { return count_; }
	std::size_t bytes() const { return count_*sizeof(T); }

private:
	static void Track(long long delta);
	T* data_ = nullptr;
	std::size_t count_ = 0;
};

long long DeviceBytesLive();
long long DeviceBytesPeak();

// Requires a device that can run sm_100a code.
void RequireDevice();

// Device time per kernel family from CUDA events recorded around launches on
// the launching stream.  Disabled by default; Collect() waits for the stream.
class Profiler {
public:
	enum Family { kAssembly = 0, kSpmv = 1, kOrtho = 2, kOther = 3, kResidual = 4, kSetup = 5, kVector = 6,
		kFamilies = 7 };
	~Profiler();
	void Enable(bool on) { enabled_ = on; }
	bool enabled() const { return enabled_; }
	void Begin(Family family, cudaStream_t stream);
	void End(cudaStream_t stream);
	void Collect();
	// Algorithmic bytes a family moved (accounted by the caller, only while enabled).
	void AddBytes(Family family, double bytes) { if (enabled_) bytes_[family] += bytes; }
	// Bytes the kernels actually move for the same work (when it differs from the algorithmic count).
	void AddMovedBytes(Family family, double bytes) { if (enabled_) moved_[family] += bytes; }
	void Totals(double* ms, long long* counts, bool reset, double* bytes = nullptr, double* moved = nullptr);

private:
	struct Mark { cudaEvent_t start, stop; int family; };
	bool enabled_ = false;
	std::vector<Mark> pool_;
	size_t used_ = 0;
	int open_ = -1;
	double ms_[kFamilies] = {};
	long long count_[kFamilies] = {};
	double bytes_[kFamilies] = {};
	double moved_[kFamilies] = {};
};

} // namespace tfiga
