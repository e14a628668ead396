// The drop-in command (tfiga_main): device-info and mesh-check
// (solvers/cuda/src/iga_cuda.cu:278-303, 604-617, 1157-1195).
#include "mesh.hpp"

#include "../../include/tfiga.h"

#include <cstdio>
#include <exception>
#include <iomanip>
#include <iostream>
#include <string>

namespace {

void PrintDevice()
{
	int device = 0;
	tfiga::CudaCheck(cudaGetDevice(&device), "cudaGetDevice");
	cudaDeviceProp prop{};
	tfiga::CudaCheck(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
	size_t free_bytes = 0, total = 0;
	tfiga::CudaCheck(cudaMemGetInfo(&free_bytes, &total), "cudaMemGetInfo");
	int runtime = 0, driver = 0;
	cudaRuntimeGetVersion(&runtime);
	cudaDriverGetVersion(&driver);
	std::cout << "device=" << device << " name=\"" << prop.name << "\" compute_capability=" << prop.major << '.'
		<< prop.minor << " sms=" << prop.multiProcessorCount
		<< " memory_free_gib=" << free_bytes/1073741824.0 << " memory_total_gib=" << total/1073741824.0 << '\n';
	std::cout << "cuda_capabilities runtime_build=" << CUDART_VERSION << " runtime_linked=" << runtime
		<< " driver=" << driver << " arch=sm_100a\n";
}

int MeshCheck(const std::string& path)
{
	tfiga::Mesh mesh(tfiga::ReadNtiga(path));
	const auto& h = mesh.host();
	std::cout << "mesh nodes=" << h.nodes << " elements=" << h.elements() << " basis_entries=" << h.connectivity.size()
		<< " extraction_nonzeros=" << h.extraction_values.size() << " max_basis=" << h.max_basis
		<< " block_nonzeros=" << mesh.pattern().columns.size()
		<< " mean_block_row=" << (double)mesh.pattern().columns.size()/h.nodes << '\n';
	std::cout << "geometry min_detJ=" << std::setprecision(17) << mesh.min_detj() << " bad_samples="
		<< mesh.bad_samples() << " device_mesh_gib=" << mesh.device_bytes()/1073741824.0 << '\n';
	return mesh.bad_samples() ? 1 : 0;
}

} // namespace

extern "C" int tfiga_main(int argc, char** argv)
{
	try {
		if (argc < 2) throw std::runtime_error("usage: iga_cuda_b200 device-info|mesh-check|navier-stokes ...");
		tfiga::RequireDevice();
		const std::string command(argv[1]);
		PrintDevice();
		if (command == "device-info") return 0;
		if (command == "mesh-check") {
			if (argc != 3) throw std::runtime_error("usage: iga_cuda_b200 mesh-check DATABASE.ntiga");
			return MeshCheck(argv[2]);
		}
		throw std::runtime_error("unknown command: "+command);
	} catch (const std::exception& error) {
		std::cerr << "iga_cuda: " << error.what() << '\n';
		return 1;
	}
}
