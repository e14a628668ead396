// iga_cuda_b200: the drop-in command line for `iga_cuda` (device-info,
// mesh-check, navier-stokes); all work happens in libtfiga_b200.so.
#include "tfiga.h"

int main(int argc, char** argv)
{
	return tfiga_main(argc, argv);
}
