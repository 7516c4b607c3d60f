// The CUDA plumbing under the law backend: the runtime (cudart, linked statically) for memory, streams, events and the
// hand-written kernels; the driver API, reached through cudaGetDriverEntryPoint (so nothing links libcuda and the
// library loads on a machine with no GPU), for run-time modules and TMA descriptors; NVRTC for the generated kernels.
// The architecture is fixed: sm_100a.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "fe_device.cuh"

namespace fe {

struct Driver {
    bool ok = false;
    std::string why;
    CUresult (*tensorMapEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
        const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
        CUtensorMapFloatOOBfill) = nullptr;
    CUresult (*moduleLoadData)(CUmodule*, const void*) = nullptr;
    CUresult (*moduleUnload)(CUmodule) = nullptr;
    CUresult (*moduleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
    CUresult (*launchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream, void**,
        void**) = nullptr;
    CUresult (*funcSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
    CUresult (*getErrorString)(CUresult, const char**) = nullptr;
    CUresult (*moduleGetGlobal)(CUdeviceptr*, size_t*, CUmodule, const char*) = nullptr;
    CUresult (*occupancyMaxActiveBlocksPerMultiprocessor)(int*, CUfunction, int, size_t) = nullptr;
};

// The driver entry points, looked up once (thread-safe). `ok` is false, with the reason, without a usable driver.
const Driver& driver();

// Sets `why` and returns false when the runtime call failed.
bool cuda_ok(cudaError_t e, const char* what, std::string& why);
bool cu_ok(CUresult r, const char* what, std::string& why);

// The device this thread works on is usable (a B200-class sm_100 part): false with the reason otherwise.
bool device_ready(std::string& why);
int sm_count();

// A tiled 3-D fp32 tensor map over a lattice (x fastest), box = (bx, by, bz) cells. The base must be 16-byte aligned
// and nx a multiple of 4 (row pitch in 16-byte units).
bool encode_map_3d(FeTensorMap* out, const float* base, int nx, int ny, int nz, int bx, int by, int bz, std::string& why);

// NVRTC: CUDA C++ source to a CUBIN for sm_100a (options: --fmad=false and friends). Results are cached on disk by a
// hash of the source, the options and the NVRTC version, under $FE_CACHE_DIR (or ~/.cache/fe_b200).
bool compile_cubin(const std::string& source, const std::string& name, std::string& cubin, std::string& log, double* ms);

std::uint64_t fnv1a(const void* data, std::size_t n, std::uint64_t h = 1469598103934665603ull);

} // namespace fe
