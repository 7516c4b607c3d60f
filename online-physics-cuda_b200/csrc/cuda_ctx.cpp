#include "cuda_ctx.hpp"

#include <nvrtc.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <sys/stat.h>
#include <vector>

namespace fe {

std::uint64_t fnv1a(const void* data, std::size_t n, std::uint64_t h)
{
    const auto* p = static_cast<const unsigned char*>(data);
    for (std::size_t i = 0; i < n; ++i) {
        h = (h ^ p[i]) * 1099511628211ull;
    }
    return h;
}

bool cuda_ok(cudaError_t e, const char* what, std::string& why)
{
    if (e == cudaSuccess) {
        return true;
    }
    why = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return false;
}

bool cu_ok(CUresult r, const char* what, std::string& why)
{
    if (r == CUDA_SUCCESS) {
        return true;
    }
    const char* text = nullptr;
    if (driver().getErrorString != nullptr) {
        driver().getErrorString(r, &text);
    }
    why = std::string(what) + ": CUresult " + std::to_string(static_cast<int>(r)) + (text ? std::string(" (") + text + ")" : "");
    return false;
}

namespace {

template <typename F>
bool entry(const char* name, F& out, std::string& why)
{
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    const cudaError_t e = cudaGetDriverEntryPoint(name, &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || fn == nullptr || q != cudaDriverEntryPointSuccess) {
        why = std::string("driver entry point ") + name + " unavailable" + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
        return false;
    }
    out = reinterpret_cast<F>(fn);
    return true;
}

} // namespace

const Driver& driver()
{
    static Driver d;
    static std::once_flag once;
    std::call_once(once, [] {
        int count = 0;
        const cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0) {
            d.why = std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "none found");
            return;
        }
        std::string why;
        const bool all = entry("cuTensorMapEncodeTiled", d.tensorMapEncodeTiled, why) && entry("cuModuleLoadData", d.moduleLoadData, why) &&
            entry("cuModuleUnload", d.moduleUnload, why) && entry("cuModuleGetFunction", d.moduleGetFunction, why) &&
            entry("cuLaunchKernel", d.launchKernel, why) && entry("cuFuncSetAttribute", d.funcSetAttribute, why) &&
            entry("cuGetErrorString", d.getErrorString, why) && entry("cuModuleGetGlobal", d.moduleGetGlobal, why) &&
            entry("cuOccupancyMaxActiveBlocksPerMultiprocessor", d.occupancyMaxActiveBlocksPerMultiprocessor, why);
        if (!all) {
            d.why = why;
            return;
        }
        d.ok = true;
    });
    return d;
}

bool device_ready(std::string& why)
{
    const Driver& d = driver();
    if (!d.ok) {
        why = d.why;
        return false;
    }
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice", why)) {
        return false;
    }
    int major = 0;
    int minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (major != 10 || minor != 0) {
        why = "this backend is built for sm_100a (B200); device " + std::to_string(dev) + " is sm_" + std::to_string(major) +
            std::to_string(minor);
        return false;
    }
    // The driver-API calls (modules, launches) run in the runtime's primary context: make it current on this thread.
    if (!cuda_ok(cudaSetDevice(dev), "cudaSetDevice", why) || !cuda_ok(cudaFree(nullptr), "context", why)) {
        return false;
    }
    return true;
}

int sm_count()
{
    int dev = 0;
    cudaGetDevice(&dev);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 148;
}

bool encode_map_3d(FeTensorMap* out, const float* base, int nx, int ny, int nz, int bx, int by, int bz, std::string& why)
{
    static_assert(sizeof(FeTensorMap) == sizeof(CUtensorMap), "FeTensorMap mirrors CUtensorMap");
    const Driver& d = driver();
    if (!d.ok) {
        why = d.why;
        return false;
    }
    if ((reinterpret_cast<std::uintptr_t>(base) & 15u) != 0 || (nx & 3) != 0) {
        why = "TMA needs a 16-byte aligned base and a row of a multiple of 16 bytes";
        return false;
    }
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(nx), static_cast<cuuint64_t>(ny), static_cast<cuuint64_t>(nz)};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(nx) * 4u, static_cast<cuuint64_t>(nx) * static_cast<cuuint64_t>(ny) * 4u};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(bx), static_cast<cuuint32_t>(by), static_cast<cuuint32_t>(bz)};
    const cuuint32_t estr[3] = {1, 1, 1};
    return cu_ok(d.tensorMapEncodeTiled(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE),
        "cuTensorMapEncodeTiled", why);
}

namespace {

std::string cache_dir()
{
    if (const char* dir = std::getenv("FE_CACHE_DIR"); dir != nullptr && dir[0] != 0) {
        return dir;
    }
    const char* home = std::getenv("HOME");
    return std::string(home != nullptr ? home : "/tmp") + "/.cache/fe_b200";
}

void make_dirs(const std::string& path)
{
    std::string part;
    for (std::size_t i = 0; i < path.size(); ++i) {
        part += path[i];
        if (path[i] == '/' || i + 1 == path.size()) {
            mkdir(part.c_str(), 0755);
        }
    }
}

} // namespace

bool compile_cubin(const std::string& source, const std::string& name, std::string& cubin, std::string& log, double* ms)
{
    const auto start = std::chrono::steady_clock::now();
    std::vector<const char*> options = {"--gpu-architecture=sm_100a", "--fmad=false", "-std=c++17", "-default-device",
        "--extra-device-vectorization", "-lineinfo"};
    int major = 0;
    int minor = 0;
    nvrtcVersion(&major, &minor);
    std::uint64_t key = fnv1a(source.data(), source.size());
    for (const char* o : options) {
        key = fnv1a(o, std::strlen(o), key);
    }
    key = fnv1a(&major, sizeof(major), key);
    key = fnv1a(&minor, sizeof(minor), key);
    char hex[32];
    std::snprintf(hex, sizeof(hex), "%016llx", static_cast<unsigned long long>(key));
    const std::string dir = cache_dir();
    const std::string path = dir + "/" + hex + ".cubin";
    {
        std::ifstream in(path, std::ios::binary);
        if (in) {
            std::ostringstream all;
            all << in.rdbuf();
            cubin = all.str();
            if (!cubin.empty()) {
                if (ms) *ms = 0.0;
                return true;
            }
        }
    }
    nvrtcProgram prog = nullptr;
    if (nvrtcCreateProgram(&prog, source.c_str(), name.c_str(), 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        log = "nvrtcCreateProgram failed";
        return false;
    }
    const nvrtcResult r = nvrtcCompileProgram(prog, static_cast<int>(options.size()), options.data());
    std::size_t log_size = 0;
    nvrtcGetProgramLogSize(prog, &log_size);
    log.assign(log_size, '\0');
    if (log_size > 0) {
        nvrtcGetProgramLog(prog, log.data());
    }
    if (r != NVRTC_SUCCESS) {
        log = std::string("NVRTC: ") + nvrtcGetErrorString(r) + "\n" + log;
        nvrtcDestroyProgram(&prog);
        return false;
    }
    std::size_t size = 0;
    nvrtcGetCUBINSize(prog, &size);
    cubin.assign(size, '\0');
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
    make_dirs(dir);
    {
        const std::string tmp = path + ".tmp" + std::to_string(static_cast<long long>(std::chrono::steady_clock::now().time_since_epoch().count()));
        std::ofstream out(tmp, std::ios::binary);
        out.write(cubin.data(), static_cast<std::streamsize>(cubin.size()));
        out.close();
        std::rename(tmp.c_str(), path.c_str());
    }
    if (ms) {
        *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
    }
    return true;
}

} // namespace fe
