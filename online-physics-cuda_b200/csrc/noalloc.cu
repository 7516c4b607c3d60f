// fe_heat7_step_noalloc: the hand-written heat step with its contracts, for callers that cannot allocate device memory.
//
// fe_heat7_step takes a caller-allocated workspace for the contract pass's per-block partial sums. Some callers cannot
// provide one: a host whose device memory belongs to another allocator and may not call cudaMalloc itself (a caching
// allocator, a memory pool sized at start-up), a plugin loaded into a process that forbids new device allocations once
// it runs, or a latency-bound loop that cannot afford cudaMalloc's implicit synchronisation. This form keeps that
// scratch in a fixed array in the library's own device memory instead, sized for at most kMaxBlocks thread blocks.
// Every GPU that loads the library holds the array (about 256 KiB) until the process exits.
//
// The array is shared by every call: each call clears what must start at zero (the block counter, and the caller's
// record with its error word) before its kernel, and calls whose kernels overlap on the GPU (several streams, several
// host threads) race on it. Serialise them on one stream.
//
// The first call on a device looks up the array's device address. That lookup may be what loads the library's device
// code on that device, and so what creates the array: a caller that may not allocate inside some region (or captures
// a stream) makes one call before it. The address is kept per device for the primary context; cudaDeviceReset makes
// it stale.
#include "../../include/fe.h"

#include "api_common.hpp"
#include "cuda_ctx.hpp"
#include "heat7.hpp"

#include <mutex>
#include <string>

namespace fe {
namespace {

constexpr int kMaxBlocks = 8192;       // thread blocks one pass may have (the partial sums of one each)
constexpr std::size_t kHeader = 128;   // error word at 0, block counter at 4
constexpr std::size_t kScratchBytes = kHeader + static_cast<std::size_t>(kMaxBlocks) * 4 * sizeof(double);

static __device__ __align__(256) unsigned char g_heat7_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_address[kMaxDevices] = {};

// The device address of the scratch array on the current device, looked up once per device (with that device
// current). The array's name in host code is only a host-side stand-in: the kernel must get this address.
bool scratch_address(void** out, std::string& why)
{
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice", why)) return false;
    if (dev < 0 || dev >= kMaxDevices) {
        why = "device index out of range";
        return false;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_address[dev] == nullptr) {
        void* p = nullptr;
        if (!cuda_ok(cudaGetSymbolAddress(&p, g_heat7_scratch), "cudaGetSymbolAddress (heat7 scratch)", why)) return false;
        g_address[dev] = p;
    }
    *out = g_address[dev];
    return true;
}

} // namespace
} // namespace fe

extern "C" int fe_heat7_step_noalloc(const float* T_dev, float* out_dev, int nx, int ny, int nz, float k, float h, float dt, float lo,
    float hi, int variant, int zchunk, int check, fe_check* record_dev, void* stream)
{
    using namespace fe;
    if (T_dev == nullptr || out_dev == nullptr || nx <= 0 || ny <= 0 || nz <= 0 || zchunk <= 0 || T_dev == out_dev) {
        return fail(FE_EINVAL, "fe_heat7_step_noalloc: bad buffers or sizes");
    }
    if (variant >= 0 && heat7_tma_rows(variant) == 0) {
        return fail(FE_EINVAL, "fe_heat7_step_noalloc: unknown variant " + std::to_string(variant));
    }
    if (variant >= 0 && ((nx & 3) != 0 || (reinterpret_cast<std::uintptr_t>(T_dev) & 15u) != 0 || (reinterpret_cast<std::uintptr_t>(out_dev) & 15u) != 0)) {
        return fail(FE_EINVAL, "fe_heat7_step_noalloc: the TMA variants need nx % 4 == 0 and 16-byte aligned buffers (use variant -1)");
    }
    if (static_cast<unsigned long long>(nx) * ny * nz >= 0xffffffffull) {
        return fail(FE_EINVAL, "fe_heat7_step_noalloc: more than 2^32 - 1 cells");
    }
    if (check && record_dev == nullptr) {
        return fail(FE_EINVAL, "fe_heat7_step_noalloc: contracts need a record (a device fe_check)");
    }
    // A TMA variant's bounded waits report a wait that gave up through an error word, which must reach the caller:
    // it lands in the record, so these variants need one even without contracts (fe_heat7_step asks a workspace).
    if (variant >= 0 && record_dev == nullptr) {
        return fail(FE_EINVAL, "fe_heat7_step_noalloc: the TMA variants need a record (a device fe_check, for their error word)");
    }
    const int blocks = variant < 0 ? heat7_plain_blocks(nx, ny, nz, zchunk) : heat7_tma_blocks(variant, nx, ny, nz, zchunk);
    if (blocks > kMaxBlocks) {
        return fail(FE_EINVAL, "fe_heat7_step_noalloc: this lattice needs " + std::to_string(blocks) + " thread blocks; the fixed scratch holds " +
            std::to_string(kMaxBlocks) + " (raise zchunk, or use fe_heat7_step with a workspace)");
    }
    std::string why;
    if (!device_ready(why)) return fail(FE_ENODEV, why);
    void* scratch = nullptr;
    if (!scratch_address(&scratch, why)) return fail(FE_ECUDA, why);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The previous call's block counter is still in the array: clear it, and the caller's record (its error word too).
    if (!cuda_ok(cudaMemsetAsync(scratch, 0, kHeader, s), "clear scratch", why)) return fail(FE_ECUDA, why);
    if (record_dev != nullptr && !cuda_ok(cudaMemsetAsync(record_dev, 0, sizeof(fe_check), s), "clear record", why)) {
        return fail(FE_ECUDA, why);
    }
    unsigned char* base = static_cast<unsigned char*>(scratch);
    HeatArgs a{};
    a.out = out_dev;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.zchunk = zchunk;
    a.k = k;
    a.h = h;
    a.dt = dt;
    a.inv_hh = exact_reciprocal(h * h);
    a.lo = lo;
    a.hi = hi;
    a.totals_before = (check & FE_HEAT7_BEFORE) ? 1 : 0;
    a.totals_after = (check & FE_HEAT7_AFTER) ? 1 : 0;
    a.rec = check ? reinterpret_cast<FeCheck*>(record_dev) : nullptr;
    // A kernel's error word lands in the caller's record (pad[0]). Without one (the plain kernel without contracts,
    // which has no waits) there is none, as with fe_heat7_step given no workspace.
    a.err = record_dev != nullptr ? &record_dev->pad[0] : nullptr;
    a.count = reinterpret_cast<unsigned*>(base + 4);
    a.partials = reinterpret_cast<double*>(base + kHeader);
    cudaError_t e;
    if (variant < 0) {
        e = launch_heat7_plain(T_dev, a, s);
    } else {
        FeTensorMap map;
        if (!encode_map_3d(&map, T_dev, nx, ny, nz, 128 + 8, heat7_tma_rows(variant) + 2, 1, why)) return fail(FE_ECUDA, why);
        e = launch_heat7_tma(variant, map, a, s);
    }
    if (!cuda_ok(e, "heat7 launch", why)) return fail(FE_ECUDA, why);
    return ok();
}
