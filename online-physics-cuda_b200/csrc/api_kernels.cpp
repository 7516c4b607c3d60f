// C-ABI of the library-level pieces and of the hand-written kernels (include/fe.h): status codes, the per-thread error
// message, the contract record helpers, the hand-written heat step and the copy roof.
#include "../../include/fe.h"

#include "api_common.hpp"
#include "cuda_ctx.hpp"
#include "heat7.hpp"

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

namespace fe {

namespace {

thread_local std::string g_error;

// A few tensor maps keyed by (pointer, shape, box): a ping-pong step alternates between two.
struct MapCache {
    struct Entry {
        const float* base;
        int nx, ny, nz, bx, by, bz;
        FeTensorMap map;
    };
    std::mutex mutex;
    std::vector<Entry> entries;
    bool get(const float* base, int nx, int ny, int nz, int bx, int by, int bz, FeTensorMap& out, std::string& why)
    {
        std::lock_guard<std::mutex> lock(mutex);
        for (const Entry& e : entries) {
            if (e.base == base && e.nx == nx && e.ny == ny && e.nz == nz && e.bx == bx && e.by == by && e.bz == bz) {
                out = e.map;
                return true;
            }
        }
        Entry e{base, nx, ny, nz, bx, by, bz, {}};
        if (!encode_map_3d(&e.map, base, nx, ny, nz, bx, by, bz, why)) {
            return false;
        }
        if (entries.size() >= 16) {
            entries.erase(entries.begin());
        }
        entries.push_back(e);
        out = e.map;
        return true;
    }
};

MapCache& map_cache()
{
    static MapCache cache;
    return cache;
}

constexpr std::size_t kCheckHeader = 128; // fe_check (64 bytes), error word, block counter, padding


} // namespace

int fail(int code, const std::string& message)
{
    g_error = message;
    return code;
}

int ok()
{
    g_error.clear();
    return FE_OK;
}

const char* last_error()
{
    return g_error.c_str();
}

} // namespace fe

using namespace fe;

extern "C" {

int fe_version(void)
{
    return 1000;
}

const char* fe_last_error(void)
{
    return fe::last_error();
}

int fe_device_check(void)
{
    std::string why;
    if (!device_ready(why)) {
        return fail(FE_ENODEV, why);
    }
    return fe::ok();
}

float fe_key_to_float(uint32_t key)
{
    const uint32_t bits = (key & 0x80000000u) ? (key & 0x7fffffffu) : ~key;
    float v = 0.0f;
    std::memcpy(&v, &bits, 4);
    return v;
}

int fe_heat7_rows(int variant)
{
    return variant < 0 ? 8 : heat7_tma_rows(variant);
}

size_t fe_heat7_workspace_bytes(int nx, int ny, int nz, int variant, int zchunk)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || zchunk <= 0) {
        return 0;
    }
    const int blocks = variant < 0 ? heat7_plain_blocks(nx, ny, nz, zchunk) : heat7_tma_blocks(variant, nx, ny, nz, zchunk);
    if (blocks <= 0) {
        return 0;
    }
    return kCheckHeader + static_cast<size_t>(blocks) * 4 * sizeof(double);
}

int fe_check_reset(void* workspace, void* stream)
{
    if (workspace == nullptr) {
        return fail(FE_EINVAL, "fe_check_reset: null workspace");
    }
    std::string why;
    if (!cuda_ok(cudaMemsetAsync(workspace, 0, kCheckHeader, static_cast<cudaStream_t>(stream)), "fe_check_reset", why)) {
        return fail(FE_ECUDA, why);
    }
    return fe::ok();
}

int fe_check_read(const void* workspace, fe_check* out, void* stream)
{
    if (workspace == nullptr || out == nullptr) {
        return fail(FE_EINVAL, "fe_check_read: null pointer");
    }
    unsigned char header[kCheckHeader];
    std::string why;
    if (!cuda_ok(cudaMemcpyAsync(header, workspace, kCheckHeader, cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)), "fe_check_read", why) ||
        !cuda_ok(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "fe_check_read sync", why)) {
        return fail(FE_ECUDA, why);
    }
    static_assert(sizeof(fe_check) == sizeof(FeCheck), "fe_check mirrors FeCheck");
    std::memcpy(out, header, sizeof(fe_check));
    unsigned err = 0;
    std::memcpy(&err, header + 64, 4);
    if (err != 0) {
        return fail(FE_EKERNEL, "a kernel raised error word " + std::to_string(err) + " (a bounded wait gave up)");
    }
    return fe::ok();
}

int fe_heat7_step(const float* T_dev, float* out_dev, int nx, int ny, int nz, float k, float h, float dt, float lo, float hi,
    int variant, int zchunk, int check, void* workspace, void* stream)
{
    if (T_dev == nullptr || out_dev == nullptr || nx <= 0 || ny <= 0 || nz <= 0 || zchunk <= 0 || T_dev == out_dev) {
        return fail(FE_EINVAL, "fe_heat7_step: bad buffers or sizes");
    }
    if (variant >= 0 && heat7_tma_rows(variant) == 0) {
        return fail(FE_EINVAL, "fe_heat7_step: unknown variant " + std::to_string(variant));
    }
    if (variant >= 0 && ((nx & 3) != 0 || (reinterpret_cast<std::uintptr_t>(T_dev) & 15u) != 0 || (reinterpret_cast<std::uintptr_t>(out_dev) & 15u) != 0)) {
        return fail(FE_EINVAL, "fe_heat7_step: the TMA variants need nx % 4 == 0 and 16-byte aligned buffers (use variant -1)");
    }
    if (static_cast<unsigned long long>(nx) * ny * nz >= 0xffffffffull) {
        return fail(FE_EINVAL, "fe_heat7_step: more than 2^32 - 1 cells");
    }
    if (check && workspace == nullptr) {
        return fail(FE_EINVAL, "fe_heat7_step: contracts need a workspace");
    }
    std::string why;
    if (!device_ready(why)) {
        return fail(FE_ENODEV, why);
    }
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
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    a.rec = check ? reinterpret_cast<FeCheck*>(ws) : nullptr;
    a.err = ws ? reinterpret_cast<unsigned*>(ws + 64) : nullptr;
    a.count = ws ? reinterpret_cast<unsigned*>(ws + 68) : nullptr;
    a.partials = ws ? reinterpret_cast<double*>(ws + kCheckHeader) : nullptr;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (variant < 0) {
        e = launch_heat7_plain(T_dev, a, s);
    } else {
        if (a.err == nullptr) {
            return fail(FE_EINVAL, "fe_heat7_step: the TMA variants need a workspace (for their error word)");
        }
        FeTensorMap map;
        if (!map_cache().get(T_dev, nx, ny, nz, 128 + 8, heat7_tma_rows(variant) + 2, 1, map, why)) {
            return fail(FE_ECUDA, why);
        }
        e = launch_heat7_tma(variant, map, a, s);
    }
    if (!cuda_ok(e, "heat7 launch", why)) {
        return fail(FE_ECUDA, why);
    }
    return fe::ok();
}

int fe_copy_f32(const float* src_dev, float* dst_dev, size_t n, void* stream)
{
    if (src_dev == nullptr || dst_dev == nullptr || (n & 3) != 0 || (reinterpret_cast<std::uintptr_t>(src_dev) & 15u) != 0 ||
        (reinterpret_cast<std::uintptr_t>(dst_dev) & 15u) != 0) {
        return fail(FE_EINVAL, "fe_copy_f32: bad buffers or size (16-byte aligned buffers, a multiple of 4 floats)");
    }
    std::string why;
    if (!device_ready(why)) {
        return fail(FE_ENODEV, why);
    }
    if (!cuda_ok(launch_copy(src_dev, dst_dev, n, sm_count(), static_cast<cudaStream_t>(stream)), "copy launch", why)) {
        return fail(FE_ECUDA, why);
    }
    return fe::ok();
}

} // extern "C"
