#include "engine.hpp"

#include "heat7.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <sstream>

namespace fe {

namespace {

using law::Op;

constexpr int kRing = 64;           // steps of contract records a deferred run may keep on the card
constexpr int kMaxSubsteps = 4096;  // Solver::kMaxSubsteps (src/field/Solver.hpp:129)
static_assert(sizeof(FePassArgs) <= 4096, "a generated pass takes its arguments as one kernel parameter of at most 4 KB");

double times(double a, double b)
{
    return a == 0.0 || b == 0.0 ? 0.0 : a * b; // 0 * infinity: nothing of it (LawBounds.cpp:8-11)
}

float key_to_float(unsigned key)
{
    const unsigned bits = (key & 0x80000000u) ? (key & 0x7fffffffu) : ~key;
    float v = 0.0f;
    std::memcpy(&v, &bits, 4);
    return v;
}

std::size_t round256(std::size_t n)
{
    return (n + 255) / 256 * 256;
}

} // namespace

Engine::~Engine()
{
    if (stream_ != nullptr) cudaStreamSynchronize(stream_);
    if (module_ != nullptr && driver().ok) driver().moduleUnload(module_);
    if (arena_ != nullptr) cudaFree(arena_);
    if (records_ != nullptr) cudaFree(records_);
    if (partials_ != nullptr) cudaFree(partials_);
    if (counts_ != nullptr) cudaFree(counts_);
    if (flags_ != nullptr) cudaFree(flags_);
    if (snapshot_ != nullptr) cudaFree(snapshot_);
    if (bounds_rec_ != nullptr) cudaFree(bounds_rec_);
    if (rotate_scratch_ != nullptr) cudaFree(rotate_scratch_);
    if (ev0_ != nullptr) cudaEventDestroy(ev0_);
    if (ev1_ != nullptr) cudaEventDestroy(ev1_);
    if (stream_ != nullptr) cudaStreamDestroy(stream_);
}

bool Engine::create(const std::vector<law::Source>& sources, int nx, int ny, int nz, double h, std::string& why)
{
    if (nx < 1 || ny < 1 || nz < 1 || !(h > 0.0)) {
        why = "the lattice needs nx, ny, nz >= 1 and h > 0";
        return false;
    }
    if (static_cast<unsigned long long>(nx) * ny * nz >= 0xffffffffull) {
        why = "more than 2^32 - 1 cells";
        return false;
    }
    nx_ = nx;
    ny_ = ny;
    nz_ = nz;
    h_ = h;
    cells_ = static_cast<std::size_t>(nx) * ny * nz;
    std::vector<std::string> errors;
    law::Law law = law::compile(sources, errors);
    if (!errors.empty()) {
        std::ostringstream all;
        for (const std::string& e : errors) all << e << "\n";
        why = all.str();
        return false;
    }
    ir::Module m = ir::lower(law);
    return create(std::move(law), std::move(m), nx, ny, nz, h, why);
}

bool Engine::create(law::Law law, ir::Module module, int nx, int ny, int nz, double h, std::string& why)
{
    if (nx < 1 || ny < 1 || nz < 1 || !(h > 0.0)) {
        why = "the lattice needs nx, ny, nz >= 1 and h > 0";
        return false;
    }
    if (static_cast<unsigned long long>(nx) * ny * nz >= 0xffffffffull) {
        why = "more than 2^32 - 1 cells";
        return false;
    }
    nx_ = nx;
    ny_ = ny;
    nz_ = nz;
    h_ = h;
    cells_ = static_cast<std::size_t>(nx) * ny * nz;
    law_ = std::move(law);
    mod_ = std::move(module);
    if (!gen::generate(mod_, law_, nx, ny, nz, h, plan_, why)) return false;
    if (!device_ready(why)) return false;
    sms_ = sm_count();
    std::string cubin;
    std::string log;
    if (!compile_cubin(plan_.source, "law.cu", cubin, log, &compile_ms_)) {
        why = "NVRTC could not compile the generated law:\n" + log;
        return false;
    }
    const Driver& d = driver();
    if (!cu_ok(d.moduleLoadData(&module_, cubin.data()), "cuModuleLoadData", why)) return false;
    std::size_t bytes = 0;
    if (!cu_ok(d.moduleGetGlobal(&params_, &bytes, module_, "FE_P"), "FE_P", why)) return false;
    if (!cu_ok(d.moduleGetGlobal(&uniforms_, &bytes, module_, "FE_U"), "FE_U", why)) return false;
    if (!plan_.net_blob.empty()) {
        // The nets' parameters (their files', or the untrained start) into the module's FE_NET.
        CUdeviceptr nets = 0;
        if (!cu_ok(d.moduleGetGlobal(&nets, &bytes, module_, "FE_NET"), "FE_NET", why)) return false;
        if (bytes < plan_.net_blob.size() * sizeof(float)) {
            why = "internal: FE_NET is smaller than the nets' parameters";
            return false;
        }
        if (!cuda_ok(cudaMemcpy(reinterpret_cast<void*>(nets), plan_.net_blob.data(), plan_.net_blob.size() * sizeof(float), cudaMemcpyHostToDevice),
                "nets", why)) {
            return false;
        }
    }
    if (!plan_.net_bf16.empty()) {
        // The `half` nets' BF16 weights, in the layout their tensor-core stage kernels copy into shared memory.
        CUdeviceptr netb = 0;
        if (!cu_ok(d.moduleGetGlobal(&netb, &bytes, module_, "FE_NETB"), "FE_NETB", why)) return false;
        if (bytes < plan_.net_bf16.size() * sizeof(unsigned short)) {
            why = "internal: FE_NETB is smaller than the half nets' weights";
            return false;
        }
        if (!cuda_ok(cudaMemcpy(reinterpret_cast<void*>(netb), plan_.net_bf16.data(), plan_.net_bf16.size() * sizeof(unsigned short),
                         cudaMemcpyHostToDevice),
                "half nets", why)) {
            return false;
        }
    }
    if (!cuda_ok(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate", why)) return false;
    if (!cuda_ok(cudaEventCreate(&ev0_), "cudaEventCreate", why) || !cuda_ok(cudaEventCreate(&ev1_), "cudaEventCreate", why)) return false;

    // One arena: every field's current buffer, the next buffer of the ping-pong ones, every stage slot.
    const std::size_t field_bytes = round256(cells_ * sizeof(float));
    const std::size_t fields = law_.fields.size();
    std::size_t buffers = fields + static_cast<std::size_t>(plan_.slots);
    for (const char pp : plan_.pingpong) buffers += pp ? 1 : 0;
    if (!cuda_ok(cudaMalloc(&arena_, std::max<std::size_t>(1, buffers) * field_bytes), "cudaMalloc (lattice)", why)) return false;
    char* base = static_cast<char*>(arena_);
    now_.assign(fields, nullptr);
    next_.assign(fields, nullptr);
    for (std::size_t f = 0; f < fields; ++f) {
        now_[f] = reinterpret_cast<float*>(base);
        base += field_bytes;
        if (plan_.pingpong[f]) {
            next_[f] = reinterpret_cast<float*>(base);
            base += field_bytes;
        }
    }
    for (int s = 0; s < plan_.slots; ++s) {
        slot_.push_back(reinterpret_cast<float*>(base));
        base += field_bytes;
    }
    bounds_.assign(fields, Bounds{});
    zero_.assign(fields, 0);
    carry_.assign(fields, Carry{});
    own_z0_ = 0;
    own_z1_ = nz;
    for (std::size_t f = 0; f < fields; ++f) {
        const float init = static_cast<float>(law_.fields[f].init);
        if (!cuda_ok(launch_fill(now_[f], cells_, init, sms_, stream_), "fill", why)) return false;
        if (next_[f] != nullptr && !cuda_ok(launch_fill(next_[f], cells_, init, sms_, stream_), "fill", why)) return false;
        bounds_[f] = Bounds{init, init};
        zero_[f] = init == 0.0f ? 1 : 0;
    }
    for (float* s : slot_) {
        if (!cuda_ok(cudaMemsetAsync(s, 0, cells_ * sizeof(float), stream_), "memset", why)) return false;
    }
    // What distance and poisson compare their input with starts unlike any input: the first look solves.
    for (const auto& [slot, bits] : plan_.slot_fill) {
        if (bits == 0u) continue;
        float v = 0.0f;
        std::memcpy(&v, &bits, sizeof(v));
        if (!cuda_ok(launch_fill(slot_[static_cast<std::size_t>(slot)], cells_, v, sms_, stream_), "fill", why)) return false;
    }
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&flags_), std::max(1, plan_.flags) * sizeof(unsigned)), "cudaMalloc (flags)", why)) return false;

    // Contract records: one per checked output of every program, per step, in a ring.
    records_per_step_ = 0;
    std::size_t partial_doubles = std::max<std::size_t>(4 * 1024, 4 * static_cast<std::size_t>(kTotalsBlocks));
    auto consider = [&](const gen::Launch& L) {
        const bool slab = L.slab;
        const int zchunk = zchunk_for(L, slab);
        const std::size_t blocks = slab ? static_cast<std::size_t>((nx_ + 127) / 128) * ((ny_ + L.ty - 1) / L.ty) * ((nz_ + zchunk - 1) / zchunk)
                                        : static_cast<std::size_t>((nx_ + 31) / 32) * ((ny_ + 7) / 8) * ((nz_ + zchunk - 1) / zchunk);
        const std::size_t plain_blocks = static_cast<std::size_t>((nx_ + 31) / 32) * ((ny_ + 7) / 8) * ((nz_ + zchunk_for(L, false) - 1) / zchunk_for(L, false));
        partial_doubles = std::max(partial_doubles, 4 * FE_MAX_OUT * std::max(blocks, plain_blocks));
    };
    for (const auto* progs : {&plan_.terms, &plan_.learned, &plan_.derives}) {
        for (const gen::ProgramPlan& pp : *progs) {
            if (pp.empty) continue;
            records_per_step_ += static_cast<int>(pp.gather.outs.size());
            consider(pp.gather);
            for (const gen::Launch& L : pp.stages) consider(L);
            for (const gen::Launch& L : pp.limit) consider(L);
        }
    }
    ring_ = kRing;
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&records_), sizeof(FeCheck) * std::max(1, records_per_step_) * ring_), "cudaMalloc (records)", why)) return false;
    if (!cuda_ok(cudaMemsetAsync(records_, 0, sizeof(FeCheck) * std::max(1, records_per_step_) * ring_, stream_), "memset", why)) return false;
    partial_doubles_ = partial_doubles;
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&partials_), partial_doubles * sizeof(double)), "cudaMalloc (partials)", why)) return false;
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&counts_), (FE_MAX_OUT + 4) * sizeof(unsigned)), "cudaMalloc (counters)", why)) return false;
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&bounds_rec_), sizeof(FeCheck)), "cudaMalloc (upload bounds)", why)) return false;
    if (!cuda_ok(cudaMemsetAsync(counts_, 0, (FE_MAX_OUT + 4) * sizeof(unsigned), stream_), "memset", why)) return false;

    param_host_ = law_.param_values;
    params_dirty_ = true;
    substeps_.assign(law_.terms.size(), 1);
    term_profile_.assign(law_.terms.size(), TermProfile{});
    return cuda_ok(cudaStreamSynchronize(stream_), "create", why);
}

bool Engine::buffer(const gen::Buf& b, float*& out) const
{
    switch (b.kind) {
    case gen::Buf::FieldNow: out = now_[static_cast<std::size_t>(b.id)]; break;
    case gen::Buf::FieldNext: out = next_[static_cast<std::size_t>(b.id)]; break;
    case gen::Buf::Slot: out = slot_[static_cast<std::size_t>(b.id)]; break;
    }
    return out != nullptr;
}

bool Engine::map_for(const float* base, int bx, int by, FeTensorMap& out, std::string& why)
{
    const auto key = std::make_tuple(base, bx, by);
    const auto found = maps_.find(key);
    if (found != maps_.end()) {
        out = found->second;
        return true;
    }
    if (!encode_map_3d(&out, base, nx_, ny_, nz_, bx, by, 1, why)) return false;
    maps_.emplace(key, out);
    return true;
}

CUfunction Engine::function(const std::string& name, unsigned smem, std::string& why)
{
    const auto found = functions_.find(name);
    if (found != functions_.end()) return found->second;
    CUfunction fn = nullptr;
    if (!cu_ok(driver().moduleGetFunction(&fn, module_, name.c_str()), ("kernel " + name).c_str(), why)) return nullptr;
    // The default cap (48 KB) counts static and dynamic shared memory together: any dynamic size gets its attribute.
    if (smem > 0 &&
        !cu_ok(driver().funcSetAttribute(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, static_cast<int>(smem)), "smem attribute", why)) {
        return nullptr;
    }
    functions_.emplace(name, fn);
    return fn;
}

int Engine::resident(const gen::Launch& L)
{
    const auto it = resident_.find(L.kernel);
    if (it != resident_.end()) return it->second;
    // The shared memory's bound (the 227 KB an SM hands out, 2 KB of it for the static part a CTA), at most 8, refined
    // by the driver's count, which also weighs the registers the compiled kernel uses.
    int per_sm = static_cast<int>(std::max<long long>(1, std::min<long long>(8, (227LL * 1024) / (static_cast<long long>(L.smem) + 2048))));
    std::string why;
    const CUfunction fn = function(L.kernel, L.smem, why);
    int n = 0;
    if (fn != nullptr && driver().occupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 256, L.smem) == CUDA_SUCCESS && n > 0) per_sm = n;
    resident_.emplace(L.kernel, per_sm);
    return per_sm;
}

int Engine::zchunk_for(const gen::Launch& L, bool slab)
{
    // Several waves of CTAs (a short last wave wastes little), and chunks long enough that the z halo is a small part of
    // what is read (2 RZ planes of every 32 RZ) — but never so long that the grid falls under two waves of resident
    // CTAs: on a small lattice the halo re-reads come from L2, an idle SM is lost for good.
    const long long tiles = slab ? static_cast<long long>((nx_ + 127) / 128) * ((ny_ + L.ty - 1) / L.ty)
                                 : static_cast<long long>((nx_ + 31) / 32) * ((ny_ + 7) / 8);
    const long long want = static_cast<long long>(sms_) * (slab ? 12 : 16);
    const long long chunks = std::max<long long>(1, (want + tiles - 1) / tiles);
    int zchunk = static_cast<int>((nz_ + chunks - 1) / chunks);
    if (L.rz > 0) {
        // A wave is every SM's resident CTAs.
        const long long per_sm = slab && L.kind == gen::Launch::Pass ? resident(L) : 8;
        const long long slots = static_cast<long long>(sms_) * per_sm;
        const long long two_waves = std::max<long long>(1, static_cast<long long>(nz_) * tiles / (2LL * slots));
        zchunk = std::max(zchunk, static_cast<int>(std::min<long long>({static_cast<long long>(nz_), 32LL * L.rz, two_waves})));
        if (slab && L.kind == gen::Launch::Pass) {
            // A lattice big enough for three waves of chunks of 8 planes or more takes the chunk length whose last wave
            // is fullest, weighed against its z halo: fill x planes / (planes + 2 RZ), fill = waves / ceil(waves). The
            // 512^3 heat gather (64 tiles, 3 CTAs an SM): 19 planes (3.89 waves) 5.09 TB/s, 27 (2.74) 4.94, 22 (3.46)
            // 4.82, 43 (1.73) 4.69, 37 (2.02) 4.58, 32 (2.31) 4.56.
            double best = 0.0;
            for (int zc = 8; zc <= std::min(nz_, 32 * L.rz); ++zc) {
                const long long ctas = tiles * ((nz_ + zc - 1) / zc);
                if (ctas < 3 * slots) continue;
                const double waves = static_cast<double>(ctas) / static_cast<double>(slots);
                const double score = waves / std::ceil(waves) * zc / (zc + 2.0 * L.rz);
                if (score > best) {
                    best = score;
                    zchunk = zc;
                }
            }
        }
    }
    return std::max(1, zchunk);
}

bool Engine::launch_solve(const gen::Launch& L, float dt, std::string& why)
{
    FePassArgs a;
    std::memset(&a, 0, sizeof(a));
    for (std::size_t k = 0; k < L.sources.size(); ++k) {
        float* p = nullptr;
        if (!buffer(L.sources[k].buf, p)) {
            why = "internal: a pass reads a buffer that does not exist";
            return false;
        }
        a.src[k] = p;
    }
    const int answer = L.outs[0].id;
    unsigned* flag = flags_ + L.flag;
    a.out[0] = slot_[static_cast<std::size_t>(L.aux)];
    a.out[1] = L.kind == gen::Launch::Distance ? slot_[static_cast<std::size_t>(L.aux + 1)] : nullptr;
    a.flag = flag;
    a.err = counts_ + FE_MAX_OUT;
    a.dt = dt;
    a.own_z0 = 0;
    a.own_z1 = nz_;
    if (!cuda_ok(cudaMemsetAsync(flag, 0, sizeof(unsigned), stream_), "flag", why)) return false;
    const unsigned gx = static_cast<unsigned>(std::min<std::size_t>((cells_ + 255) / 256, static_cast<std::size_t>(sms_) * 4));
    a.blocks = static_cast<int>(gx);
    CUfunction fn = function(L.kernel, 0, why);
    if (fn == nullptr) return false;
    void* params[] = {&a};
    ++launches_;
    if (!cu_ok(driver().launchKernel(fn, gx, 1, 1, 256, 1, 1, 0, reinterpret_cast<CUstream>(stream_), params, nullptr), ("launch " + L.kernel).c_str(), why)) {
        return false;
    }
    const float hf = static_cast<float>(h_);
    if (L.kind == gen::Launch::Distance) {
        float* slots[7];
        slots[0] = slot_[static_cast<std::size_t>(answer)];
        for (int k = 0; k < 6; ++k) slots[1 + k] = slot_[static_cast<std::size_t>(L.aux + k)];
        launches_ += 7;
        return cuda_ok(launch_distance_solve(slots, nx_, ny_, nz_, hf, flag, sms_, stream_), "distance", why);
    }
    launches_ += L.iterations + (L.iterations % 2);
    return cuda_ok(launch_poisson_solve(slot_[static_cast<std::size_t>(answer)], slot_[static_cast<std::size_t>(L.aux + 1)],
                       slot_[static_cast<std::size_t>(L.aux)], L.iterations, nx_, ny_, nz_, hf, flag, sms_, stream_),
        "poisson", why);
}

bool Engine::launch(const gen::Launch& L, float dt, int flags, FeCheck* const* recs, std::string& why, const FeCheck* const* carry)
{
    if (L.kind == gen::Launch::Distance || L.kind == gen::Launch::Poisson) return launch_solve(L, dt, why);
    FePassArgs a;
    std::memset(&a, 0, sizeof(a));
    const bool slab = L.kind == gen::Launch::Pass && L.slab;
    for (std::size_t k = 0; k < L.sources.size(); ++k) {
        float* p = nullptr;
        if (!buffer(L.sources[k].buf, p)) {
            why = "internal: a pass reads a buffer that does not exist";
            return false;
        }
        a.src[k] = p;
        if (slab && !map_for(p, 128 + 2 * L.sources[k].ax, L.ty + 2 * L.sources[k].ry, a.map[k], why)) return false;
    }
    for (std::size_t j = 0; j < L.outs.size(); ++j) {
        if (!buffer(L.outs[j], a.out[j])) {
            why = "internal: a pass writes a buffer that does not exist";
            return false;
        }
        const int f = j < L.checked_fields.size() ? L.checked_fields[j] : -1;
        a.rec[j] = (recs != nullptr && f >= 0) ? recs[j] : nullptr;
        a.carry[j] = (a.rec[j] != nullptr && carry != nullptr) ? carry[j] : nullptr;
        // Whatever held the totals of this field's contents no longer does; the caller renews it after a checked gather.
        if (L.outs[j].kind != gen::Buf::Slot && L.outs[j].id >= 0) carry_[static_cast<std::size_t>(L.outs[j].id)] = Carry{};
        a.lo[j] = f >= 0 ? static_cast<float>(law_.fields[static_cast<std::size_t>(f)].lo) : -3.0e38f;
        a.hi[j] = f >= 0 ? static_cast<float>(law_.fields[static_cast<std::size_t>(f)].hi) : 3.0e38f;
    }
    a.own_z0 = own_z0_;
    a.own_z1 = own_z1_;
    a.partials = partials_;
    a.count = counts_;
    a.err = counts_ + FE_MAX_OUT;
    a.dt = dt;
    a.flags = flags;
    void* params[] = {&a};
    unsigned gx = 1, gy = 1, gz = 1, block = 256, smem = 0;
    std::string name = L.kernel;
    switch (L.kind) {
    case gen::Launch::Pass: {
        const int zchunk = zchunk_for(L, slab);
        a.zchunk = zchunk;
        if (slab) {
            gx = static_cast<unsigned>((nx_ + 127) / 128);
            gy = static_cast<unsigned>((ny_ + L.ty - 1) / L.ty);
            smem = L.smem;
        } else {
            name = L.plain_kernel;
            gx = static_cast<unsigned>((nx_ + 31) / 32);
            gy = static_cast<unsigned>((ny_ + 7) / 8);
        }
        gz = static_cast<unsigned>((nz_ + zchunk - 1) / zchunk);
        break;
    }
    case gen::Launch::TridiagX:
        if (L.tri_rows > 0) {
            // A warp a line (y, z), kTriWarps lines a block.
            const unsigned long long lines = static_cast<unsigned long long>(ny_) * nz_;
            gx = static_cast<unsigned>((lines + gen::kTriWarps - 1) / gen::kTriWarps);
            block = 32 * gen::kTriWarps;
        } else {
            gx = static_cast<unsigned>((ny_ + 31) / 32);
            gy = static_cast<unsigned>(nz_);
            block = 32;
        }
        smem = L.smem;
        break;
    case gen::Launch::TridiagYZ: {
        if (L.tri_rows > 0) {
            // 32 consecutive x a block, one block a (z of a y line | y of a z line), tri_segs segments a line.
            gx = static_cast<unsigned>((nx_ + 31) / 32);
            gy = static_cast<unsigned>(L.axis == 1 ? nz_ : ny_);
            block = static_cast<unsigned>(32 * L.tri_segs);
        } else {
            const unsigned long long lines = L.axis == 1 ? static_cast<unsigned long long>(nx_) * nz_ : static_cast<unsigned long long>(nx_) * ny_;
            block = 128;
            gx = static_cast<unsigned>((lines + 127) / 128);
        }
        break;
    }
    case gen::Launch::Reduce:
        block = 256;
        gx = static_cast<unsigned>(std::min<std::size_t>((cells_ + 255) / 256, static_cast<std::size_t>(sms_) * 4));
        break;
    case gen::Launch::Net: {
        // Persistent: one CTA of 128 threads a 128-cell tile, as many CTAs as can hold tensor memory at once.
        const std::size_t tiles = (cells_ + 127) / 128;
        block = 128;
        gx = static_cast<unsigned>(std::min<std::size_t>(tiles, static_cast<std::size_t>(sms_) * static_cast<std::size_t>(L.per_sm)));
        smem = L.smem;
        break;
    }
    case gen::Launch::Distance:
    case gen::Launch::Poisson:
        break; // launch_solve, above
    }
    a.blocks = static_cast<int>(gx * gy * gz);
    if (L.kind == gen::Launch::Pass && (own_z0_ > 0 || own_z1_ < nz_) &&
        std::any_of(L.checked_fields.begin(), L.checked_fields.end(), [](int f) { return f >= 0; })) {
        name += "_halo";
    }
    // Passes and reductions keep per-block partial sums; the solves and net stages keep none.
    const bool partials = L.kind == gen::Launch::Pass || L.kind == gen::Launch::Reduce;
    if (partials && static_cast<std::size_t>(a.blocks) * 4 * FE_MAX_OUT > partial_doubles_) {
        why = "internal: too few partial sums for a launch";
        return false;
    }
    CUfunction fn = function(name, smem, why);
    if (fn == nullptr) return false;
    ++launches_;
    return cu_ok(driver().launchKernel(fn, gx, gy, gz, block, 1, 1, smem, reinterpret_cast<CUstream>(stream_), params, nullptr),
        ("launch " + name).c_str(), why);
}

bool Engine::conserved_by(int term, int field) const
{
    for (const std::vector<int>& group : law_.terms[static_cast<std::size_t>(term)].conserves) {
        for (const int f : group) {
            if (f == field) return true;
        }
    }
    return false;
}

bool Engine::set_param(int id, double value)
{
    if (id < 0 || static_cast<std::size_t>(id) >= param_host_.size()) return false;
    param_host_[static_cast<std::size_t>(id)] = value;
    law_.param_values[static_cast<std::size_t>(id)] = value;
    params_dirty_ = true;
    return true;
}

bool Engine::upload(int field, const void* src, bool device, std::string& why)
{
    if (field < 0 || static_cast<std::size_t>(field) >= now_.size()) {
        why = "no field " + std::to_string(field);
        return false;
    }
    if (!sync(why)) return false;
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    float* dst = now_[static_cast<std::size_t>(field)];
    if (!cuda_ok(cudaMemcpyAsync(dst, src, cells_ * sizeof(float), kind, stream_), "upload", why)) return false;
    // The bounds of what arrived, for the idle-term test (CudaSolver.cpp:820-920 looks over uploaded planes the same
    // way), taken on the card once the cells are there: one read at HBM rate instead of a host loop over every cell.
    // The caller's buffer is read only during the call: measure_bounds waits for the copy.
    return measure_bounds(field, why);
}

bool Engine::measure_bounds(int field, std::string& why)
{
    float* dst = now_[static_cast<std::size_t>(field)];
    FeCheck* rec = bounds_rec_;
    if (!cuda_ok(cudaMemsetAsync(rec, 0, sizeof(FeCheck), stream_), "bounds", why)) return false;
    if (!cuda_ok(launch_bounds(dst, cells_, rec, sms_, stream_), "bounds", why)) return false;
    FeCheck got{};
    if (!cuda_ok(cudaMemcpyAsync(&got, rec, sizeof(FeCheck), cudaMemcpyDeviceToHost, stream_), "bounds", why)) return false;
    if (!cuda_ok(cudaStreamSynchronize(stream_), "bounds", why)) return false;
    Bounds b{};
    const unsigned lo_key = ~got.lo_inv;
    if (got.hi_key != 0u && lo_key != 0xffffffffu) b = Bounds{key_to_float(lo_key), key_to_float(got.hi_key)};
    bounds_[static_cast<std::size_t>(field)] = b;
    zero_[static_cast<std::size_t>(field)] = (b.lo == 0.0 && b.hi == 0.0) ? 1 : 0;
    carry_[static_cast<std::size_t>(field)] = Carry{};
    return true;
}

bool Engine::shift(int dx, int dy, int dz, std::string& why)
{
    if (!sync(why)) return false;
    auto wrap = [](int v, int n) { return ((v % n) + n) % n; };
    dx = wrap(dx, nx_);
    dy = wrap(dy, ny_);
    dz = wrap(dz, nz_);
    if (dx == 0 && dy == 0 && dz == 0) return true;
    if (rotate_scratch_ == nullptr &&
        !cuda_ok(cudaMalloc(reinterpret_cast<void**>(&rotate_scratch_), cells_ * sizeof(float)), "cudaMalloc (window)", why)) {
        return false;
    }
    // Every field's cells and every slot (the stages are recomputed, but distance's seeds and poisson's warm start are
    // kept from step to step and move with the window as a ring's would).
    std::vector<float*> moving(now_.begin(), now_.end());
    moving.insert(moving.end(), slot_.begin(), slot_.end());
    for (float* buf : moving) {
        if (!cuda_ok(launch_rotate(buf, rotate_scratch_, nx_, ny_, nz_, dx, dy, dz, sms_, stream_), "window", why)) return false;
        if (!cuda_ok(cudaMemcpyAsync(buf, rotate_scratch_, cells_ * sizeof(float), cudaMemcpyDeviceToDevice, stream_), "window", why)) {
            return false;
        }
    }
    // The same values, so the same bounds; the totals are summed afresh (in the new cell order).
    carry_.assign(carry_.size(), Carry{});
    return cuda_ok(cudaStreamSynchronize(stream_), "window", why);
}

bool Engine::upload_box(int field, const float* host, const int box[6], std::string& why)
{
    if (field < 0 || static_cast<std::size_t>(field) >= now_.size()) {
        why = "no field " + std::to_string(field);
        return false;
    }
    const int x0 = std::max(0, box[0]), y0 = std::max(0, box[1]), z0 = std::max(0, box[2]);
    const int x1 = std::min(nx_, box[3]), y1 = std::min(ny_, box[4]), z1 = std::min(nz_, box[5]);
    if (x0 >= x1 || y0 >= y1 || z0 >= z1) return true;
    if (!sync(why)) return false;
    float* dst = now_[static_cast<std::size_t>(field)];
    const std::size_t pitch = static_cast<std::size_t>(nx_) * sizeof(float);
    for (int z = z0; z < z1; ++z) {
        const std::size_t at = (static_cast<std::size_t>(z) * ny_ + y0) * nx_ + x0;
        if (!cuda_ok(cudaMemcpy2DAsync(dst + at, pitch, host + at, pitch, static_cast<std::size_t>(x1 - x0) * sizeof(float),
                         static_cast<std::size_t>(y1 - y0), cudaMemcpyHostToDevice, stream_),
                "upload box", why)) {
            return false;
        }
    }
    return measure_bounds(field, why);
}

bool Engine::upload_planes(int field, const float* host, const unsigned char* planes, std::string& why)
{
    if (field < 0 || static_cast<std::size_t>(field) >= now_.size()) {
        why = "no field " + std::to_string(field);
        return false;
    }
    if (!sync(why)) return false;
    float* dst = now_[static_cast<std::size_t>(field)];
    const std::size_t plane = static_cast<std::size_t>(nx_) * ny_;
    bool any = false;
    for (int z = 0; z < nz_;) {
        if (!planes[z]) {
            ++z;
            continue;
        }
        int end = z + 1;
        while (end < nz_ && planes[end]) ++end;
        // A run of flagged planes is one contiguous copy.
        if (!cuda_ok(cudaMemcpyAsync(dst + plane * z, host + plane * z, plane * (end - z) * sizeof(float), cudaMemcpyHostToDevice, stream_),
                "upload planes", why)) {
            return false;
        }
        any = true;
        z = end;
    }
    return !any || measure_bounds(field, why);
}

void Engine::mark_halo(int field)
{
    if (field < 0 || static_cast<std::size_t>(field) >= now_.size()) return;
    bounds_[static_cast<std::size_t>(field)] = Bounds{};
    zero_[static_cast<std::size_t>(field)] = 0;
}

bool Engine::set_owned_z(int z0, int z1)
{
    if (z0 < 0 || z1 > nz_ || z0 >= z1) return false;
    // The totals of a field's current contents were taken over the old range.
    carry_.assign(carry_.size(), Carry{});
    own_z0_ = z0;
    own_z1_ = z1;
    return true;
}

std::vector<GroupTotals> Engine::take_totals()
{
    std::vector<GroupTotals> out;
    out.swap(totals_log_);
    return out;
}

void plan_z_reach(const gen::Plan& plan, int& reach, bool& reductions, bool& z_solves)
{
    reach = 0;
    reductions = false;
    z_solves = false;
    // The planes along z one program reads beyond a cell, summed over its launches in order.
    auto program_reach = [&](const gen::ProgramPlan& pp) {
        int r = 0;
        if (pp.empty) return r;
        auto count = [&](const gen::Launch& L) {
            if (L.kind == gen::Launch::Pass || L.kind == gen::Launch::Net) r += L.rz;
            if (L.kind == gen::Launch::Reduce || L.kind == gen::Launch::Distance || L.kind == gen::Launch::Poisson) reductions = true;
            if (L.kind == gen::Launch::TridiagYZ && L.axis == 2) z_solves = true;
        };
        for (const gen::Launch& L : pp.stages) count(L);
        for (const gen::Launch& L : pp.limit) count(L);
        count(pp.gather);
        return r;
    };
    // A term runs either its learned equations (kept) or its classical ones (the learned step undone, or learned
    // schemes off), never both on the same state: its reach is the larger of the two. The learned programs are
    // scanned even while learned schemes are off, since a caller may turn them on after planning.
    for (std::size_t t = 0; t < plan.terms.size(); ++t) {
        int r = program_reach(plan.terms[t]);
        if (t < plan.learned.size()) r = std::max(r, program_reach(plan.learned[t]));
        reach += r;
    }
    for (const gen::ProgramPlan& pp : plan.derives) reach += program_reach(pp);
}

void Engine::mark_edited(int field)
{
    if (field < 0 || static_cast<std::size_t>(field) >= now_.size()) return;
    bounds_[static_cast<std::size_t>(field)] = Bounds{};
    zero_[static_cast<std::size_t>(field)] = 0;
    carry_[static_cast<std::size_t>(field)] = Carry{};
}

bool Engine::fetch(int field, void* dst, bool device, std::string& why)
{
    if (field < 0 || static_cast<std::size_t>(field) >= now_.size()) {
        why = "no field " + std::to_string(field);
        return false;
    }
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (!cuda_ok(cudaMemcpyAsync(dst, now_[static_cast<std::size_t>(field)], cells_ * sizeof(float), kind, stream_), "fetch", why)) return false;
    return cuda_ok(cudaStreamSynchronize(stream_), "fetch", why);
}

// ---- the idle-term test (LawBounds.cpp:13-213 over the IR) ---------------------------------------------------------------

// One forward pass over the instructions up to `id` (every argument has a lower id than its user), so a value the
// law reuses through lets is bounded once, not once per path to it.
Bounds Engine::bounds_of(int id, const std::vector<Bounds>& fields) const
{
    std::vector<Bounds> memo(static_cast<std::size_t>(id) + 1);
    for (int i = 0; i <= id; ++i) memo[static_cast<std::size_t>(i)] = bounds_one(i, fields, memo);
    return memo[static_cast<std::size_t>(id)];
}

Bounds Engine::bounds_one(int id, const std::vector<Bounds>& fields, const std::vector<Bounds>& memo) const
{
    const ir::Inst& in = mod_.insts[static_cast<std::size_t>(id)];
    auto arg = [&](std::size_t i) { return memo[static_cast<std::size_t>(in.args[i])]; };
    auto clean = [](double lo, double hi) {
        return Bounds{std::isnan(lo) ? -std::numeric_limits<double>::infinity() : lo, std::isnan(hi) ? std::numeric_limits<double>::infinity() : hi};
    };
    auto spread = [](const Bounds& b) { return b.lo == b.hi ? 0.0 : b.hi - b.lo; };
    switch (in.op) {
    case Op::Const: return Bounds{in.number, in.number};
    case Op::Param: {
        const double v = static_cast<float>(law_.param_values[static_cast<std::size_t>(in.index)]);
        return Bounds{v, v};
    }
    case Op::Cell: return Bounds{h_, h_};
    case Op::Rim: return Bounds{0.0, 1.0};
    case Op::Field: return fields[static_cast<std::size_t>(in.index)];
    case Op::Neg: { const Bounds a = arg(0); return Bounds{-a.hi, -a.lo}; }
    case Op::Add: { const Bounds a = arg(0), b = arg(1); return clean(a.lo + b.lo, a.hi + b.hi); }
    case Op::Sub: { const Bounds a = arg(0), b = arg(1); return clean(a.lo - b.hi, a.hi - b.lo); }
    case Op::Mul: {
        const Bounds a = arg(0), b = arg(1);
        const double c[4] = {times(a.lo, b.lo), times(a.lo, b.hi), times(a.hi, b.lo), times(a.hi, b.hi)};
        return Bounds{*std::min_element(c, c + 4), *std::max_element(c, c + 4)};
    }
    case Op::Div: {
        const Bounds a = arg(0), b = arg(1);
        if (a.none() || b.none()) return Bounds{0.0, 0.0};
        if (b.lo <= 0.0 && b.hi >= 0.0) return Bounds{};
        const double c[4] = {a.lo / b.lo, a.lo / b.hi, a.hi / b.lo, a.hi / b.hi};
        return clean(*std::min_element(c, c + 4), *std::max_element(c, c + 4));
    }
    case Op::Pow: {
        const Bounds a = arg(0), b = arg(1);
        if (a.none() && b.lo > 0.0) return Bounds{0.0, 0.0};
        if (a.lo >= 0.0 && b.lo == b.hi && b.lo > 0.0) return clean(std::pow(a.lo, b.lo), std::pow(a.hi, b.lo));
        return Bounds{};
    }
    case Op::Min: { const Bounds a = arg(0), b = arg(1); return Bounds{std::min(a.lo, b.lo), std::min(a.hi, b.hi)}; }
    case Op::Max: { const Bounds a = arg(0), b = arg(1); return Bounds{std::max(a.lo, b.lo), std::max(a.hi, b.hi)}; }
    case Op::Abs: {
        const Bounds a = arg(0);
        const double most = std::max(std::abs(a.lo), std::abs(a.hi));
        return Bounds{a.lo <= 0.0 && a.hi >= 0.0 ? 0.0 : std::min(std::abs(a.lo), std::abs(a.hi)), most};
    }
    case Op::Sqrt: { const Bounds a = arg(0); return Bounds{std::sqrt(std::max(0.0, a.lo)), std::sqrt(std::max(0.0, a.hi))}; }
    case Op::Exp: { const Bounds a = arg(0); return Bounds{std::exp(std::min(a.lo, 80.0)), std::exp(std::min(a.hi, 80.0))}; }
    case Op::Log: { const Bounds a = arg(0); return Bounds{std::log(std::max(a.lo, 1e-30)), std::log(std::max(a.hi, 1e-30))}; }
    case Op::Step: { const Bounds a = arg(0); return Bounds{a.lo > 0.0 ? 1.0 : 0.0, a.hi > 0.0 ? 1.0 : 0.0}; }
    case Op::Pos: { const Bounds a = arg(0); return Bounds{std::max(a.lo, 0.0), std::max(a.hi, 0.0)}; }
    case Op::Clamp: {
        const Bounds a = arg(0), lo = arg(1), hi = arg(2);
        return Bounds{std::min(std::max(a.lo, lo.lo), std::max(lo.hi, hi.hi)), std::min(std::max(a.hi, lo.hi), std::max(lo.hi, hi.hi))};
    }
    case Op::Shift: case Op::MaxOf: case Op::MinOf: return arg(0);
    case Op::Lap: { const double most = 6.0 * spread(arg(0)) / (h_ * h_); return Bounds{-most, most}; }
    case Op::Gx: case Op::Gy: case Op::Gz: { const double most = spread(arg(0)) / h_; return Bounds{-most, most}; }
    case Op::Diffuse: {
        const Bounds k = arg(0);
        const double most = times(12.0 * std::max(std::abs(k.lo), std::abs(k.hi)), spread(arg(1))) / (h_ * h_);
        return Bounds{-most, most};
    }
    case Op::Adv: case Op::Fall: case Op::Spread: case Op::Topple: case Op::SumOf: {
        const Bounds a = arg(0);
        return a.none() ? a : Bounds{};
    }
    default:
        return Bounds{};
    }
}

bool Engine::always_zero(int id) const
{
    std::vector<char> memo(static_cast<std::size_t>(id) + 1, 0);
    for (int i = 0; i <= id; ++i) memo[static_cast<std::size_t>(i)] = zero_one(i, memo) ? 1 : 0;
    return memo[static_cast<std::size_t>(id)] != 0;
}

bool Engine::zero_one(int id, const std::vector<char>& memo) const
{
    const ir::Inst& in = mod_.insts[static_cast<std::size_t>(id)];
    auto arg = [&](std::size_t i) { return memo[static_cast<std::size_t>(in.args[i])] != 0; };
    switch (in.op) {
    case Op::Const: return in.number == 0.0;
    case Op::Param: return law_.param_values[static_cast<std::size_t>(in.index)] == 0.0;
    case Op::Field: return zero_[static_cast<std::size_t>(in.index)] != 0;
    case Op::Neg: case Op::Abs: case Op::Sqrt: case Op::Step: case Op::Pos: case Op::Shift: case Op::Lap: case Op::Gx: case Op::Gy:
    case Op::Gz: case Op::MaxOf: case Op::MinOf: case Op::SumOf:
        return arg(0);
    case Op::Mul: case Op::Div: return arg(0) || arg(1);
    case Op::Add: case Op::Sub: case Op::Min: case Op::Max: return arg(0) && arg(1);
    case Op::Diffuse: return arg(0) || arg(1);
    case Op::Adv: case Op::Fall: case Op::Spread: case Op::Topple: return arg(0);
    default: return false;
    }
}

bool Engine::idle(const ir::Program& p) const
{
    return std::all_of(p.equations.begin(), p.equations.end(),
        [&](const ir::Equation& eq) { return always_zero(eq.value) || bounds_of(eq.value, bounds_).none(); });
}

// What a term of `substeps` Euler substeps may have done to the bounds of what it writes (LawBounds.cpp:219-268).
void Engine::flow_bounds(const ir::Program& p, double dt, int substeps)
{
    const int n = std::max(substeps, 1);
    const double sub = dt / n;
    const std::vector<Bounds> before = bounds_;
    for (int s = 0; s < n; ++s) {
        const std::vector<Bounds> start = bounds_;
        std::vector<Bounds> now = bounds_;
        for (int round = 0; round < 2; ++round) {
            std::vector<Bounds> next = now;
            for (const ir::Equation& eq : p.equations) {
                const ir::Inst& in = mod_.insts[static_cast<std::size_t>(eq.value)];
                const bool within = in.op == Op::Diffuse && mod_.insts[static_cast<std::size_t>(in.args[1])].op == Op::Field &&
                    mod_.insts[static_cast<std::size_t>(in.args[1])].index == eq.target;
                if (within) continue;
                const auto t = static_cast<std::size_t>(eq.target);
                const Bounds rate = bounds_of(eq.value, now);
                next[t].lo = std::min(next[t].lo, start[t].lo + times(sub, std::min(rate.lo, 0.0)));
                next[t].hi = std::max(next[t].hi, start[t].hi + times(sub, std::max(rate.hi, 0.0)));
            }
            now = std::move(next);
        }
        bool moved = false;
        for (std::size_t f = 0; f < now.size() && !moved; ++f) moved = now[f].lo != bounds_[f].lo || now[f].hi != bounds_[f].hi;
        bounds_ = std::move(now);
        if (!moved) break;
    }
    for (const ir::Equation& eq : p.equations) {
        const auto t = static_cast<std::size_t>(eq.target);
        const law::FieldDecl& decl = law_.fields[t];
        Bounds& b = bounds_[t];
        if (b.lo != before[t].lo || b.hi != before[t].hi) {
            b.lo -= 1e-6 * n * std::abs(b.lo);
            b.hi += 1e-6 * n * std::abs(b.hi);
        }
        if (decl.clamp) {
            b.lo = std::clamp(b.lo, decl.lo, decl.hi);
            b.hi = std::clamp(b.hi, decl.lo, decl.hi);
        }
        zero_[t] = (b.lo == 0.0 && b.hi == 0.0) ? 1 : 0;
    }
}

// A max_dt on the host: numbers, params, h, and reductions read back from the card (CudaSolver.cpp:450-488).
double Engine::scalar_value(int id, bool& ok, std::string& why)
{
    const ir::Inst& in = mod_.insts[static_cast<std::size_t>(id)];
    auto a = [&](std::size_t k) { return scalar_value(in.args[k], ok, why); };
    switch (in.op) {
    case Op::Const: return in.number;
    case Op::Param: return law_.param_values[static_cast<std::size_t>(in.index)];
    case Op::Cell: return h_;
    case Op::Neg: return -a(0);
    case Op::Abs: return std::abs(a(0));
    case Op::Sqrt: return std::sqrt(std::max(0.0, a(0)));
    case Op::Exp: return std::exp(std::min(a(0), 80.0));
    case Op::Log: return std::log(std::max(a(0), 1e-30));
    case Op::Step: return a(0) > 0.0 ? 1.0 : 0.0;
    case Op::Pos: return std::max(a(0), 0.0);
    case Op::Add: return a(0) + a(1);
    case Op::Sub: return a(0) - a(1);
    case Op::Mul: return a(0) * a(1);
    case Op::Div: { const double b = a(1); return b == 0.0 ? 0.0 : a(0) / b; }
    case Op::Pow: return std::pow(a(0), a(1));
    case Op::Min: return std::min(a(0), a(1));
    case Op::Max: return std::max(a(0), a(1));
    case Op::Clamp: { const double lo = a(1); return std::clamp(a(0), lo, std::max(lo, a(2))); }
    case Op::MaxOf: case Op::MinOf: case Op::SumOf: {
        const int u = plan_.uniform_of[static_cast<std::size_t>(id)];
        if (u < 0) return 0.0;
        float value = 0.0f;
        if (!cuda_ok(cudaMemcpyAsync(&value, reinterpret_cast<const char*>(uniforms_) + 4 * u, 4, cudaMemcpyDeviceToHost, stream_), "uniform", why) ||
            !cuda_ok(cudaStreamSynchronize(stream_), "uniform", why)) {
            ok = false;
        }
        return value;
    }
    default:
        return 0.0;
    }
}

bool Engine::run_program(int index, const ir::Program& p, const gen::ProgramPlan& pp, double dt, bool respect, bool check,
    PendingStep& pending, std::string& why)
{
    TermProfile& tp = term_profile_[static_cast<std::size_t>(index)];
    tp = TermProfile{};
    const int launches_before = launches_;
    substeps_[static_cast<std::size_t>(index)] = 1;
    if (pp.empty) return true;
    if (idle(p)) {
        tp.idle = true;
        return true;
    }
    int count = 1;
    if (respect && p.max_dt >= 0) {
        for (const gen::Launch& L : pp.limit) {
            if (!launch(L, 0.0f, 0, nullptr, why)) return false;
        }
        bool ok = true;
        const double limit = scalar_value(p.max_dt, ok, why);
        if (!ok) return false;
        if (limit > 0.0 && std::isfinite(limit) && dt > limit) {
            const double wanted = std::ceil(dt / limit);
            if (wanted > kMaxSubsteps) {
                Violation v;
                v.kind = 3;
                v.term = index;
                v.step = steps_;
                v.detail = "max_dt " + std::to_string(limit) + " asks for " + std::to_string(wanted) + " substeps; capped at " +
                    std::to_string(kMaxSubsteps);
                violations_.push_back(v);
                count = kMaxSubsteps;
            } else {
                count = static_cast<int>(wanted);
            }
        }
    }
    substeps_[static_cast<std::size_t>(index)] = count;
    const float sub_dt = static_cast<float>(dt / count);
    FeCheck* recs[FE_MAX_OUT] = {};
    const FeCheck* carried[FE_MAX_OUT] = {};
    int rec_index[FE_MAX_OUT] = {};
    if (check) {
        for (std::size_t j = 0; j < pp.gather.outs.size(); ++j) {
            const int r = static_cast<int>(pending.refs.size());
            const int f = pp.gather.checked_fields[j];
            rec_index[j] = r;
            recs[j] = records_ + static_cast<std::size_t>(pending.ring) * records_per_step_ + r;
            pending.refs.push_back(RecordRef{index, f, r, count, true});
            if (f < 0) continue;
            // The totals before the term: those after the checked pass that last wrote the field (still in the ring),
            // else, for a conserved field, summed now.
            const Carry& c = carry_[static_cast<std::size_t>(f)];
            if (c.step >= 0 && steps_ - c.step < ring_ - 2) {
                carried[j] = records_ + static_cast<std::size_t>(c.ring) * records_per_step_ + c.rec;
            } else if (conserved_by(index, f)) {
                const std::size_t plane = static_cast<std::size_t>(nx_) * ny_;
                if (!cuda_ok(launch_totals(now_[static_cast<std::size_t>(f)] + plane * own_z0_, plane * (own_z1_ - own_z0_), recs[j], partials_,
                                 counts_ + FE_MAX_OUT + 1, stream_),
                        "totals", why)) {
                    return false;
                }
            }
        }
    }
    for (int s = 0; s < count; ++s) {
        for (const gen::Launch& L : pp.stages) {
            if (!launch(L, sub_dt, 0, nullptr, why)) return false;
        }
        const int flags = s == count - 1 ? FE_PASS_AFTER | FE_PASS_RANGE : 0;
        if (!launch(pp.gather, sub_dt, flags, check ? recs : nullptr, why, s == 0 ? carried : nullptr)) return false;
        for (const int f : pp.swaps) std::swap(now_[static_cast<std::size_t>(f)], next_[static_cast<std::size_t>(f)]);
    }
    if (check) {
        for (std::size_t j = 0; j < pp.gather.outs.size(); ++j) {
            const int f = pp.gather.checked_fields[j];
            if (f >= 0) carry_[static_cast<std::size_t>(f)] = Carry{pending.ring, rec_index[j], steps_};
        }
    }
    flow_bounds(p, dt, count);
    tp.launches = launches_ - launches_before;
    tp.substeps = count;
    return true;
}

bool Engine::push_params(std::string& why)
{
    std::vector<float> p(1024, 0.0f);
    for (std::size_t i = 0; i < param_host_.size() && i < 1024; ++i) p[i] = static_cast<float>(param_host_[i]);
    if (!cuda_ok(cudaMemcpyAsync(reinterpret_cast<void*>(params_), p.data(), 1024 * sizeof(float), cudaMemcpyHostToDevice, stream_), "params", why) ||
        !cuda_ok(cudaStreamSynchronize(stream_), "params", why)) {
        return false;
    }
    params_dirty_ = false;
    return true;
}

bool Engine::step(double dt, bool respect_max_dt, std::string& why)
{
    if (!deferred_) violations_.clear();
    launches_ = 0;
    if (params_dirty_ && !push_params(why)) return false;
    const bool check = (steps_ % check_every_) == 0;
    PendingStep pending;
    pending.step = steps_;
    pending.ring = ring_next_;
    if (check) {
        ring_next_ = (ring_next_ + 1) % ring_;
        if (records_per_step_ > 0 &&
            !cuda_ok(cudaMemsetAsync(records_ + static_cast<std::size_t>(pending.ring) * records_per_step_, 0, sizeof(FeCheck) * records_per_step_, stream_),
                "records", why)) {
            return false;
        }
    }
    cudaEventRecord(ev0_, stream_);
    fallbacks_ = 0;
    for (std::size_t t = 0; t < mod_.terms.size(); ++t) {
        if (!apply_term(static_cast<int>(t), dt, respect_max_dt, check, pending, why)) return false;
    }
    for (std::size_t d = 0; d < mod_.derives.size(); ++d) {
        const gen::ProgramPlan& pp = plan_.derives[d];
        if (pp.empty) continue;
        FeCheck* recs[FE_MAX_OUT] = {};
        if (check) {
            const int r = static_cast<int>(pending.refs.size());
            recs[0] = records_ + static_cast<std::size_t>(pending.ring) * records_per_step_ + r;
            pending.refs.push_back(RecordRef{-1, pp.gather.checked_fields[0], r, 1, false});
        }
        for (const gen::Launch& L : pp.stages) {
            if (!launch(L, 0.0f, 0, nullptr, why)) return false;
        }
        if (!launch(pp.gather, 0.0f, FE_PASS_RANGE, check ? recs : nullptr, why)) return false;
        for (const int f : pp.swaps) std::swap(now_[static_cast<std::size_t>(f)], next_[static_cast<std::size_t>(f)]);
    }
    cudaEventRecord(ev1_, stream_);
    ++steps_;
    gpu_ms_ = 0.0;
    if (!check) return cuda_ok(cudaPeekAtLastError(), "step", why);
    pending_.push_back(std::move(pending));
    if (!deferred_ || static_cast<int>(pending_.size()) >= ring_ - 1) {
        if (!sync(why)) return false;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess) gpu_ms_ = ms;
    }
    return true;
}

bool Engine::derive(std::string& why)
{
    for (std::size_t d = 0; d < mod_.derives.size(); ++d) {
        const gen::ProgramPlan& pp = plan_.derives[d];
        if (pp.empty) continue;
        for (const gen::Launch& L : pp.stages) {
            if (!launch(L, 0.0f, 0, nullptr, why)) return false;
        }
        if (!launch(pp.gather, 0.0f, 0, nullptr, why)) return false;
        for (const int f : pp.swaps) std::swap(now_[static_cast<std::size_t>(f)], next_[static_cast<std::size_t>(f)]);
    }
    return cuda_ok(cudaStreamSynchronize(stream_), "derive", why);
}

bool Engine::sync(std::string& why)
{
    if (!cuda_ok(cudaStreamSynchronize(stream_), "sync", why)) return false;
    unsigned err = 0;
    if (!cuda_ok(cudaMemcpy(&err, counts_ + FE_MAX_OUT, 4, cudaMemcpyDeviceToHost), "error word", why)) return false;
    if (err != 0) {
        why = "a kernel raised error word " + std::to_string(err) + " (a bounded wait gave up)";
        return false;
    }
    for (std::size_t i = 0; i < pending_.size(); ++i) {
        if (!judge(pending_[i], why)) return false;
        if (i + 1 == pending_.size()) {
            // The latest step's records are the fields' exact bounds now.
            std::vector<FeCheck> recs(static_cast<std::size_t>(std::max(1, records_per_step_)));
            cudaMemcpy(recs.data(), records_ + static_cast<std::size_t>(pending_[i].ring) * records_per_step_, sizeof(FeCheck) * records_per_step_,
                cudaMemcpyDeviceToHost);
            for (const RecordRef& r : pending_[i].refs) {
                const FeCheck& c = recs[static_cast<std::size_t>(r.rec)];
                if (r.field < 0) continue;
                const unsigned lo_key = ~c.lo_inv;
                if (c.hi_key != 0u && lo_key != 0xffffffffu) {
                    bounds_[static_cast<std::size_t>(r.field)] = Bounds{key_to_float(lo_key), key_to_float(c.hi_key)};
                    zero_[static_cast<std::size_t>(r.field)] = (key_to_float(lo_key) == 0.0f && key_to_float(c.hi_key) == 0.0f) ? 1 : 0;
                }
            }
        }
    }
    pending_.clear();
    return true;
}

// The host's judgement of one step's records (CudaSolver.cpp:530-571; the tolerance is Solver.cpp:439-453's).
bool Engine::apply_term(int t, double dt, bool respect, bool check, PendingStep& pending, std::string& why)
{
    const std::size_t ti = static_cast<std::size_t>(t);
    const bool guarded = learned_ && ti < mod_.learned.size() && !mod_.learned[ti].equations.empty() && ti < plan_.learned.size() &&
        !plan_.learned[ti].empty;
    if (!guarded) return run_program(t, mod_.terms[ti], plan_.terms[ti], dt, respect, check, pending, why);
    // GUARDED: what the term writes goes aside; the learned scheme runs with its contracts checked and judged now.
    const ir::Program& lp = mod_.learned[ti];
    std::vector<int> writes = lp.writes;
    for (const int w : mod_.terms[ti].writes) {
        if (std::find(writes.begin(), writes.end(), w) == writes.end()) writes.push_back(w);
    }
    if (snapshot_fields_ < writes.size()) {
        if (snapshot_ != nullptr) cudaFree(snapshot_);
        snapshot_ = nullptr;
        snapshot_fields_ = 0;
        if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&snapshot_), writes.size() * cells_ * sizeof(float)), "cudaMalloc (snapshot)", why)) return false;
        snapshot_fields_ = writes.size();
    }
    for (std::size_t w = 0; w < writes.size(); ++w) {
        if (!cuda_ok(cudaMemcpyAsync(snapshot_ + w * cells_, now_[static_cast<std::size_t>(writes[w])], cells_ * sizeof(float), cudaMemcpyDeviceToDevice,
                         stream_),
                "snapshot", why)) {
            return false;
        }
    }
    const std::vector<Bounds> bounds_before = bounds_;
    const std::vector<char> zero_before = zero_;
    const std::size_t mark = pending.refs.size();
    // Its records start empty (on an unchecked step the slot was not cleared for it).
    if (!cuda_ok(cudaMemsetAsync(records_ + static_cast<std::size_t>(pending.ring) * records_per_step_ + mark, 0,
                     plan_.learned[ti].gather.outs.size() * sizeof(FeCheck), stream_),
            "records", why)) {
        return false;
    }
    if (!run_program(t, lp, plan_.learned[ti], dt, respect, true, pending, why)) return false;
    std::vector<Violation> broken;
    if (pending.refs.size() > mark) {
        if (!cuda_ok(cudaStreamSynchronize(stream_), "guard", why)) return false;
        PendingStep trial;
        trial.step = pending.step;
        trial.ring = pending.ring;
        trial.refs.assign(pending.refs.begin() + static_cast<std::ptrdiff_t>(mark), pending.refs.end());
        if (!judge_into(trial, broken, why)) return false;
    }
    TermProfile& tp = term_profile_[ti];
    if (broken.empty()) {
        tp.learned = !tp.idle;
        if (!check) pending.refs.resize(mark); // an unchecked step keeps no records of it
        return true;
    }
    // Undo it: the snapshot back, its records cleared, the bounds as they were; then the classical scheme.
    for (std::size_t w = 0; w < writes.size(); ++w) {
        const std::size_t f = static_cast<std::size_t>(writes[w]);
        if (!cuda_ok(cudaMemcpyAsync(now_[f], snapshot_ + w * cells_, cells_ * sizeof(float), cudaMemcpyDeviceToDevice, stream_), "undo", why)) return false;
        carry_[f] = Carry{};
    }
    const std::size_t used = pending.refs.size() - mark;
    if (!cuda_ok(cudaMemsetAsync(records_ + static_cast<std::size_t>(pending.ring) * records_per_step_ + mark, 0, used * sizeof(FeCheck), stream_), "records",
            why)) {
        return false;
    }
    pending.refs.resize(mark);
    bounds_ = bounds_before;
    zero_ = zero_before;
    ++fallbacks_;
    if (!run_program(t, mod_.terms[ti], plan_.terms[ti], dt, respect, check, pending, why)) return false;
    term_profile_[ti].fell_back = true;
    return true;
}

bool Engine::judge(PendingStep& pending, std::string& why)
{
    return judge_into(pending, violations_, why);
}

bool Engine::judge_into(const PendingStep& pending, std::vector<Violation>& out, std::string& why)
{
    if (pending.refs.empty()) return true;
    std::vector<FeCheck> recs(static_cast<std::size_t>(records_per_step_));
    if (!cuda_ok(cudaMemcpy(recs.data(), records_ + static_cast<std::size_t>(pending.ring) * records_per_step_, sizeof(FeCheck) * records_per_step_,
                     cudaMemcpyDeviceToHost),
            "records", why)) {
        return false;
    }
    // Conservation, per term and group.
    for (std::size_t t = 0; t < law_.terms.size(); ++t) {
        const law::Term& term = law_.terms[t];
        for (const std::vector<int>& group : term.conserves) {
            double before = 0.0, after = 0.0, scale = 0.0;
            int substeps = 1;
            bool any = false;
            for (const int f : group) {
                for (const RecordRef& r : pending.refs) {
                    if (r.term == static_cast<int>(t) && r.field == f) {
                        const FeCheck& c = recs[static_cast<std::size_t>(r.rec)];
                        before += c.before;
                        after += c.after;
                        scale += c.before_abs;
                        substeps = r.substeps;
                        any = true;
                    }
                }
            }
            if (!any) continue; // the term was idle: nothing moved
            if (external_conservation_) {
                totals_log_.push_back(GroupTotals{pending.step, static_cast<int>(t), static_cast<int>(&group - term.conserves.data()), substeps, before,
                    after, scale});
                continue;
            }
            const double tolerance = 1e-5 * (scale + 1.0) * std::sqrt(static_cast<double>(substeps));
            if (std::abs(after - before) > tolerance) {
                Violation v;
                v.kind = 2;
                v.term = static_cast<int>(t);
                v.field = group.front();
                v.before = before;
                v.after = after;
                v.tolerance = tolerance;
                v.step = pending.step;
                std::ostringstream d;
                d << "total went " << before << " -> " << after << " (tolerance " << tolerance << ")";
                v.detail = d.str();
                out.push_back(v);
            }
        }
    }
    // Range and NaN, per written field.
    for (const RecordRef& r : pending.refs) {
        const FeCheck& c = recs[static_cast<std::size_t>(r.rec)];
        if (c.out_of_range == 0 && c.not_finite == 0) continue;
        Violation v;
        v.kind = c.not_finite != 0 ? 1 : 0;
        v.term = r.term;
        v.field = r.field;
        v.count = c.out_of_range + c.not_finite;
        v.first_cell = ~c.first_bad;
        v.step = pending.step;
        const law::FieldDecl& decl = law_.fields[static_cast<std::size_t>(r.field)];
        const unsigned first = v.first_cell;
        std::ostringstream d;
        d << v.count << " cell(s); first " << decl.name << " at (" << first % nx_ << "," << (first / nx_) % ny_ << "," << first / (static_cast<unsigned>(nx_) * ny_)
          << "), declared range [" << decl.lo << ", " << decl.hi << "]";
        v.detail = d.str();
        out.push_back(v);
    }
    return true;
}

bool Engine::time_gather(int term, int launches, float& ms, std::string& why)
{
    if (term < 0 || static_cast<std::size_t>(term) >= plan_.terms.size() || plan_.terms[static_cast<std::size_t>(term)].empty) {
        why = "no such term";
        return false;
    }
    const gen::ProgramPlan& pp = plan_.terms[static_cast<std::size_t>(term)];
    FeCheck* recs[FE_MAX_OUT] = {};
    for (std::size_t j = 0; j < pp.gather.outs.size(); ++j) recs[j] = records_ + j; // scratch records (ring slot 0)
    // Ring slot 0 no longer holds what a carried total points at.
    carry_.assign(carry_.size(), Carry{});
    cudaEventRecord(ev0_, stream_);
    for (int i = 0; i < launches; ++i) {
        if (!launch(pp.gather, static_cast<float>(0.0), FE_PASS_AFTER | FE_PASS_RANGE, recs, why)) return false;
    }
    cudaEventRecord(ev1_, stream_);
    if (!cuda_ok(cudaEventSynchronize(ev1_), "time", why)) return false;
    return cuda_ok(cudaEventElapsedTime(&ms, ev0_, ev1_), "time", why);
}

bool Engine::time_stage(int term, int stage, int launches, double dt, float& ms, std::string& kernel, std::string& why)
{
    if (term < 0 || static_cast<std::size_t>(term) >= plan_.terms.size() || plan_.terms[static_cast<std::size_t>(term)].empty) {
        why = "no such term";
        return false;
    }
    const gen::ProgramPlan& pp = plan_.terms[static_cast<std::size_t>(term)];
    if (stage < 0 || static_cast<std::size_t>(stage) >= pp.stages.size()) {
        why = "no such stage";
        return false;
    }
    const gen::Launch& L = pp.stages[static_cast<std::size_t>(stage)];
    kernel = L.kernel;
    if (params_dirty_ && !push_params(why)) return false;
    FeCheck* recs[FE_MAX_OUT] = {};
    cudaEventRecord(ev0_, stream_);
    for (int i = 0; i < launches; ++i) {
        if (!launch(L, static_cast<float>(dt), 0, recs, why)) return false;
    }
    cudaEventRecord(ev1_, stream_);
    if (!cuda_ok(cudaEventSynchronize(ev1_), "time", why)) return false;
    return cuda_ok(cudaEventElapsedTime(&ms, ev0_, ev1_), "time", why);
}

} // namespace fe
