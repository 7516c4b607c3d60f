// Many instances of one law on uneven lattices, stepped together (include/fe.h, "batched instances").
//
// The reference batches only what fits one lattice: every instance a z-plane (or a run of planes) of one grid, all of
// the same nx x ny (bench/finance.py:253-288, bench/pdebench.py:71-92). Here instances may differ in every extent and in
// h. Instances of equal (nx, ny, h) share one lattice, stacked along z, when the law couples nothing along z (no value
// read across planes, no lattice-wide reduction, distance or poisson, no solve along z, no `rim`, which marks the
// lattice's z faces): the reference's convention, with each instance's own depth. Otherwise an instance is a lattice of
// its own. Each lattice is a law handle with its own stream; a batch step launches every lattice's step without waiting
// (deferred judging), then judges them all, so lattices too small to fill the GPU run side by side.
#include "../../include/fe.h"

#include "api_common.hpp"
#include "codegen.hpp"
#include "engine.hpp"
#include "ir.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

struct fe_batch {
    struct Lattice {
        fe_law* law = nullptr;
        int nx = 0, ny = 0, nz = 0;
        double h = 0.0;
        std::vector<int> members; // instances, in the order their planes are stacked
        int seen = 0;             // violations the handle held after the last batch step (deferred judging keeps them)
    };
    struct Where {
        int lattice = 0;
        int z0 = 0, nz = 0;       // the instance's planes in its lattice
    };
    std::vector<Lattice> lattices;
    std::vector<Where> where;     // per instance
    std::vector<std::pair<int, fe_violation>> violations; // (instance, record); -1: the whole lattice (a conserved total)
    bool stacked = false;

    ~fe_batch()
    {
        for (Lattice& l : lattices) {
            if (l.law != nullptr) fe_law_destroy(l.law);
        }
    }
};

namespace {

// Whether the law's step on a lattice leaves every z-plane's update to that plane alone (*independent); FE_ELAW when
// the law does not compile, FE_EUNSUP when this backend cannot run it.
int planes_independent(const char* law_text, int nx, int ny, double h, bool* independent)
{
    std::vector<std::string> errors;
    const fe::law::Law law = fe::law::compile({fe::law::Source{"law", law_text}}, errors);
    if (!errors.empty()) {
        std::string why;
        for (const std::string& e : errors) why += e + "\n";
        return fe::fail(FE_ELAW, why);
    }
    const fe::ir::Module m = fe::ir::lower(law);
    fe::gen::Plan plan;
    std::string why;
    if (!fe::gen::generate(m, law, nx, ny, 2, h, plan, why)) return fe::fail(FE_EUNSUP, why);
    int reach = 0;
    bool reductions = false, z_solves = false;
    fe::plan_z_reach(plan, reach, reductions, z_solves);
    const bool rim = std::any_of(m.insts.begin(), m.insts.end(), [](const fe::ir::Inst& in) { return in.op == fe::law::Op::Rim; });
    *independent = reach == 0 && !reductions && !z_solves && !rim;
    return fe::ok();
}

// Which lattice each instance goes into (equal nx, ny, h stacked when the planes are independent), the lattices'
// extents, and each instance's first plane.
struct Grouping {
    bool stacked = false;
    std::vector<fe_batch::Lattice> lattices;
    std::vector<fe_batch::Where> where;
};

int group_instances(const char* law_text, const fe_batch_desc* descs, int n, Grouping& g)
{
    if (law_text == nullptr || descs == nullptr || n < 1) return fe::fail(FE_EINVAL, "fe_batch: bad argument");
    for (int i = 0; i < n; ++i) {
        if (descs[i].nx < 1 || descs[i].ny < 1 || descs[i].nz < 1 || !(descs[i].h > 0.0)) {
            return fe::fail(FE_EINVAL, "fe_batch: instance " + std::to_string(i) + " has a bad lattice");
        }
    }
    const int rc = planes_independent(law_text, descs[0].nx, descs[0].ny, descs[0].h, &g.stacked);
    if (rc != FE_OK) return rc;
    g.where.resize(static_cast<std::size_t>(n));
    std::map<std::tuple<int, int, double>, int> by_shape;
    for (int i = 0; i < n; ++i) {
        const fe_batch_desc& d = descs[i];
        int at = -1;
        if (g.stacked) {
            const auto key = std::make_tuple(d.nx, d.ny, d.h);
            const auto found = by_shape.find(key);
            if (found != by_shape.end()) at = found->second;
            else by_shape.emplace(key, at = static_cast<int>(g.lattices.size()));
        }
        if (at < 0 || static_cast<std::size_t>(at) == g.lattices.size()) {
            at = static_cast<int>(g.lattices.size());
            fe_batch::Lattice l;
            l.nx = d.nx;
            l.ny = d.ny;
            l.h = d.h;
            g.lattices.push_back(l);
        }
        fe_batch::Lattice& l = g.lattices[static_cast<std::size_t>(at)];
        g.where[static_cast<std::size_t>(i)] = fe_batch::Where{at, l.nz, d.nz};
        l.nz += d.nz;
        l.members.push_back(i);
    }
    return fe::ok();
}

bool instance_ok(const fe_batch* b, int instance)
{
    return b != nullptr && instance >= 0 && static_cast<std::size_t>(instance) < b->where.size();
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fe::fail(FE_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// The instance's planes of a field: host <-> the lattice's current device buffer, on the lattice's stream.
int transfer(fe_batch* b, int instance, int field, float* host, bool up)
{
    if (!instance_ok(b, instance)) return fe::fail(FE_EINVAL, "no such instance");
    const fe_batch::Where& w = b->where[static_cast<std::size_t>(instance)];
    fe_batch::Lattice& l = b->lattices[static_cast<std::size_t>(w.lattice)];
    if (field < 0 || field >= fe_law_field_count(l.law)) return fe::fail(FE_EINVAL, "bad field");
    const float* dev = nullptr;
    int rc = fe_law_field_device_ptr(l.law, field, &dev);
    if (rc != FE_OK) return rc;
    void* stream = nullptr;
    if ((rc = fe_law_stream(l.law, &stream)) != FE_OK) return rc;
    const std::size_t plane = static_cast<std::size_t>(l.nx) * l.ny;
    float* at = const_cast<float*>(dev) + plane * static_cast<std::size_t>(w.z0);
    const std::size_t bytes = plane * static_cast<std::size_t>(w.nz) * sizeof(float);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Whatever the lattice's last step queued comes first.
    cudaError_t e = up ? cudaMemcpyAsync(at, host, bytes, cudaMemcpyHostToDevice, s) : cudaMemcpyAsync(host, at, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, up ? "fe_batch_upload" : "fe_batch_fetch");
    return up ? fe_law_mark_edited(l.law, field) : fe::ok();
}

} // namespace

extern "C" {

int fe_batch_create(const char* law_text, const fe_batch_desc* descs, int n, fe_batch** out)
{
    if (out == nullptr) return fe::fail(FE_EINVAL, "fe_batch_create: null argument");
    *out = nullptr;
    Grouping g;
    int rc = group_instances(law_text, descs, n, g);
    if (rc != FE_OK) return rc;
    auto b = std::make_unique<fe_batch>();
    b->stacked = g.stacked;
    b->where = std::move(g.where);
    b->lattices = std::move(g.lattices);
    for (fe_batch::Lattice& l : b->lattices) {
        if ((rc = fe_law_create(law_text, "batch", l.nx, l.ny, l.nz, l.h, &l.law)) != FE_OK) return rc;
        if ((rc = fe_law_set_deferred(l.law, 1)) != FE_OK) return rc;
    }
    *out = b.release();
    return fe::ok();
}

int fe_batch_plan(const char* law_text, const fe_batch_desc* descs, int n, int* lattices, int* stacked, int* lattice_of, int* z0)
{
    Grouping g;
    const int rc = group_instances(law_text, descs, n, g);
    if (rc != FE_OK) return rc;
    if (lattices != nullptr) *lattices = static_cast<int>(g.lattices.size());
    if (stacked != nullptr) *stacked = g.stacked ? 1 : 0;
    for (int i = 0; i < n; ++i) {
        if (lattice_of != nullptr) lattice_of[i] = g.where[static_cast<std::size_t>(i)].lattice;
        if (z0 != nullptr) z0[i] = g.where[static_cast<std::size_t>(i)].z0;
    }
    return fe::ok();
}

void fe_batch_destroy(fe_batch* b)
{
    delete b;
}

int fe_batch_info(const fe_batch* b, int* lattices, int* stacked)
{
    if (b == nullptr) return fe::fail(FE_EINVAL, "null handle");
    if (lattices != nullptr) *lattices = static_cast<int>(b->lattices.size());
    if (stacked != nullptr) *stacked = b->stacked ? 1 : 0;
    return fe::ok();
}

int fe_batch_law(fe_batch* b, int instance, fe_law** law, int* z0)
{
    if (!instance_ok(b, instance) || law == nullptr) return fe::fail(FE_EINVAL, "fe_batch_law: bad argument");
    const fe_batch::Where& w = b->where[static_cast<std::size_t>(instance)];
    *law = b->lattices[static_cast<std::size_t>(w.lattice)].law;
    if (z0 != nullptr) *z0 = w.z0;
    return fe::ok();
}

int fe_batch_set_param(fe_batch* b, int param, double value)
{
    if (b == nullptr) return fe::fail(FE_EINVAL, "null handle");
    for (fe_batch::Lattice& l : b->lattices) {
        const int rc = fe_law_set_param(l.law, param, value);
        if (rc != FE_OK) return rc;
    }
    return fe::ok();
}

int fe_batch_upload(fe_batch* b, int instance, int field, const float* host)
{
    if (host == nullptr) return fe::fail(FE_EINVAL, "fe_batch_upload: null buffer");
    return transfer(b, instance, field, const_cast<float*>(host), true);
}

int fe_batch_fetch(fe_batch* b, int instance, int field, float* host)
{
    if (host == nullptr) return fe::fail(FE_EINVAL, "fe_batch_fetch: null buffer");
    return transfer(b, instance, field, host, false);
}

int fe_batch_step(fe_batch* b, double dt, int flags, int* violations)
{
    if (b == nullptr) return fe::fail(FE_EINVAL, "null handle");
    b->violations.clear();
    fe_step_info info{};
    for (fe_batch::Lattice& l : b->lattices) {
        const int rc = fe_law_step(l.law, dt, flags, &info);
        if (rc != FE_OK) return rc;
    }
    for (std::size_t k = 0; k < b->lattices.size(); ++k) {
        fe_batch::Lattice& l = b->lattices[k];
        int rc = fe_law_sync(l.law, &info);
        if (rc != FE_OK) return rc;
        const std::size_t plane = static_cast<std::size_t>(l.nx) * l.ny;
        for (int i = l.seen; i < info.violations; ++i) {
            fe_violation v{};
            if ((rc = fe_law_violation(l.law, i, &v)) != FE_OK) return rc;
            int instance = -1;
            if (v.kind == FE_RANGE || v.kind == FE_NOT_FINITE) {
                const int z = static_cast<int>(v.first_cell / plane);
                for (const int m : l.members) {
                    const fe_batch::Where& w = b->where[static_cast<std::size_t>(m)];
                    if (z >= w.z0 && z < w.z0 + w.nz) {
                        instance = m;
                        v.first_cell -= static_cast<uint32_t>(plane * static_cast<std::size_t>(w.z0));
                    }
                }
            } else if (l.members.size() == 1) {
                instance = l.members[0];
            }
            b->violations.emplace_back(instance, v);
        }
        l.seen = info.violations;
    }
    if (violations != nullptr) *violations = static_cast<int>(b->violations.size());
    return fe::ok();
}

int fe_batch_violation(const fe_batch* b, int index, int* instance, fe_violation* out)
{
    if (b == nullptr || out == nullptr || index < 0 || static_cast<std::size_t>(index) >= b->violations.size()) {
        return fe::fail(FE_EINVAL, "fe_batch_violation: bad argument");
    }
    if (instance != nullptr) *instance = b->violations[static_cast<std::size_t>(index)].first;
    *out = b->violations[static_cast<std::size_t>(index)].second;
    return fe::ok();
}

} // extern "C"
