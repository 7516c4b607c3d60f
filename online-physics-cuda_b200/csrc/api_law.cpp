// C-ABI of the law backend (include/fe.h, "the law backend").
#include "../../include/fe.h"

#include "adjoint.hpp"
#include "api_common.hpp"
#include "engine.hpp"
#include "ir_json.hpp"

#include <cstring>
#include <memory>
#include <string>

struct fe_law {
    fe::Engine engine;
};

namespace {

std::vector<fe::law::Source> sources_of(const char* text, const char* name)
{
    return {fe::law::Source{name != nullptr && name[0] != 0 ? name : "law", text != nullptr ? text : ""}};
}

int put_text(const std::string& text, char* buf, size_t cap, size_t* needed)
{
    if (needed != nullptr) *needed = text.size() + 1;
    if (buf != nullptr && cap > 0) {
        const size_t n = std::min(cap - 1, text.size());
        std::memcpy(buf, text.data(), n);
        buf[n] = 0;
    }
    return fe::ok();
}

bool compile_law(const char* text, fe::law::Law& law, std::string& why)
{
    std::vector<std::string> errors;
    law = fe::law::compile(sources_of(text, "law"), errors);
    if (errors.empty()) return true;
    for (const std::string& e : errors) why += e + "\n";
    return false;
}

bool field_ok(const fe_law* l, int field)
{
    return l != nullptr && field >= 0 && static_cast<size_t>(field) < l->engine.law().fields.size();
}

void fill_info(const fe_law* l, fe_step_info* info)
{
    if (info == nullptr) return;
    info->violations = static_cast<int>(l->engine.violations().size());
    info->launches = l->engine.launches_last_step();
    info->gpu_ms = l->engine.gpu_ms_last_step();
    info->fallbacks = l->engine.fallbacks_last_step();
}

} // namespace

extern "C" {

int fe_law_create(const char* law_text, const char* source_name, int nx, int ny, int nz, double h, fe_law** out)
{
    if (law_text == nullptr || out == nullptr) return fe::fail(FE_EINVAL, "fe_law_create: null argument");
    *out = nullptr;
    auto l = std::make_unique<fe_law>();
    std::string why;
    if (!l->engine.create(sources_of(law_text, source_name), nx, ny, nz, h, why)) {
        fe::law::Law law;
        std::string law_why;
        const bool law_ok = compile_law(law_text, law, law_why);
        int code = FE_ECUDA;
        if (!law_ok) code = FE_ELAW;
        else if (why.find("does not run") != std::string::npos || why.find("at most") != std::string::npos) code = FE_EUNSUP;
        else if (why.find("no CUDA device") != std::string::npos || why.find("built for sm_100a") != std::string::npos ||
            why.find("entry point") != std::string::npos) code = FE_ENODEV;
        return fe::fail(code, why);
    }
    *out = l.release();
    return fe::ok();
}

int fe_law_create_ir(const char* ir_json, int nx, int ny, int nz, double h, fe_law** out)
{
    if (ir_json == nullptr || out == nullptr) return fe::fail(FE_EINVAL, "fe_law_create_ir: null argument");
    *out = nullptr;
    fe::law::Law law;
    fe::ir::Module m;
    std::string why;
    if (!fe::law_from_ir_json(ir_json, law, m, why)) return fe::fail(FE_ELAW, why);
    auto l = std::make_unique<fe_law>();
    if (!l->engine.create(std::move(law), std::move(m), nx, ny, nz, h, why)) {
        int code = FE_ECUDA;
        if (why.find("does not run") != std::string::npos || why.find("at most") != std::string::npos) code = FE_EUNSUP;
        else if (why.find("no CUDA device") != std::string::npos || why.find("built for sm_100a") != std::string::npos ||
            why.find("entry point") != std::string::npos) code = FE_ENODEV;
        else if (why.find("lattice needs") != std::string::npos || why.find("2^32") != std::string::npos) code = FE_EINVAL;
        return fe::fail(code, why);
    }
    *out = l.release();
    return fe::ok();
}

int fe_law_ir_check(const char* ir_json, char* buf, size_t cap, size_t* needed)
{
    if (ir_json == nullptr) return fe::fail(FE_EINVAL, "fe_law_ir_check: null argument");
    fe::law::Law law;
    fe::ir::Module m;
    std::string why;
    if (!fe::law_from_ir_json(ir_json, law, m, why)) return fe::fail(FE_ELAW, why);
    return put_text(fe::ir::to_json(m, law), buf, cap, needed);
}

void fe_law_destroy(fe_law* law)
{
    delete law;
}

int fe_law_ir_json(const char* law_text, char* buf, size_t cap, size_t* needed)
{
    fe::law::Law law;
    std::string why;
    if (!compile_law(law_text, law, why)) return fe::fail(FE_ELAW, why);
    const fe::ir::Module m = fe::ir::lower(law);
    return put_text(fe::ir::to_json(m, law), buf, cap, needed);
}

int fe_law_ir_listing(const char* law_text, char* buf, size_t cap, size_t* needed)
{
    fe::law::Law law;
    std::string why;
    if (!compile_law(law_text, law, why)) return fe::fail(FE_ELAW, why);
    const fe::ir::Module m = fe::ir::lower(law);
    return put_text(fe::ir::describe(m, law), buf, cap, needed);
}

int fe_law_adjoint(const char* law_text, const char* term, char* buf, size_t cap, size_t* needed)
{
    fe::law::Law law;
    std::string why;
    if (!compile_law(law_text, law, why)) return fe::fail(FE_ELAW, why);
    const std::string text = fe::adjoint::adjoint_law(law, term ? term : "", why);
    if (text.empty()) return fe::fail(FE_EUNSUP, why);
    return put_text(text, buf, cap, needed);
}

int fe_law_source(const char* law_text, int nx, int ny, int nz, double h, char* buf, size_t cap, size_t* needed)
{
    fe::law::Law law;
    std::string why;
    if (!compile_law(law_text, law, why)) return fe::fail(FE_ELAW, why);
    if (nx < 1 || ny < 1 || nz < 1 || !(h > 0.0)) return fe::fail(FE_EINVAL, "bad lattice");
    const fe::ir::Module m = fe::ir::lower(law);
    fe::gen::Plan plan;
    if (!fe::gen::generate(m, law, nx, ny, nz, h, plan, why)) return fe::fail(FE_EUNSUP, why);
    return put_text(plan.source, buf, cap, needed);
}

int fe_law_source_ir(const char* ir_json, int nx, int ny, int nz, double h, char* buf, size_t cap, size_t* needed)
{
    if (ir_json == nullptr) return fe::fail(FE_EINVAL, "fe_law_source_ir: null argument");
    if (nx < 1 || ny < 1 || nz < 1 || !(h > 0.0)) return fe::fail(FE_EINVAL, "bad lattice");
    fe::law::Law law;
    fe::ir::Module m;
    std::string why;
    if (!fe::law_from_ir_json(ir_json, law, m, why)) return fe::fail(FE_ELAW, why);
    fe::gen::Plan plan;
    if (!fe::gen::generate(m, law, nx, ny, nz, h, plan, why)) return fe::fail(FE_EUNSUP, why);
    return put_text(plan.source, buf, cap, needed);
}

int fe_law_compile_check(const char* law_text, int nx, int ny, int nz, double h)
{
    fe::law::Law law;
    std::string why;
    if (!compile_law(law_text, law, why)) return fe::fail(FE_ELAW, why);
    if (nx < 1 || ny < 1 || nz < 1 || !(h > 0.0)) return fe::fail(FE_EINVAL, "bad lattice");
    const fe::ir::Module m = fe::ir::lower(law);
    fe::gen::Plan plan;
    if (!fe::gen::generate(m, law, nx, ny, nz, h, plan, why)) return fe::fail(FE_EUNSUP, why);
    std::string cubin, log;
    if (!fe::compile_cubin(plan.source, "law.cu", cubin, log, nullptr)) return fe::fail(FE_ECUDA, log);
    return fe::ok();
}

int fe_law_field_count(const fe_law* law)
{
    return law == nullptr ? -1 : static_cast<int>(law->engine.law().fields.size());
}

int fe_law_field_id(const fe_law* law, const char* name)
{
    return law == nullptr || name == nullptr ? -1 : law->engine.law().field_id(name);
}

int fe_law_field_name(const fe_law* law, int field, char* buf, size_t cap)
{
    if (!field_ok(law, field)) return fe::fail(FE_EINVAL, "no such field");
    return put_text(law->engine.law().fields[static_cast<size_t>(field)].name, buf, cap, nullptr);
}

int fe_law_field_info(const fe_law* law, int field, fe_field_info* out)
{
    if (!field_ok(law, field) || out == nullptr) return fe::fail(FE_EINVAL, "no such field");
    const fe::law::FieldDecl& d = law->engine.law().fields[static_cast<size_t>(field)];
    out->init = d.init;
    out->lo = d.lo;
    out->hi = d.hi;
    out->is_static = d.is_static ? 1 : 0;
    out->derived = d.derived ? 1 : 0;
    out->clamp = d.clamp ? 1 : 0;
    return fe::ok();
}

int fe_law_term_count(const fe_law* law)
{
    return law == nullptr ? -1 : static_cast<int>(law->engine.law().terms.size());
}

int fe_law_term_name(const fe_law* law, int term, char* buf, size_t cap)
{
    if (law == nullptr || term < 0 || static_cast<size_t>(term) >= law->engine.law().terms.size()) return fe::fail(FE_EINVAL, "no such term");
    return put_text(law->engine.law().terms[static_cast<size_t>(term)].name, buf, cap, nullptr);
}

int fe_law_param_count(const fe_law* law)
{
    return law == nullptr ? -1 : static_cast<int>(law->engine.law().param_names.size());
}

int fe_law_param_id(const fe_law* law, const char* name)
{
    return law == nullptr || name == nullptr ? -1 : law->engine.law().param_id(name);
}

int fe_law_set_param(fe_law* law, int param, double value)
{
    if (law == nullptr || !law->engine.set_param(param, value)) return fe::fail(FE_EINVAL, "no such param");
    return fe::ok();
}

int fe_law_get_param(const fe_law* law, int param, double* value)
{
    if (law == nullptr || value == nullptr || param < 0 || static_cast<size_t>(param) >= law->engine.law().param_values.size()) {
        return fe::fail(FE_EINVAL, "no such param");
    }
    *value = law->engine.law().param_values[static_cast<size_t>(param)];
    return fe::ok();
}

int fe_law_upload(fe_law* law, int field, const float* host)
{
    std::string why;
    if (!field_ok(law, field) || host == nullptr) return fe::fail(FE_EINVAL, "fe_law_upload: bad field or pointer");
    if (!law->engine.upload(field, host, false, why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_upload_device(fe_law* law, int field, const float* dev)
{
    std::string why;
    if (!field_ok(law, field) || dev == nullptr) return fe::fail(FE_EINVAL, "fe_law_upload_device: bad field or pointer");
    if (!law->engine.upload(field, dev, true, why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_shift(fe_law* law, int dx, int dy, int dz)
{
    std::string why;
    if (law == nullptr) return fe::fail(FE_EINVAL, "fe_law_shift: null handle");
    if (!law->engine.shift(dx, dy, dz, why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_upload_box(fe_law* law, int field, const float* host, int x0, int y0, int z0, int x1, int y1, int z1)
{
    std::string why;
    if (!field_ok(law, field) || host == nullptr) return fe::fail(FE_EINVAL, "fe_law_upload_box: bad field or pointer");
    const int box[6] = {x0, y0, z0, x1, y1, z1};
    if (!law->engine.upload_box(field, host, box, why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_upload_planes(fe_law* law, int field, const float* host, const unsigned char* planes)
{
    std::string why;
    if (!field_ok(law, field) || host == nullptr || planes == nullptr) return fe::fail(FE_EINVAL, "fe_law_upload_planes: bad field or pointer");
    if (!law->engine.upload_planes(field, host, planes, why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_fetch(fe_law* law, int field, float* host)
{
    std::string why;
    if (!field_ok(law, field) || host == nullptr) return fe::fail(FE_EINVAL, "fe_law_fetch: bad field or pointer");
    if (!law->engine.fetch(field, host, false, why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_fetch_device(fe_law* law, int field, float* dev)
{
    std::string why;
    if (!field_ok(law, field) || dev == nullptr) return fe::fail(FE_EINVAL, "fe_law_fetch_device: bad field or pointer");
    if (!law->engine.fetch(field, dev, true, why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_mark_edited(fe_law* law, int field)
{
    if (!field_ok(law, field)) return fe::fail(FE_EINVAL, "bad field");
    law->engine.mark_edited(field);
    return fe::ok();
}

int fe_law_set_owned_z(fe_law* law, int z0, int z1)
{
    if (law == nullptr) return fe::fail(FE_EINVAL, "null handle");
    if (!law->engine.set_owned_z(z0, z1)) return fe::fail(FE_EINVAL, "fe_law_set_owned_z: need 0 <= z0 < z1 <= nz");
    return fe::ok();
}

int fe_law_mark_halo(fe_law* law, int field)
{
    if (!field_ok(law, field)) return fe::fail(FE_EINVAL, "bad field");
    law->engine.mark_halo(field);
    return fe::ok();
}

int fe_law_set_external_conservation(fe_law* law, int on)
{
    if (law == nullptr) return fe::fail(FE_EINVAL, "null handle");
    law->engine.set_external_conservation(on != 0);
    return fe::ok();
}

int fe_law_take_totals(fe_law* law, fe_group_totals* out, int max, int* n)
{
    if (law == nullptr || n == nullptr || max < 0 || (max > 0 && out == nullptr)) return fe::fail(FE_EINVAL, "fe_law_take_totals: bad arguments");
    const std::vector<fe::GroupTotals> all = law->engine.take_totals();
    if (static_cast<int>(all.size()) > max) return fe::fail(FE_EINVAL, "fe_law_take_totals: " + std::to_string(all.size()) + " entries, room for " + std::to_string(max));
    for (std::size_t i = 0; i < all.size(); ++i) {
        std::memset(&out[i], 0, sizeof(out[i]));
        out[i].step = all[i].step;
        out[i].term = all[i].term;
        out[i].group = all[i].group;
        out[i].substeps = all[i].substeps;
        out[i].before = all[i].before;
        out[i].after = all[i].after;
        out[i].scale = all[i].scale;
    }
    *n = static_cast<int>(all.size());
    return fe::ok();
}

int fe_law_plan_z_reach(const char* law_text, int nx, int ny, int nz, double h, int* reach, int* flags)
{
    if (reach == nullptr || flags == nullptr) return fe::fail(FE_EINVAL, "null argument");
    fe::law::Law law;
    std::string why;
    if (!compile_law(law_text, law, why)) return fe::fail(FE_ELAW, why);
    if (nx < 1 || ny < 1 || nz < 1 || !(h > 0.0)) return fe::fail(FE_EINVAL, "bad lattice");
    const fe::ir::Module m = fe::ir::lower(law);
    fe::gen::Plan plan;
    if (!fe::gen::generate(m, law, nx, ny, nz, h, plan, why)) return fe::fail(FE_EUNSUP, why);
    bool reductions = false, z_solves = false;
    fe::plan_z_reach(plan, *reach, reductions, z_solves);
    *flags = (reductions ? 1 : 0) | (z_solves ? 2 : 0);
    return fe::ok();
}

int fe_law_field_device_ptr(const fe_law* law, int field, const float** dev)
{
    if (!field_ok(law, field) || dev == nullptr) return fe::fail(FE_EINVAL, "bad field");
    *dev = law->engine.device_field(field);
    return fe::ok();
}

int fe_law_step(fe_law* law, double dt, int flags, fe_step_info* info)
{
    if (law == nullptr || !(dt >= 0.0)) return fe::fail(FE_EINVAL, "fe_law_step: bad handle or dt");
    std::string why;
    if (!law->engine.step(dt, (flags & FE_STEP_IGNORE_MAX_DT) == 0, why)) {
        return fe::fail(why.find("error word") != std::string::npos ? FE_EKERNEL : FE_ECUDA, why);
    }
    fill_info(law, info);
    return fe::ok();
}

int fe_law_derive(fe_law* law)
{
    if (law == nullptr) return fe::fail(FE_EINVAL, "null handle");
    std::string why;
    if (!law->engine.derive(why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_check_every(fe_law* law, int steps)
{
    if (law == nullptr || steps < 1) return fe::fail(FE_EINVAL, "fe_law_check_every: steps >= 1");
    law->engine.check_every(steps);
    return fe::ok();
}

int fe_law_set_deferred(fe_law* law, int on)
{
    if (law == nullptr) return fe::fail(FE_EINVAL, "null handle");
    std::string why;
    if (!on && !law->engine.sync(why)) return fe::fail(FE_ECUDA, why);
    law->engine.set_deferred(on != 0);
    return fe::ok();
}

int fe_law_sync(fe_law* law, fe_step_info* info)
{
    if (law == nullptr) return fe::fail(FE_EINVAL, "null handle");
    std::string why;
    if (!law->engine.sync(why)) return fe::fail(why.find("error word") != std::string::npos ? FE_EKERNEL : FE_ECUDA, why);
    fill_info(law, info);
    return fe::ok();
}

int fe_law_violation(const fe_law* law, int index, fe_violation* out)
{
    if (law == nullptr || out == nullptr || index < 0 || static_cast<size_t>(index) >= law->engine.violations().size()) {
        return fe::fail(FE_EINVAL, "no such violation");
    }
    const fe::Violation& v = law->engine.violations()[static_cast<size_t>(index)];
    std::memset(out, 0, sizeof(*out));
    out->kind = v.kind;
    out->term = v.term;
    out->field = v.field;
    out->count = v.count;
    out->first_cell = v.first_cell;
    out->before = v.before;
    out->after = v.after;
    out->tolerance = v.tolerance;
    out->step = v.step;
    std::strncpy(out->detail, v.detail.c_str(), sizeof(out->detail) - 1);
    return fe::ok();
}

int fe_law_set_learned(fe_law* law, int on)
{
    if (law == nullptr) return fe::fail(FE_EINVAL, "null handle");
    law->engine.set_learned(on != 0);
    return fe::ok();
}

int fe_law_term_learned(const fe_law* law, int term)
{
    if (law == nullptr || term < 0 || static_cast<size_t>(term) >= law->engine.term_profile().size()) return -1;
    const fe::TermProfile& p = law->engine.term_profile()[static_cast<size_t>(term)];
    return p.fell_back ? 2 : (p.learned ? 1 : 0);
}

int fe_law_substeps(const fe_law* law, int term)
{
    if (law == nullptr || term < 0 || static_cast<size_t>(term) >= law->engine.substeps().size()) return -1;
    return law->engine.substeps()[static_cast<size_t>(term)];
}

int fe_law_term_idle(const fe_law* law, int term)
{
    if (law == nullptr || term < 0 || static_cast<size_t>(term) >= law->engine.term_profile().size()) return -1;
    return law->engine.term_profile()[static_cast<size_t>(term)].idle ? 1 : 0;
}

int fe_law_digest(fe_law* law, uint64_t* out)
{
    if (law == nullptr || out == nullptr) return fe::fail(FE_EINVAL, "null argument");
    std::uint64_t h = 1469598103934665603ull;
    std::vector<float> host(law->engine.cells());
    std::string why;
    // FieldSet::digest (src/field/Grid.cpp:60-74): each field's name, then its values' bits, in declaration order.
    for (size_t f = 0; f < law->engine.law().fields.size(); ++f) {
        if (!law->engine.fetch(static_cast<int>(f), host.data(), false, why)) return fe::fail(FE_ECUDA, why);
        const std::string& name = law->engine.law().fields[f].name;
        h = fe::fnv1a(name.data(), name.size(), h);
        h = fe::fnv1a(host.data(), host.size() * sizeof(float), h);
    }
    *out = h;
    return fe::ok();
}

int fe_law_stream(const fe_law* law, void** stream)
{
    if (law == nullptr || stream == nullptr) return fe::fail(FE_EINVAL, "null argument");
    *stream = law->engine.stream();
    return fe::ok();
}

int fe_law_time_gather(fe_law* law, int term, int launches, float* ms)
{
    if (law == nullptr || ms == nullptr || launches < 1) return fe::fail(FE_EINVAL, "bad argument");
    std::string why;
    if (!law->engine.time_gather(term, launches, *ms, why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_law_time_stage(fe_law* law, int term, int stage, int launches, double dt, float* ms, char* kernel, size_t cap)
{
    if (law == nullptr || ms == nullptr || launches < 1) return fe::fail(FE_EINVAL, "fe_law_time_stage: bad argument");
    std::string why, name;
    if (!law->engine.time_stage(term, stage, launches, dt, *ms, name, why)) return fe::fail(FE_EINVAL, why);
    if (kernel != nullptr && cap > 0) {
        const size_t n = std::min(cap - 1, name.size());
        std::memcpy(kernel, name.data(), n);
        kernel[n] = 0;
    }
    return fe::ok();
}

} // extern "C"
