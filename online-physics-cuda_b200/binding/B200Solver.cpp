// The reference's CUDA backend, replaced by the B200 library: a LawBackend (src/field/Backend.hpp:67-84) over the C ABI
// of include/fe.h. It is compiled into the reference in place of src/field/cuda/CudaSolver.cpp: it defines the same
// three entry points (CudaSolver::create, ::unavailable, ::source; src/field/cuda/CudaSolver.hpp:24-33), so the
// reference's own Solver::use_gpu (src/field/Solver.cpp:173-200) and everything above it (lawc, the gates, the game)
// run on it unchanged. Link with libfe_b200.so.
//
// How it maps the interface:
//   create    the Law (as the reference holds it, compiled and possibly edited) is lowered by the reference's own IR and
//             handed over as its JSON (fe_law_create_ir), so what runs is the reference's IR exactly;
//   step      the host's edits go up first (FieldEdits: everything, flagged planes, or a moved window and its arriving
//             boxes), then params (they may have changed since), the learned flag, the step; violations, substeps and
//             the per-term profile come back; without lazy readback every field the step may have changed comes back
//             into the FieldSet, with it they stay on the card until fetch();
//   derive    the same for Solver::refresh_derived;
//   fetch     the fields asked for, from the card.
// The host FieldSet is the truth between steps, as with the reference's own backend (Solver.hpp:30-53).
#include "field/Backend.hpp"
#include "field/Grid.hpp"
#include "field/Law.hpp"
#include "field/cuda/CudaSolver.hpp"
#include "field/ir/LawIR.hpp"

#include "fe.h"

#include <chrono>
#include <memory>
#include <string>
#include <vector>

namespace fieldengine::field {

namespace {

class B200Solver final : public LawBackend {
public:
    B200Solver(fe_law* handle, const Law& law, const GridShape& shape) : h_(handle), shape_(shape)
    {
        profile_.backend = "CUDA sm_100a (B200)";
        profile_.terms.resize(law.terms.size());
        for (std::size_t t = 0; t < law.terms.size(); ++t) profile_.terms[t].name = law.terms[t].name;
    }
    ~B200Solver() override { fe_law_destroy(h_); }
    B200Solver(const B200Solver&) = delete;
    B200Solver& operator=(const B200Solver&) = delete;

    void step(double dt, bool respect_max_dt, bool learned, Law& law, FieldSet& fields, FieldEdits& edits, std::vector<char>& changed,
        std::vector<Violation>& violations, std::vector<int>& substeps) override
    {
        const auto start = std::chrono::steady_clock::now();
        profile_.upload_bytes = profile_.download_bytes = 0;
        upload(law, fields, edits);
        params(law);
        fe_law_set_learned(h_, learned ? 1 : 0);
        fe_step_info info{};
        if (!ok(fe_law_step(h_, dt, respect_max_dt ? 0 : FE_STEP_IGNORE_MAX_DT, &info), violations)) return;
        profile_.gpu_ms = info.gpu_ms;
        profile_.launches = info.launches;
        profile_.fallbacks = info.fallbacks;
        for (int i = 0; i < info.violations; ++i) {
            fe_violation v{};
            if (fe_law_violation(h_, i, &v) != FE_OK) continue;
            Violation out;
            out.kind = static_cast<Violation::Kind>(v.kind);
            out.term = v.term >= 0 ? law.terms[static_cast<std::size_t>(v.term)].name : "";
            out.field = v.field >= 0 ? law.fields[static_cast<std::size_t>(v.field)].name : "";
            out.detail = v.detail;
            violations.push_back(std::move(out));
        }
        substeps.assign(law.terms.size(), 1);
        changed.assign(fields.count(), 0);
        for (std::size_t t = 0; t < law.terms.size(); ++t) {
            TermProfile& tp = profile_.terms[t];
            tp.substeps = substeps[t] = fe_law_substeps(h_, static_cast<int>(t));
            tp.idle = fe_law_term_idle(h_, static_cast<int>(t)) == 1;
            const int l = fe_law_term_learned(h_, static_cast<int>(t));
            tp.learned = l == 1;
            tp.fell_back = l == 2;
            if (tp.idle) continue;
            // What the term wrote may have moved (the learned equations write a subset of the classical targets).
            for (const Equation& eq : law.terms[t].equations) changed[static_cast<std::size_t>(eq.target)] = 1;
        }
        for (const Derive& d : law.derives) changed[static_cast<std::size_t>(d.target)] = 1;
        if (!lazy_) fetch(fields, changed);
        profile_.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
    }

    void derive(Law& law, FieldSet& fields, FieldEdits& edits, std::vector<char>& changed) override
    {
        upload(law, fields, edits);
        params(law);
        const auto start = std::chrono::steady_clock::now();
        fe_law_derive(h_);
        profile_.derive_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
        changed.assign(fields.count(), 0);
        for (const Derive& d : law.derives) changed[static_cast<std::size_t>(d.target)] = 1;
        if (!lazy_) fetch(fields, changed);
    }

    void check_contracts_every(int steps) override { fe_law_check_every(h_, steps); }
    void set_lazy(bool on) override { lazy_ = on; }

    void fetch(FieldSet& fields, const std::vector<char>& which) override
    {
        const auto start = std::chrono::steady_clock::now();
        for (std::size_t f = 0; f < which.size() && f < fields.count(); ++f) {
            if (!which[f]) continue;
            fe_law_fetch(h_, static_cast<int>(f), fields.values(static_cast<int>(f)).data());
            profile_.download_bytes += shape_.cells() * sizeof(float);
        }
        profile_.download_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
    }

    [[nodiscard]] const std::string& adapter() const override { return adapter_; }
    [[nodiscard]] const char* api() const override { return "CUDA (sm_100a, libfe_b200)"; }
    [[nodiscard]] const StepProfile& profile() const override { return profile_; }

private:
    // A failing call leaves the world as it was and says why, as a violation a designer sees.
    bool ok(int status, std::vector<Violation>& violations)
    {
        if (status == FE_OK) return true;
        Violation v;
        v.kind = Violation::Kind::NotFinite;
        v.detail = std::string("B200 backend: ") + fe_last_error();
        violations.push_back(std::move(v));
        return false;
    }

    void params(const Law& law)
    {
        for (std::size_t p = 0; p < law.param_values.size(); ++p) fe_law_set_param(h_, static_cast<int>(p), law.param_values[p]);
    }

    // The host's edits since the card last saw the fields (CudaSolver.cpp:779-920 takes them the same way).
    void upload(const Law& law, FieldSet& fields, FieldEdits& edits)
    {
        const auto start = std::chrono::steady_clock::now();
        const std::size_t plane = static_cast<std::size_t>(shape_.nx) * static_cast<std::size_t>(shape_.ny);
        if (!edits.all && edits.shifted()) {
            // The window moved: move the card's cells, then send only what arrived, for the fields the law does not
            // derive (the derives recompute theirs).
            fe_law_shift(h_, edits.shift[0], edits.shift[1], edits.shift[2]);
            for (std::size_t f = 0; f < fields.count(); ++f) {
                if (law.fields[f].derived) continue;
                for (const CellBox& b : edits.boxes) {
                    fe_law_upload_box(h_, static_cast<int>(f), fields.values(static_cast<int>(f)).data(), b.x0, b.y0, b.z0, b.x1, b.y1, b.z1);
                    profile_.upload_bytes += static_cast<std::size_t>(std::max(0, b.x1 - b.x0)) * std::max(0, b.y1 - b.y0) *
                        std::max(0, b.z1 - b.z0) * sizeof(float);
                }
            }
        }
        for (std::size_t f = 0; f < fields.count(); ++f) {
            const float* host = fields.values(static_cast<int>(f)).data();
            if (edits.all) {
                fe_law_upload(h_, static_cast<int>(f), host);
                profile_.upload_bytes += shape_.cells() * sizeof(float);
                continue;
            }
            if (f >= edits.planes.size() || edits.planes[f].empty()) continue;
            std::vector<unsigned char> marks(static_cast<std::size_t>(shape_.nz), 0);
            std::size_t sent = 0;
            for (std::size_t z = 0; z < marks.size() && z < edits.planes[f].size(); ++z) {
                marks[z] = edits.planes[f][z] != 0 ? 1 : 0;
                sent += marks[z];
            }
            if (sent == 0) continue;
            fe_law_upload_planes(h_, static_cast<int>(f), host, marks.data());
            profile_.upload_bytes += sent * plane * sizeof(float);
        }
        edits.all = false;
        edits.planes.clear();
        edits.shift[0] = edits.shift[1] = edits.shift[2] = 0;
        edits.boxes.clear();
        profile_.upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
    }

    fe_law* h_;
    GridShape shape_;
    bool lazy_ = false;
    StepProfile profile_;
    std::string adapter_ = "NVIDIA B200 (sm_100a)";
};

} // namespace

std::shared_ptr<LawBackend> CudaSolver::create(Law& law, const GridShape& shape, std::string& why)
{
    if (fe_device_check() != FE_OK) {
        why = fe_last_error();
        return nullptr;
    }
    const std::string json = ir::to_json(ir::lower(law), law);
    fe_law* h = nullptr;
    if (fe_law_create_ir(json.c_str(), shape.nx, shape.ny, shape.nz, shape.cell, &h) != FE_OK) {
        why = fe_last_error();
        return nullptr;
    }
    return std::make_shared<B200Solver>(h, law, shape);
}

std::string CudaSolver::unavailable()
{
    return fe_device_check() == FE_OK ? std::string() : std::string(fe_last_error());
}

std::string CudaSolver::source(const Law& law)
{
    // The generated translation unit (lawc --cuda prints it). Kernels are generated per lattice, whose extents are
    // compile-time constants in them: this is the one for a 128^3 lattice of unit cells.
    const std::string json = ir::to_json(ir::lower(law), law);
    std::size_t needed = 0;
    if (fe_law_source_ir(json.c_str(), 128, 128, 128, 1.0, nullptr, 0, &needed) != FE_OK) return std::string("// ") + fe_last_error() + "\n";
    std::string text(needed, '\0');
    fe_law_source_ir(json.c_str(), 128, 128, 128, 1.0, text.data(), needed, &needed);
    text.resize(needed > 0 ? needed - 1 : 0);
    return text;
}

} // namespace fieldengine::field
