// Reverse mode through N steps of one term of a law, natively (include/fe.h, "reverse mode"): the primal law and its
// adjoint law (fe_law_adjoint) as two law handles, the forward keeping every K-th state on the device
// (K = ceil(sqrt(N)) by default), the backward recomputing each segment's K states from its checkpoint and stepping the
// adjoint law back over them.
//
// The reference does this in its lawc (tools/lawc/main.cpp:274-361): every state kept on the host, uploaded before
// each adjoint step. Here the states never leave the card, and memory is about 2 sqrt(N) copies of the moving fields
// instead of N.
#include "../../include/fe.h"

#include "api_common.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

struct fe_vjp {
    fe_law* primal = nullptr;
    fe_law* adj = nullptr;
    int term = 0;
    std::size_t cells = 0;
    // The primal's moving fields (checkpointed: a segment is recomputed from them); which of them the adjoint law
    // reads, as (index in `state`, its static copy in the adjoint law); the primal's static fields it reads.
    std::vector<int> state;
    std::vector<std::pair<int, int>> state_to_adj;
    std::vector<int> statics, statics_in_adj;
    int steps = 0, every = 1;
    double dt = 0.0;
    std::vector<float*> checkpoints; // per checkpoint: the state fields, one after the other (kept across forwards)
    std::size_t checkpoint_bytes = 0;
    std::size_t used = 0;            // checkpoints the last forward filled
    int seen = 0;                    // violations the primal held after the last forward (deferred judging keeps them)
    float* segment = nullptr;        // every x state fields: a segment's recomputed states
    std::size_t segment_states = 0;

    ~fe_vjp()
    {
        release();
        if (adj != nullptr) fe_law_destroy(adj);
        if (primal != nullptr) fe_law_destroy(primal);
    }

    void release()
    {
        for (float* p : checkpoints) cudaFree(p);
        checkpoints.clear();
        checkpoint_bytes = 0;
        used = 0;
        if (segment != nullptr) cudaFree(segment);
        segment = nullptr;
        segment_states = 0;
    }
};

namespace {

std::string name_of(const fe_law* law, int field)
{
    char buf[256];
    if (fe_law_field_name(law, field, buf, sizeof(buf)) != FE_OK) return {};
    return buf;
}

// The state fields of the primal into `dst` (one after the other), or back from `src`.
int save_state(fe_vjp* v, float* dst)
{
    for (std::size_t k = 0; k < v->state.size(); ++k) {
        const int rc = fe_law_fetch_device(v->primal, v->state[k], dst + k * v->cells);
        if (rc != FE_OK) return rc;
    }
    return FE_OK;
}

int restore_state(fe_vjp* v, const float* src)
{
    for (std::size_t k = 0; k < v->state.size(); ++k) {
        const int rc = fe_law_upload_device(v->primal, v->state[k], src + k * v->cells);
        if (rc != FE_OK) return rc;
    }
    return FE_OK;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fe::fail(FE_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

} // namespace

extern "C" {

int fe_vjp_create(const char* law_text, const char* term, int nx, int ny, int nz, double h, fe_vjp** out)
{
    if (law_text == nullptr || out == nullptr) return fe::fail(FE_EINVAL, "fe_vjp_create: null argument");
    *out = nullptr;
    std::size_t needed = 0;
    int rc = fe_law_adjoint(law_text, term, nullptr, 0, &needed);
    if (rc != FE_OK) return rc;
    std::string adjoint(needed, '\0');
    rc = fe_law_adjoint(law_text, term, adjoint.data(), adjoint.size(), &needed);
    if (rc != FE_OK) return rc;
    adjoint.resize(needed > 0 ? needed - 1 : 0);

    auto v = std::make_unique<fe_vjp>();
    if ((rc = fe_law_create(law_text, "law", nx, ny, nz, h, &v->primal)) != FE_OK) return rc;
    if ((rc = fe_law_create(adjoint.c_str(), "law__adj", nx, ny, nz, h, &v->adj)) != FE_OK) return rc;
    v->cells = static_cast<std::size_t>(nx) * ny * nz;
    v->term = 0;
    if (term != nullptr && term[0] != 0) {
        const int terms = fe_law_term_count(v->primal);
        char buf[256];
        for (v->term = 0; v->term < terms; ++v->term) {
            if (fe_law_term_name(v->primal, v->term, buf, sizeof(buf)) == FE_OK && std::string(buf) == term) break;
        }
        if (v->term == terms) return fe::fail(FE_EINVAL, std::string("the law has no term '") + term + "'");
    }
    // The adjoint law's static fields that are primal fields: the primal's state at the step being differentiated
    // when the field moves, the forward's input otherwise.
    const int primal_fields = fe_law_field_count(v->primal);
    for (int f = 0; f < primal_fields; ++f) {
        fe_field_info info{};
        if (fe_law_field_info(v->primal, f, &info) == FE_OK && !info.is_static) v->state.push_back(f);
    }
    const int adj_fields = fe_law_field_count(v->adj);
    for (int f = 0; f < adj_fields; ++f) {
        fe_field_info info{};
        if (fe_law_field_info(v->adj, f, &info) != FE_OK || !info.is_static) continue;
        const int in_primal = fe_law_field_id(v->primal, name_of(v->adj, f).c_str());
        if (in_primal < 0) continue;
        const auto moving = std::find(v->state.begin(), v->state.end(), in_primal);
        if (moving != v->state.end()) {
            v->state_to_adj.emplace_back(static_cast<int>(moving - v->state.begin()), f);
        } else {
            v->statics.push_back(in_primal);
            v->statics_in_adj.push_back(f);
        }
    }
    for (fe_law* l : {v->primal, v->adj}) {
        if ((rc = fe_law_set_deferred(l, 1)) != FE_OK) return rc;
    }
    *out = v.release();
    return fe::ok();
}

void fe_vjp_destroy(fe_vjp* v)
{
    delete v;
}

int fe_vjp_laws(fe_vjp* v, fe_law** primal, fe_law** adjoint)
{
    if (v == nullptr) return fe::fail(FE_EINVAL, "fe_vjp_laws: null handle");
    if (primal != nullptr) *primal = v->primal;
    if (adjoint != nullptr) *adjoint = v->adj;
    return fe::ok();
}

int fe_vjp_set_param(fe_vjp* v, const char* name, double value)
{
    if (v == nullptr || name == nullptr) return fe::fail(FE_EINVAL, "fe_vjp_set_param: null argument");
    const int p = fe_law_param_id(v->primal, name);
    if (p < 0) return fe::fail(FE_EINVAL, std::string("the law has no param '") + name + "'");
    int rc = fe_law_set_param(v->primal, p, value);
    if (rc != FE_OK) return rc;
    const int q = fe_law_param_id(v->adj, name);
    return q >= 0 ? fe_law_set_param(v->adj, q, value) : fe::ok();
}

int fe_vjp_forward(fe_vjp* v, double dt, int steps, int every)
{
    if (v == nullptr) return fe::fail(FE_EINVAL, "fe_vjp_forward: null handle");
    if (steps < 1 || !(dt > 0.0)) return fe::fail(FE_EINVAL, "fe_vjp_forward: steps >= 1 and dt > 0");
    v->steps = steps;
    v->dt = dt;
    v->every = every > 0 ? every : std::max(1, static_cast<int>(std::ceil(std::sqrt(static_cast<double>(steps)))));
    const std::size_t bytes = std::max<std::size_t>(v->cells * v->state.size() * sizeof(float), 4);
    const std::size_t count = static_cast<std::size_t>((steps + v->every - 1) / v->every);
    // The checkpoint buffers of the last forward serve this one when they fit (a calibration's repeated forwards
    // allocate once: cudaFree waits for the whole device).
    if (v->checkpoint_bytes != bytes) v->release();
    while (v->checkpoints.size() < count) {
        float* p = nullptr;
        const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), bytes);
        if (e != cudaSuccess) {
            v->release();
            return cuda_fail(e, "cudaMalloc (checkpoint)");
        }
        v->checkpoints.push_back(p);
        v->checkpoint_bytes = bytes;
    }
    v->used = 0;
    fe_step_info info{};
    for (int s = 0; s < steps; ++s) {
        int rc = FE_OK;
        if (s % v->every == 0 && (rc = save_state(v, v->checkpoints[static_cast<std::size_t>(s / v->every)])) != FE_OK) return rc;
        if ((rc = fe_law_step(v->primal, dt, 0, &info)) != FE_OK) return rc;
        const int sub = fe_law_substeps(v->primal, v->term);
        if (sub != 1) {
            return fe::fail(FE_EINVAL, "the differentiated term took " + std::to_string(sub) + " substeps: give a dt within its max_dt");
        }
    }
    int rc = fe_law_sync(v->primal, &info);
    if (rc != FE_OK) return rc;
    const int before = v->seen;
    v->seen = info.violations;
    if (info.violations > before) {
        fe_violation bad{};
        fe_law_violation(v->primal, before, &bad);
        return fe::fail(FE_ELAW, std::string("the forward broke a contract: ") + bad.detail);
    }
    v->used = count;
    return fe::ok();
}

int fe_vjp_backward(fe_vjp* v)
{
    if (v == nullptr) return fe::fail(FE_EINVAL, "fe_vjp_backward: null handle");
    if (v->used == 0) return fe::fail(FE_EINVAL, "fe_vjp_backward: no forward to go back over");
    const std::size_t per = v->cells * v->state.size();
    const std::size_t want = static_cast<std::size_t>(std::max(v->every, 1)) * std::max<std::size_t>(per, 1);
    if (v->segment_states < want) {
        if (v->segment != nullptr) cudaFree(v->segment);
        v->segment = nullptr;
        const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&v->segment), std::max(want, v->cells) * sizeof(float));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc (segment)");
        v->segment_states = std::max(want, v->cells);
    }
    // The static inputs as the forward saw them (they do not move): the primal's into the adjoint law's copies.
    int rc = FE_OK;
    for (std::size_t k = 0; k < v->statics.size(); ++k) {
        if ((rc = fe_law_fetch_device(v->primal, v->statics[k], v->segment)) != FE_OK) return rc;
        if ((rc = fe_law_upload_device(v->adj, v->statics_in_adj[k], v->segment)) != FE_OK) return rc;
    }
    fe_step_info info{};
    for (int seg = static_cast<int>(v->used) - 1; seg >= 0; --seg) {
        const int start = seg * v->every;
        const int end = std::min(v->steps, start + v->every);
        if ((rc = restore_state(v, v->checkpoints[static_cast<std::size_t>(seg)])) != FE_OK) return rc;
        for (int s = start; s < end; ++s) {
            if ((rc = save_state(v, v->segment + static_cast<std::size_t>(s - start) * per)) != FE_OK) return rc;
            if (s + 1 < end && (rc = fe_law_step(v->primal, v->dt, 0, &info)) != FE_OK) return rc;
        }
        for (int s = end - 1; s >= start; --s) {
            const float* at = v->segment + static_cast<std::size_t>(s - start) * per;
            for (const auto& [k, f] : v->state_to_adj) {
                if ((rc = fe_law_upload_device(v->adj, f, at + static_cast<std::size_t>(k) * v->cells)) != FE_OK) return rc;
            }
            if ((rc = fe_law_step(v->adj, v->dt, 0, &info)) != FE_OK) return rc;
        }
    }
    if ((rc = fe_law_sync(v->primal, &info)) != FE_OK) return rc;
    return fe_law_sync(v->adj, &info);
}

int fe_vjp_param_grad(fe_vjp* v, const char* param, double* grad)
{
    if (v == nullptr || param == nullptr || grad == nullptr) return fe::fail(FE_EINVAL, "fe_vjp_param_grad: null argument");
    const int f = fe_law_field_id(v->adj, (std::string(param) + "__adj").c_str());
    if (f < 0) return fe::fail(FE_EINVAL, std::string("the adjoint law carries no cotangent of '") + param + "'");
    std::vector<float> host(v->cells);
    const int rc = fe_law_fetch(v->adj, f, host.data());
    if (rc != FE_OK) return rc;
    double s = 0.0;
    for (const float x : host) s += x;
    *grad = s;
    return fe::ok();
}

} // extern "C"
