// The law backend on one B200: a compiled law on one lattice, its device buffers, and the step.
//
// Replaces the reference's CudaSolver (src/field/cuda/CudaSolver.cpp:46-1140) behind the same LawBackend semantics
// (src/field/Backend.hpp:67-84): Lie splitting over terms in declaration order, substeps from max_dt (capped at 4096),
// gather-then-apply with in-place or ping-pong stores, derives after the terms, the contracts (conserved totals,
// range/NaN) checked on the card and judged by the host, idle terms skipped by the bounds test. What differs is the
// schedule: the contracts ride in the gather pass, a step issues no host round trip unless it reads a max_dt reduction
// or judges its contracts, and the judging may be deferred (records kept on the card until fe_law_sync).
#pragma once

#include "codegen.hpp"
#include "cuda_ctx.hpp"
#include "ir.hpp"
#include "law.hpp"

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace fe {

struct Violation {
    int kind = 0;   // 0 range, 1 not finite, 2 conservation, 3 substep cap (Backend.hpp:16-22)
    int term = -1;  // -1: a derive
    int field = -1;
    unsigned count = 0;
    unsigned first_cell = 0;
    double before = 0.0, after = 0.0, tolerance = 0.0;
    long long step = 0;
    std::string detail;
};

struct Bounds {
    double lo = -1.0 / 0.0;
    double hi = 1.0 / 0.0;
    [[nodiscard]] bool none() const { return lo == 0.0 && hi == 0.0; }
};

// The totals of one conserves group over one checked step, kept for a judge outside the engine (a lattice split in
// z-slabs over ranks is conserved as a whole, not slab by slab).
struct GroupTotals {
    long long step = 0;
    int term = 0;
    int group = 0;
    int substeps = 1;
    double before = 0.0, after = 0.0, scale = 0.0;
};

// How many planes along z one step of a planned law reads beyond a cell (the sum over its passes, in order; a term with
// learned equations counts the larger of its learned and classical programs), and whether it reduces over the lattice
// or solves along z (neither splits into z-slabs), its learned programs included.
void plan_z_reach(const gen::Plan& plan, int& reach, bool& reductions, bool& z_solves);

struct TermProfile {
    int launches = 0;
    int substeps = 0;
    bool idle = false;
    bool learned = false;   // the term's learned scheme ran and was kept
    bool fell_back = false; // it ran, broke a contract, was undone, and the classical scheme ran instead
};

class Engine {
public:
    ~Engine();
    bool create(const std::vector<law::Source>& sources, int nx, int ny, int nz, double h, std::string& why);
    // From a law already compiled and lowered (a law given as its IR).
    bool create(law::Law law, ir::Module module, int nx, int ny, int nz, double h, std::string& why);

    // Host <-> card.
    bool upload(int field, const void* src, bool device, std::string& why);
    // The lattice's window moved by (dx, dy, dz) cells: the cell now at c holds what was at c + d (FieldEdits::shift,
    // src/field/Backend.hpp:31-39). Every field and per-cell slot is carried over, the cells that left wrapping round
    // to the arriving side, as a ring-addressed lattice would read them; the caller then uploads the arriving boxes.
    bool shift(int dx, int dy, int dz, std::string& why);
    // Uploads only the cells of a box [x0, x1) x [y0, y1) x [z0, z1), or only the flagged z-planes, from a host array
    // of the whole field (the reference's host FieldSet is the truth between steps; CudaSolver.cpp:779-920).
    bool upload_box(int field, const float* host, const int box[6], std::string& why);
    bool upload_planes(int field, const float* host, const unsigned char* planes, std::string& why);
    // A field's cells were changed in place on the device by someone else (ordered on the engine's stream): what the
    // engine knew of its bounds no longer holds.
    void mark_edited(int field);
    // Halo planes of a field (outside the owned z-range) were written by someone else: its bounds are unknown, while
    // the totals of the owned planes still hold.
    void mark_halo(int field);
    // Contracts (totals, bounds, range, change) cover planes [z0, z1) only: the rest are halo planes another rank owns.
    bool set_owned_z(int z0, int z1);
    // Conservation is judged outside: each checked step's group totals go to a log instead (take_totals).
    void set_external_conservation(bool on) { external_conservation_ = on; }
    std::vector<GroupTotals> take_totals();
    bool fetch(int field, void* dst, bool device, std::string& why);
    const float* device_field(int field) const { return now_[static_cast<std::size_t>(field)]; }

    bool set_param(int id, double value);
    bool step(double dt, bool respect_max_dt, std::string& why);
    bool derive(std::string& why);
    bool sync(std::string& why); // judges pending contract records

    void check_every(int steps) { check_every_ = steps < 1 ? 1 : steps; }
    void set_deferred(bool on) { deferred_ = on; }
    // Learned schemes under guard (Solver::set_learned, Solver.cpp:314-336): a term with learned equations runs them
    // first on a snapshot of what it writes; a broken contract undoes the step and the classical equations run.
    void set_learned(bool on) { learned_ = on; }
    int fallbacks_last_step() const { return fallbacks_; }

    const law::Law& law() const { return law_; }
    const ir::Module& module() const { return mod_; }
    const gen::Plan& plan() const { return plan_; }
    const std::vector<Violation>& violations() const { return violations_; }
    const std::vector<int>& substeps() const { return substeps_; }
    const std::vector<TermProfile>& term_profile() const { return term_profile_; }
    int launches_last_step() const { return launches_; }
    double gpu_ms_last_step() const { return gpu_ms_; }
    cudaStream_t stream() const { return stream_; }
    long long steps_taken() const { return steps_; }
    int nx() const { return nx_; }
    int ny() const { return ny_; }
    int nz() const { return nz_; }
    std::size_t cells() const { return cells_; }
    double compile_ms() const { return compile_ms_; }
    const std::vector<Bounds>& bounds() const { return bounds_; }

    // Times one term's gather pass alone (the measured kernel of the roofline): `launches` back-to-back launches of the
    // gather on the current state (ping-pong targets are written to their next buffer; nothing is swapped).
    bool time_gather(int term, int launches, float& ms, std::string& why);
    // Times stage `stage` of term `term` (its stored stages and tridiagonal solves, in order) the same way, at step dt.
    bool time_stage(int term, int stage, int launches, double dt, float& ms, std::string& kernel, std::string& why);

private:
    struct RecordRef {
        int term;      // -1 derive
        int field;
        int rec;       // index of the FeCheck in the ring slot
        int substeps;
        bool totals;   // this record carries before/after totals
    };
    struct PendingStep {
        long long step;
        int ring;      // ring slot
        std::vector<RecordRef> refs;
        std::vector<std::vector<std::vector<int>>> conserves; // per term: groups of fields
    };

    bool push_params(std::string& why);
    bool launch(const gen::Launch& L, float dt, int flags, FeCheck* const* recs, std::string& why, const FeCheck* const* carry = nullptr);
    bool conserved_by(int term, int field) const;
    bool launch_solve(const gen::Launch& L, float dt, std::string& why);
    bool buffer(const gen::Buf& b, float*& out) const;
    bool map_for(const float* base, int bx, int by, FeTensorMap& out, std::string& why);
    CUfunction function(const std::string& name, unsigned smem, std::string& why);
    int zchunk_for(const gen::Launch& L, bool slab);
    // CTAs of a slab pass an SM holds at once (its shared memory and its registers both counted), cached by kernel.
    int resident(const gen::Launch& L);
    bool run_program(int index, const ir::Program& p, const gen::ProgramPlan& pp, double dt, bool respect, bool check,
        PendingStep& pending, std::string& why);
    bool judge(PendingStep& pending, std::string& why);
    bool judge_into(const PendingStep& pending, std::vector<Violation>& out, std::string& why);
    bool apply_term(int t, double dt, bool respect, bool check, PendingStep& pending, std::string& why);
    double scalar_value(int id, bool& ok, std::string& why);
    bool idle(const ir::Program& p) const;
    Bounds bounds_of(int id, const std::vector<Bounds>& fields) const;
    Bounds bounds_one(int id, const std::vector<Bounds>& fields, const std::vector<Bounds>& memo) const;
    bool always_zero(int id) const;
    bool zero_one(int id, const std::vector<char>& memo) const;
    void flow_bounds(const ir::Program& p, double dt, int substeps);

    law::Law law_;
    ir::Module mod_;
    gen::Plan plan_;
    int nx_ = 0, ny_ = 0, nz_ = 0;
    double h_ = 1.0;
    std::size_t cells_ = 0;
    cudaStream_t stream_ = nullptr;
    CUmodule module_ = nullptr;
    std::map<std::string, CUfunction> functions_;
    std::map<std::string, int> resident_;
    CUdeviceptr params_ = 0;
    CUdeviceptr uniforms_ = 0;
    void* arena_ = nullptr;
    std::vector<float*> now_, next_, slot_;
    std::map<std::tuple<const float*, int, int>, FeTensorMap> maps_;
    // Contracts: a ring of per-step record blocks, shared partials and block counters.
    FeCheck* records_ = nullptr;
    int records_per_step_ = 0;
    int ring_ = 0;
    int ring_next_ = 0;
    double* partials_ = nullptr;
    std::size_t partial_doubles_ = 0;
    unsigned* counts_ = nullptr; // FE_MAX_OUT counters, then the error word
    unsigned* flags_ = nullptr;  // change flags of the distance and poisson ops
    FeCheck* bounds_rec_ = nullptr; // the bounds of an upload (lo_inv / hi_key keys)
    float* rotate_scratch_ = nullptr; // one field's cells, for moving the window (allocated at the first shift)
    bool measure_bounds(int field, std::string& why); // the field's exact bounds, taken on the card
    std::vector<PendingStep> pending_;
    std::vector<double> param_host_;
    bool params_dirty_ = true;
    int check_every_ = 1;
    bool deferred_ = false;
    long long steps_ = 0;
    std::vector<Violation> violations_;
    std::vector<int> substeps_;
    std::vector<TermProfile> term_profile_;
    std::vector<Bounds> bounds_;
    std::vector<char> zero_;
    // Per field: the record holding the totals of its current contents (ring slot, index, step), written by the checked
    // gather that last wrote it; step -1 when none does (never checked, edited since, or written unchecked).
    struct Carry {
        int ring = -1;
        int rec = -1;
        long long step = -1;
    };
    std::vector<Carry> carry_;
    int own_z0_ = 0, own_z1_ = 0;
    bool learned_ = false;
    int fallbacks_ = 0;
    float* snapshot_ = nullptr;   // what a guarded learned scheme writes, kept to undo it
    std::size_t snapshot_fields_ = 0;
    bool external_conservation_ = false;
    std::vector<GroupTotals> totals_log_;
    int launches_ = 0;
    double gpu_ms_ = 0.0;
    double compile_ms_ = 0.0;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    int sms_ = 148;
};

} // namespace fe
