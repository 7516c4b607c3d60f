/* fe.h — the C ABI of the B200 (sm_100a) backend for Field Engine laws.
 *
 * Plain pointers and sizes only. Every call returns an int status (FE_OK = 0, else an FE_E* code) and leaves a message
 * for fe_last_error() on the calling thread; no call throws or aborts. Host pointers passed in are read or written only
 * during the call. Device pointers are CUDA device addresses on the current device; `stream` is a cudaStream_t (NULL =
 * the legacy default stream).
 *
 * Each function names the reference interface it replaces (file:line in NotTruecCoder/online-physics-cuda).
 */
#ifndef FE_H
#define FE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FE_OK 0
#define FE_EINVAL 1    /* bad argument (sizes, ids, null pointers) */
#define FE_ENODEV 2    /* no usable sm_100 device / driver */
#define FE_ECUDA 3     /* a CUDA runtime, driver or NVRTC call failed */
#define FE_ELAW 4      /* the law does not compile (parse or validation errors) */
#define FE_EUNSUP 5    /* the law uses an op this backend does not run */
#define FE_EKERNEL 6   /* a kernel reported an error word (for example a bounded wait that gave up) */

/* ---- library ------------------------------------------------------------------------------------------------- */

/* ABI version (major * 1000 + minor). */
int fe_version(void);
/* The message of the last failing call on this thread ("" if none). */
const char* fe_last_error(void);
/* Whether an sm_100 device is usable; FE_ENODEV with the reason otherwise. Replaces CudaSolver::unavailable
 * (src/field/cuda/CudaSolver.hpp:30-32). */
int fe_device_check(void);

/* ---- contract record ---------------------------------------------------------------------------------------------
 * What one fused pass records per checked field (the reference keeps these in its record words R, filled by k_rows /
 * k_planes / k_range / k_bounds: src/field/cuda/CudaCodegen.cpp:182-250, judged in CudaSolver.cpp:530-571). */
typedef struct fe_check {
    double before;      /* sum of the field before the term (FP64, fixed order) */
    double before_abs;  /* sum of |field| before the term */
    double after;       /* sum after the term */
    double after_abs;   /* 0: the fused passes do not keep it (the judge scales by before_abs) */
    uint32_t out_of_range;
    uint32_t not_finite;
    uint32_t first_bad; /* ~(linear index of the first bad cell); 0 if none */
    uint32_t lo_inv;    /* ~key of the least value after the pass (fe_key_to_float(~lo_inv)) */
    uint32_t hi_key;    /* key of the largest value (fe_key_to_float(hi_key)); 0 = no finite value seen */
    uint32_t changed;   /* any cell moved */
    uint32_t pad[2];
} fe_check;

float fe_key_to_float(uint32_t key);

/* ---- the hand-written 7-point heat step --------------------------------------------------------------------------
 * d T = diffuse(k, T) with one k: next = T + ((max(k,0) * acc) / (h*h)) * dt, acc the sum of (neighbour - T) over the
 * faces inside the lattice in the order -x,+x,-y,+y,-z,+z. The bit-identity witness for the generated step; replaces the
 * reference's hand-written `heat` kernel (bench/stencil_bench.cpp:46-65), in the law's operation order.
 *
 * T_dev and out_dev: nx*ny*nz floats (x fastest), distinct buffers. variant: 0..3 picks the TMA tile (see fe_heat7_rows),
 * -1 the plain-load kernel (any nx). zchunk: z-planes a CTA marches (>= 1). With `check` non-zero the pass fills the
 * fe_check at the start of `workspace` (FE_HEAT7_BEFORE / FE_HEAT7_AFTER say which totals); workspace holds
 * fe_heat7_workspace_bytes(...) bytes and must be reset by fe_check_reset before the pass. */
#define FE_HEAT7_BEFORE 1
#define FE_HEAT7_AFTER 2
size_t fe_heat7_workspace_bytes(int nx, int ny, int nz, int variant, int zchunk);
int fe_heat7_rows(int variant);
int fe_heat7_step(const float* T_dev, float* out_dev, int nx, int ny, int nz, float k, float h, float dt, float lo, float hi,
    int variant, int zchunk, int check, void* workspace, void* stream);
/* Sets a workspace's fe_check and error word to their empty state (all zero bytes) on `stream`, asynchronously. */
int fe_check_reset(void* workspace, void* stream);
/* Copies the fe_check at the start of `workspace` to the host (synchronises `stream`); also reports a kernel error word
 * as FE_EKERNEL. */
int fe_check_read(const void* workspace, fe_check* out, void* stream);

/* A device-to-device copy of n floats (n a multiple of 4, 16-byte aligned): the bandwidth roof for the roofline. */
int fe_copy_f32(const float* src_dev, float* dst_dev, size_t n, void* stream);

/* fe_heat7_step without a workspace, for callers that cannot allocate device memory (their device memory belongs to
 * another allocator or pool, they are plugins in a process that forbids new device allocations, or they cannot afford
 * cudaMalloc's synchronisation in their loop). It has no counterpart in the reference. The contract pass's per-block
 * partial sums live in a fixed array in the library's device memory (every GPU that loads the library holds it, about
 * 256 KiB, until exit), which limits a pass to 8192 thread blocks: larger lattices are refused with FE_EINVAL (raise
 * zchunk). The caller passes the field buffers and a device fe_check `record_dev`, which the call clears and the pass
 * fills: needed with `check` (the contracts) and with a TMA variant (variant >= 0) even without `check`, since a
 * bounded wait that gives up raises the kernel's error word in record_dev->pad[0] (bit 1: a wait gave up; 0: none),
 * which the caller reads after the stream has run; optional for the plain kernel without `check`. The array is shared
 * by every call; each call clears what must start at zero, and calls that overlap on the GPU (several streams or host
 * threads) race on it: serialise them on one stream. The first call on a device looks up the array's device address
 * (once per device, with that device current); that first call may load the library's device code and with it create
 * the array, so make one call (for example on a one-cell lattice) before a region that may not allocate and before any
 * stream capture. The address is kept for the device's primary context: after cudaDeviceReset, or from another
 * context, it is stale. Nothing here calls cudaMalloc or cudaFree. */
int fe_heat7_step_noalloc(const float* T_dev, float* out_dev, int nx, int ny, int nz, float k, float h, float dt, float lo,
    float hi, int variant, int zchunk, int check, fe_check* record_dev, void* stream);

/* ---- the law backend ------------------------------------------------------------------------------------------------
 * A law (the reference's .law text, unchanged) compiled for one lattice nx*ny*nz of cell size h: parsed, lowered to the
 * SSA IR with the reference's rules, turned into sm_100a kernels (NVRTC), with its fields on the card. The handle is
 * single-threaded; handles are independent (each has its own stream). Replaces the reference's CudaSolver behind its
 * LawBackend interface (src/field/Backend.hpp:67-84; src/field/cuda/CudaSolver.cpp:46-1167). */
typedef struct fe_law fe_law;

/* Violation kinds (Violation::Kind, src/field/Backend.hpp:16-22). */
#define FE_RANGE 0
#define FE_NOT_FINITE 1
#define FE_CONSERVATION 2
#define FE_SUBSTEP_CAP 3

typedef struct fe_violation {
    int kind;
    int term;            /* the term's index, -1 for a derive */
    int field;           /* the field (the first of a conserved group), -1 for a substep cap */
    uint32_t count;      /* cells out of range / not finite */
    uint32_t first_cell; /* linear index (x fastest) of the first bad cell */
    double before, after, tolerance; /* conservation: the group's totals and the tolerance */
    long long step;      /* the step (0-based) the records belong to */
    char detail[160];
} fe_violation;

/* One conserves group's totals over one checked step, for a judge outside the handle (fe_law_take_totals). */
typedef struct fe_group_totals {
    long long step;      /* the step (0-based) */
    int term;            /* the term's index */
    int group;           /* the conserves group's index within the term */
    int substeps;        /* substeps the term took */
    int reserved;
    double before, after; /* sum of the group's fields before the term and after it, over the owned planes */
    double scale;        /* sum of |v| before the term (the tolerance scale, Solver.cpp:439-453) */
} fe_group_totals;

typedef struct fe_step_info {
    int violations;      /* violations now held (fe_law_violation) */
    int launches;        /* kernels the step launched */
    double gpu_ms;       /* the step's device time (0 when it did not wait for the card) */
    int fallbacks;       /* learned schemes undone this step (a broken contract; the classical scheme ran) */
} fe_step_info;

typedef struct fe_field_info {
    double init, lo, hi;
    int is_static, derived, clamp;
} fe_field_info;

/* Step flags. */
#define FE_STEP_IGNORE_MAX_DT 1 /* Solver::set_respect_max_dt(false): the falsification hook (Solver.hpp:91-93) */

/* Compiles `law_text` (one or more law sources joined; `source_name` names it in errors) for the lattice and puts its
 * fields on the current device at their `init` values. FE_ELAW with the compiler's messages, FE_EUNSUP for ops this
 * backend does not run. Replaces CudaSolver::create (src/field/cuda/CudaSolver.hpp:27, CudaSolver.cpp:1143-1152). */
int fe_law_create(const char* law_text, const char* source_name, int nx, int ny, int nz, double h, fe_law** out);
void fe_law_destroy(fe_law* law);
/* The same from the law's IR as the reference writes it (ir::to_json, src/field/ir/LawIR.cpp:528-593; lawc --ir-json):
 * for a host that holds a compiled Law rather than its text (the reference's CudaSolver::create takes a Law and lowers
 * it, CudaSolver.cpp:122). Nets' weights are read from the files the JSON names (the untrained start when a net has
 * none). The IR must lower back to itself here (same instructions and programs), else FE_ELAW. fe_law_ir_check does the
 * rebuilding and lowering without a device and writes this backend's JSON of it (text as for fe_law_ir_json). */
int fe_law_create_ir(const char* ir_json, int nx, int ny, int nz, double h, fe_law** out);
int fe_law_ir_check(const char* ir_json, char* buf, size_t cap, size_t* needed);
/* fe_law_source for a law given as its IR JSON (CudaSolver::source, src/field/cuda/CudaSolver.hpp:32). */
int fe_law_source_ir(const char* ir_json, int nx, int ny, int nz, double h, char* buf, size_t cap, size_t* needed);

/* Compile-only services, no device needed: the IR as the reference's JSON (lawc --ir-json, src/field/ir/LawIR.cpp:528-593)
 * or listing (lawc --ir, LawIR.cpp:595-656), and the generated CUDA translation unit (lawc --cuda, CudaSolver::source).
 * Text goes to buf (capacity cap, NUL-terminated); *needed gets the full length + 1. fe_law_compile_check also runs NVRTC
 * on the generated source (no GPU needed). */
int fe_law_ir_json(const char* law_text, char* buf, size_t cap, size_t* needed);
int fe_law_ir_listing(const char* law_text, char* buf, size_t cap, size_t* needed);
/* The adjoint law of `term` (NULL or "": the first), as law text: reverse mode over the term's SSA instructions, the
 * primal fields as static inputs, X__adj the cotangent of field or param X, tridiagonal solves by their transposes
 * (replaces src/field/ir/Adjoint.hpp:24 adjoint_law, which refuses tridiag). FE_EUNSUP with the reason for ops that
 * have no adjoint here. */
int fe_law_adjoint(const char* law_text, const char* term, char* buf, size_t cap, size_t* needed);
int fe_law_source(const char* law_text, int nx, int ny, int nz, double h, char* buf, size_t cap, size_t* needed);
int fe_law_compile_check(const char* law_text, int nx, int ny, int nz, double h);

/* Fields and params (Law::field_id / param_id, Solver::set_param; src/field/Law.hpp:196-199, Solver.hpp:55-56). */
int fe_law_field_count(const fe_law* law);
int fe_law_field_id(const fe_law* law, const char* name);
int fe_law_field_name(const fe_law* law, int field, char* buf, size_t cap);
int fe_law_field_info(const fe_law* law, int field, fe_field_info* out);
int fe_law_term_count(const fe_law* law);
int fe_law_term_name(const fe_law* law, int term, char* buf, size_t cap);
int fe_law_param_count(const fe_law* law);
int fe_law_param_id(const fe_law* law, const char* name);
int fe_law_set_param(fe_law* law, int param, double value);
int fe_law_get_param(const fe_law* law, int param, double* value);

/* Whole-field transfers (the host FieldSet <-> the card; FieldEdits::all and LawBackend::fetch, Backend.hpp:31-40, 79).
 * `host` holds nx*ny*nz floats, x fastest. The _device forms copy from / to a device buffer of the same size. */
int fe_law_upload(fe_law* law, int field, const float* host);
int fe_law_upload_device(fe_law* law, int field, const float* dev);
int fe_law_fetch(fe_law* law, int field, float* host);
int fe_law_fetch_device(fe_law* law, int field, float* dev);
/* Part of a field from the host array of the whole field (nx*ny*nz floats, x fastest): only the box [x0, x1) x [y0, y1)
 * x [z0, z1), or only the z-planes whose flag in `planes` (nz bytes) is set. The edits of the reference's host FieldSet
 * (FieldEdits::planes and ::boxes, src/field/Backend.hpp:28-40; the uploads of CudaSolver.cpp:779-920). */
int fe_law_upload_box(fe_law* law, int field, const float* host, int x0, int y0, int z0, int x1, int y1, int z1);
int fe_law_upload_planes(fe_law* law, int field, const float* host, const unsigned char* planes);
/* The window moved by (dx, dy, dz) cells (FieldEdits::shift, Backend.hpp:31-39; Solver::shift_window): the cell now at c
 * holds what was at c + d. Every field, and what distance and poisson keep from step to step (seeds, warm start),
 * moves on the card, the cells that left wrapping round to the side that arrives, as the reference's ring-addressed
 * lattice reads them after its origin moves (CudaCodegen.cpp:45-51); the caller then uploads the arriving boxes
 * (fe_law_upload_box). Here the cells move once a shift, at HBM rate, so that no kernel pays ring addressing every step. */
int fe_law_shift(fe_law* law, int dx, int dy, int dz);
/* The card's current buffer of a field (valid until the next step). */
/* The field's current device buffer was changed in place by the caller, on the handle's stream (fe_law_stream) after
 * its last step: the backend forgets what it knew of the field's bounds (no counterpart in the reference, whose host
 * FieldSet is written through FieldEdits instead). */
int fe_law_mark_edited(fe_law* law, int field);

/* A lattice split along z over ranks (no counterpart in the reference, whose CudaSolver runs one lattice on one GPU;
 * the z-slab form of CudaSolver::step over several GPUs). A rank's handle holds its slab plus halo planes copied from its
 * neighbours after every step:
 *   fe_law_set_owned_z: contracts (totals, bounds, range, change flag) cover planes [z0, z1) only;
 *   fe_law_mark_halo: the field's halo planes were written by the caller (its bounds are forgotten, the owned totals kept);
 *   fe_law_set_external_conservation: checked steps log each conserves group's totals (fe_law_take_totals, which hands
 *     over and clears the log, at most `max`, *n the count) instead of judging them: the caller sums over ranks;
 *   fe_law_plan_z_reach: for law text on a lattice (planned, not compiled): planes along z one step reads beyond a cell
 *     (*reach, summed over the step's passes; a term with learned equations counts the larger of its learned and
 *     classical passes) and flags: 1 the law reduces over the lattice, 2 it solves along z (neither splits into slabs;
 *     learned equations included, whether or not fe_law_set_learned turns them on later). */
int fe_law_set_owned_z(fe_law* law, int z0, int z1);
int fe_law_mark_halo(fe_law* law, int field);
int fe_law_set_external_conservation(fe_law* law, int on);
int fe_law_take_totals(fe_law* law, fe_group_totals* out, int max, int* n);
int fe_law_plan_z_reach(const char* law_text, int nx, int ny, int nz, double h, int* reach, int* flags);
int fe_law_field_device_ptr(const fe_law* law, int field, const float** dev);

/* One step of dt: every term in declaration order with its substeps, then the derives (Solver::step,
 * src/field/Solver.cpp:273-285; LawBackend::step). With contracts checked this step (fe_law_check_every) and not
 * deferred, waits for the card and judges them: fe_law_violation reads what broke. */
int fe_law_step(fe_law* law, double dt, int flags, fe_step_info* info);
/* Recomputes the derived fields (LawBackend::derive, Solver::refresh_derived). */
int fe_law_derive(fe_law* law);
/* Contracts looked at one step in `steps` (LawBackend::check_contracts_every). */
int fe_law_check_every(fe_law* law, int steps);
/* Deferred judging: checked steps keep their records on the card (up to 63 steps) and fe_law_sync judges them; the
 * steps then never wait for the host. Violations carry the step they belong to. */
int fe_law_set_deferred(fe_law* law, int on);
int fe_law_sync(fe_law* law, fe_step_info* info);
int fe_law_violation(const fe_law* law, int index, fe_violation* out);
/* Substeps term `term` took in the last step (Solver::last_substeps). */
int fe_law_substeps(const fe_law* law, int term);
/* Whether the term did nothing in the last step (its bounds said idle; TermProfile::idle). */
int fe_law_term_idle(const fe_law* law, int term);
/* Learned schemes under guard (Solver::set_learned, Solver.hpp; the guard Solver.cpp:314-336, CudaSolver.cpp:663-708):
 * with `on`, a term with `learned` equations runs them first on a snapshot of what it writes, its contracts judged at
 * once; a broken one undoes the step (never reported) and the classical equations run. fe_law_term_learned: 1 the
 * term's learned scheme was kept in the last step, 2 it was undone, 0 the classical scheme ran alone, -1 no such term. */
int fe_law_set_learned(fe_law* law, int on);
int fe_law_term_learned(const fe_law* law, int term);
/* FNV-1a over each field's name and then its values' bits, in declaration order (FieldSet::digest,
 * src/field/Grid.cpp:60-77): a state equal to the bit to a reference FieldSet gives the same digest. */
int fe_law_digest(fe_law* law, uint64_t* out);
/* The handle's stream (a cudaStream_t), for callers that order their own work after its steps. */
int fe_law_stream(const fe_law* law, void** stream);
/* Device time of `launches` back-to-back launches of term `term`'s fused gather pass (the roofline's kernel). */
int fe_law_time_gather(fe_law* law, int term, int launches, float* ms);
/* The same for stage `stage` of the term (its stored stages and tridiagonal solves, in launch order) at step dt; its
 * kernel's name goes to `kernel` (capacity cap). FE_EINVAL when the term has no such stage. */
int fe_law_time_stage(fe_law* law, int term, int stage, int launches, double dt, float* ms, char* kernel, size_t cap);

/* ---- batched instances: one law on many uneven lattices ---------------------------------------------------------------
 * The reference batches instances as the z-planes of one lattice, all of the same nx x ny (bench/finance.py:253-288,
 * bench/pdebench.py:71-92). fe_batch_create takes n instances of any extents and h. Instances of equal (nx, ny, h) share
 * one lattice, stacked along z in order, when the law couples nothing along z (no value read across planes, no
 * lattice-wide reduction, distance or poisson, no solve along z, no `rim`); otherwise every instance is a lattice of
 * its own (fe_batch_info: how many, and whether stacked; fe_batch_plan: the same grouping without a device). Each
 * lattice is a law handle with its own stream (fe_batch_law: an instance's handle and first plane, for params and
 * profiles); fe_batch_step launches every lattice's step, then judges all their contracts. A stacked lattice's
 * conserved totals are judged over all its instances together, as the reference's z-plane batches are. Violations
 * carry their instance (-1: a conserved total of a lattice holding several), range/NaN cells numbered within the
 * instance. fe_batch_set_param sets a param everywhere; fe_batch_upload / _fetch move one instance's field
 * (nx*ny*nz floats, x fastest) from / to the host. */
typedef struct fe_batch_desc {
    int nx, ny, nz;
    double h;
} fe_batch_desc;
typedef struct fe_batch fe_batch;
int fe_batch_create(const char* law_text, const fe_batch_desc* descs, int n, fe_batch** out);
/* lattice_of and z0: arrays of n (or NULL) that get each instance's lattice and its first plane there. */
int fe_batch_plan(const char* law_text, const fe_batch_desc* descs, int n, int* lattices, int* stacked, int* lattice_of, int* z0);
void fe_batch_destroy(fe_batch* batch);
int fe_batch_info(const fe_batch* batch, int* lattices, int* stacked);
int fe_batch_law(fe_batch* batch, int instance, fe_law** law, int* z0);
int fe_batch_set_param(fe_batch* batch, int param, double value);
int fe_batch_upload(fe_batch* batch, int instance, int field, const float* host);
int fe_batch_fetch(fe_batch* batch, int instance, int field, float* host);
int fe_batch_step(fe_batch* batch, double dt, int flags, int* violations);
int fe_batch_violation(const fe_batch* batch, int index, int* instance, fe_violation* out);

/* ---- reverse mode through a law's steps ------------------------------------------------------------------------------
 * N steps of one term of a law and their vector-Jacobian product, natively (replaces the reference's lawc --vjp driver,
 * tools/lawc/main.cpp:274-361, which keeps every state on the host and uploads one before each adjoint step). The handle
 * holds two law handles (fe_vjp_laws): the primal law, and its adjoint law (fe_law_adjoint: X__adj the cotangent of
 * field or param X). The differentiated term must be the only one that moves anything, one substep a step.
 *   fe_vjp_forward: steps the primal `steps` times from its current fields, keeping every `every`-th state of its
 *     moving fields on the device (every <= 0: ceil(sqrt(steps))); FE_EINVAL when the term took more than one substep,
 *     FE_ELAW when a contract broke;
 *   fe_vjp_backward: from the cotangents the caller put in the adjoint law's X__adj fields (the seeds; the adjoint law's
 *     other fields are filled here), steps the adjoint law back over the forward's states, each segment recomputed
 *     from its checkpoint; afterwards X__adj holds the cotangent of X at the forward's start, and the primal's fields
 *     are left at a recomputed state;
 *   fe_vjp_param_grad: a param's gradient, the FP64 sum of its cotangent field.
 * Device memory: about (steps / every + every) copies of the moving fields. */
typedef struct fe_vjp fe_vjp;
int fe_vjp_create(const char* law_text, const char* term, int nx, int ny, int nz, double h, fe_vjp** out);
void fe_vjp_destroy(fe_vjp* vjp);
int fe_vjp_laws(fe_vjp* vjp, fe_law** primal, fe_law** adjoint);
int fe_vjp_set_param(fe_vjp* vjp, const char* name, double value);
int fe_vjp_forward(fe_vjp* vjp, double dt, int steps, int every);
int fe_vjp_backward(fe_vjp* vjp);
int fe_vjp_param_grad(fe_vjp* vjp, const char* param, double* grad);

/* ---- batched Heston ADI: many options on uneven grids in one persistent launch -----------------------------------------
 * The reference prices a batch as the z-planes of one lattice, every option on the same grid (bench/finance.py:253-288,
 * bench/laws/heston_adi.law); here every option has its own grid and all are stepped by one persistent kernel of 8-CTA
 * clusters that keeps each option's state in shared memory from its first step to its last (an option of more than 16K
 * cells split by rows over 2, 4 or 8 CTAs of a cluster, neighbours read over distributed shared memory), with the law's
 * discretisation (tests/laws/heston_douglas.law, heston_hv.law): x lines by warp segments (PCR/Thomas hybrid), y lines
 * by the partition method across the CTAs. x = ln S on [ln K - 3, ln K + 3] with h = 6 / nx; the variance rows var_j =
 * sigma (j + 1/2) h; the put payoff averaged over each cell; price at (ln spot, v0) by bilinear interpolation between
 * cell centres. No counterpart in the reference's C++ API. */
#define FE_ADI_DOUGLAS 0
#define FE_ADI_HV 1
typedef struct fe_heston_option {
    int nx, ny;           /* powers of two: nx in [4, 512], ny in [4, 256] */
    float strike, maturity, spot, v0;
    float kappa, theta, sigma, rho, r;
} fe_heston_option;
typedef struct fe_heston_batch fe_heston_batch;
/* n in [1, 65535] options, `steps` time steps each to its maturity, scheme FE_ADI_DOUGLAS or FE_ADI_HV. */
int fe_heston_batch_create(const fe_heston_option* options, int n, int steps, int scheme, fe_heston_batch** out);
void fe_heston_batch_destroy(fe_heston_batch* batch);
/* The split of the work: mx cells a lane holds in the x solves (4, 8 or 16; an x line takes nx / mx lanes of a warp,
 * at most 32 for every option), sy the most row blocks a CTA cuts a column into for the y solves (1, 2, 4, 8 or 16),
 * threads a CTA (256, 384 or 512: fewer threads, more registers each). */
int fe_heston_batch_set_split(fe_heston_batch* batch, int mx, int sy, int threads);
/* Times short runs of every split that fits the batch and keeps the fastest (the outputs may be NULL). */
int fe_heston_batch_autotune(fe_heston_batch* batch, int* mx, int* sy, int* threads);
/* The persistent grid's 8-CTA clusters and the batch's tasks (8 / C options split over C CTAs each). */
int fe_heston_batch_layout(const fe_heston_batch* batch, int* clusters, int* tasks);
/* Sets up the payoffs and steps every option to maturity (asynchronous on the batch's stream). With use_graph the
 * launch sequence is captured once into a CUDA graph and replayed. */
int fe_heston_batch_run(fe_heston_batch* batch, int use_graph);
/* Device time of one run (ms). */
int fe_heston_batch_time(fe_heston_batch* batch, int use_graph, float* ms);
/* The prices of the last run (n floats) and one option's grid (nx * ny floats, x fastest). Both wait for the run. */
int fe_heston_batch_prices(fe_heston_batch* batch, float* host_prices);
int fe_heston_batch_grid(fe_heston_batch* batch, int option, float* host_grid);

/* ---- learned coarse-lattice correction on the tensor cores ----------------------------------------------------------------
 * A small network applied per cell of a coarse 2-D lattice (each z-plane a sample) after the plain law's step: the 3 x 3
 * neighbourhood of (u, v), edge repeating, -> 64 (ReLU) -> 64 (ReLU) -> 2, added to (u, v): a 3x3 convolution, then two
 * pointwise layers, BF16 on the tensor cores (tcgen05) with FP32 accumulation, trained by the library's own forward and
 * backward kernels (loss 1/2 mean over cells of the squared error against a target state; Adam on FP32 masters). It
 * replaces the reference's fp16 mma.sync net stages (src/field/cuda/CudaNet.cpp:175-369) for this form; the plain fine
 * law stays the judge, and fe_corr_apply is guarded: the corrected state replaces the plain step's only if every cell is
 * finite and within [lo, hi] (decided on the card). Weights are fe_corr_weight_count() floats: W1 (32 x 64) | W2 (80 x 64)
 * | W3 (80 x 16), row-major, rows = inputs (W1 rows 0..17 the neighbourhood as (u, v) pairs row by row, row 18 the bias,
 * row 19 the `time` input; W2, W3 row 64 the bias; other rows, and W3 columns past 1, zero). `time` is the time since the
 * start of the solve of the state being corrected. Device pointers are float32 nx * ny * nz lattices; `stream` is a
 * cudaStream_t (NULL: the legacy stream). */
typedef struct fe_corrector fe_corrector;
int fe_corr_create(fe_corrector** out);
void fe_corr_destroy(fe_corrector* corr);
int fe_corr_weight_count(void);
int fe_corr_set_weights(fe_corrector* corr, const float* host_weights);
int fe_corr_get_weights(fe_corrector* corr, float* host_weights);
/* The loss and its gradient (host_grads may be NULL) of the network on (u, v) against (target_u, target_v). */
int fe_corr_grads(fe_corrector* corr, const float* u, const float* v, const float* target_u, const float* target_v, int nx, int ny,
                  int nz, float time, void* stream, double* host_loss, float* host_grads);
/* One Adam step (learning rate lr) on that gradient; host_loss (may be NULL) is the loss before the step. */
int fe_corr_train_step(fe_corrector* corr, const float* u, const float* v, const float* target_u, const float* target_v, int nx,
                       int ny, int nz, float time, void* stream, float lr, double* host_loss);
/* (u, v) += the network's correction, in place, guarded; *reverted (may be NULL: no wait for the verdict) is 1 when the
 * plain step's state was kept. */
int fe_corr_apply(fe_corrector* corr, float* u, float* v, int nx, int ny, int nz, float time, float lo, float hi, void* stream,
                  int* reverted);

#ifdef __cplusplus
}
#endif

#endif /* FE_H */
