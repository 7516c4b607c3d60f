// IR to CUDA C++ for sm_100a (compiled by NVRTC at run time), and the launch plan the engine follows.
//
// What the reference's generator emits (src/field/cuda/CudaCodegen.cpp:300-908) is one thread a cell reading the fields
// through a ring-addressed constant table; this generator instead emits, per program, passes that march z through
// TMA-staged slabs of every buffer they read (the skeletons are fe_device.cuh's fe_slab_pass / fe_plain_pass), with the
// contracts of the term fused into the gather. The per-cell arithmetic is the reference's generated arithmetic, op for
// op (fp32, no FMA contraction), so a law's step on the card is the same numbers.
#pragma once

#include "ir.hpp"

#include <string>
#include <vector>

namespace fe::gen {

// A buffer a launch reads or writes.
struct Buf {
    enum Kind : unsigned char { FieldNow, FieldNext, Slot } kind = FieldNow;
    int id = -1; // field id or slot index
    bool operator==(const Buf& o) const { return kind == o.kind && id == o.id; }
};

struct Source {
    Buf buf;
    int ax = 0, ry = 0; // staged halo (ax a multiple of 4)
};

struct Launch {
    enum Kind : unsigned char { Pass, TridiagX, TridiagYZ, Reduce, Distance, Poisson, Net } kind = Pass;
    std::string kernel;       // the slab (TMA) kernel, or the only one
    std::string plain_kernel; // the plain-load twin of a Pass
    std::vector<Source> sources;
    std::vector<Buf> outs;
    std::vector<int> checked_fields; // per out: the field it checks (-1: not a contract output)
    int ty = 16;              // slab tile rows
    int nst = 4;              // ring depth
    int rz = 0;
    unsigned smem = 0;        // dynamic shared memory of the slab kernel (or the tridiag x kernel)
    int uniform = -1;         // Reduce: the uniform it writes
    int axis = 0;
    bool slab = true;         // the TMA variant is usable
    // Distance / Poisson: the kernel is the seed pass (the argument against what was last solved, a flag when it
    // changed); `aux` the first of the op's own slots, `flag` its word, `iterations` Poisson's sweeps.
    int aux = -1;
    int flag = -1;
    int iterations = 0;
    // Net: a `half` net op on the tensor cores (128 threads a CTA, persistent); at most this many CTAs an SM hold
    // tensor memory at once (the shared memory asked for keeps more from being resident).
    int per_sm = 0;
    // TridiagX: rows a lane of the warp-a-line partition solve (0: the 32-lines-a-block Thomas pass). TridiagYZ: rows
    // a segment of the 32-lines-a-block partition solve, `tri_segs` segments a line (0: a thread a line).
    int tri_rows = 0;
    int tri_segs = 0;
};

// The warp-a-line x solve: up to this many rows a lane (lines of up to 32 x this many cells), this many warps a block.
constexpr int kTriLaneRows = 16;
constexpr int kTriWarps = 4;

struct ProgramPlan {
    bool empty = true;
    std::vector<Launch> stages;       // per substep, in order
    std::vector<Launch> limit;        // before the substeps (the reductions max_dt reads)
    Launch gather;
    std::vector<int> swaps;           // fields whose next buffer becomes now after the gather (ping-pong)
    bool in_place = false;
};

struct Plan {
    int slots = 0;
    int uniforms = 0;
    std::vector<int> slot_of;     // per inst: its stored slot (stored stages, tridiag answers), or -1
    std::vector<int> uniform_of;  // per inst: reductions' uniform, or -1
    std::vector<int> aux_of;      // per inst: a distance's or poisson's own slots (after its answer), or -1
    int flags = 0;                // change flags of the distance and poisson ops
    std::vector<std::pair<int, unsigned>> slot_fill; // slots to fill at creation with a bit pattern
    std::vector<float> net_blob;  // the nets' parameters as the module's FE_NET holds them (weights, shift, scale, out scale)
    std::vector<unsigned short> net_bf16; // the `half` nets' weights as FE_NETB holds them (BF16, per layer K x N, core layout)
    std::vector<char> pingpong;   // per field: has a next buffer
    std::vector<ProgramPlan> terms, learned, derives;
    std::string source;           // the translation unit
};

// Generates the plan and the source for a lattice nx*ny*nz at cell size h. Returns false with `why` when the law uses
// what this backend does not run.
bool generate(const ir::Module& m, const law::Law& law, int nx, int ny, int nz, double h, Plan& plan, std::string& why);

// The embedded device prelude (fe_device.cuh).
const char* device_prelude();

} // namespace fe::gen
