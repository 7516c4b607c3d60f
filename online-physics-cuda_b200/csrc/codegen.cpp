#include "codegen.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <functional>
#include <map>
#include <set>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <sstream>

namespace fe::gen {

const char* device_prelude()
{
    static const char* text =
#include "fe_device_prelude.inc"
        ;
    return text;
}

namespace {

using ir::Inst;
using ir::Shape;
using law::Op;

// A float literal as the reference prints it (%.9g of the float value; CudaCodegen.cpp:278-295).
std::string literal(double v)
{
    if (!std::isfinite(v)) return v > 0 ? "1e30f" : (v < 0 ? "(-1e30f)" : "0.f");
    const float f = static_cast<float>(v);
    if (!std::isfinite(f)) return f > 0 ? "__int_as_float(0x7f800000)" : "__int_as_float(0xff800000)";
    char text[48];
    std::snprintf(text, sizeof(text), "%.9g", static_cast<double>(f));
    std::string s = text;
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return "(" + s + "f)";
}

struct Radius {
    int x = 0, y = 0, z = 0;
};

// How far along each axis an op reads its arguments from its own cell.
Radius axis_radius(const Inst& in)
{
    switch (in.op) {
    case Op::Shift: case Op::ShiftT:
        return {std::abs(in.offset[0]), std::abs(in.offset[1]), std::abs(in.offset[2])};
    case Op::Lap: case Op::Diffuse: case Op::Adv: case Op::Topple:
        return {1, 1, 1};
    case Op::Gx: case Op::GxT: return {1, 0, 0};
    case Op::Gy: case Op::GyT: return {0, 1, 0};
    case Op::Gz: case Op::GzT: return {0, 0, 1};
    case Op::Fall: return {0, 0, 1};
    case Op::Spread: return {1, 1, 0};
    case Op::Flux: return {1, 1, 1};
    case Op::LDiffuse: return {2, 2, 2};
    default: return {};
    }
}

// The offsets (dx, dy, dz) at which an op reads its arguments, relative to its own cell: the exact points of the
// stencils, the whole box where the points depend on values (spread, topple) or run over a range (the transposed
// shifts), and the cell itself for the pointwise ops.
void read_points(const Inst& in, std::vector<std::array<int, 3>>& pts)
{
    pts.clear();
    auto box = [&](int rx, int ry, int rz) {
        for (int dz = -rz; dz <= rz; ++dz)
            for (int dy = -ry; dy <= ry; ++dy)
                for (int dx = -rx; dx <= rx; ++dx) pts.push_back({dx, dy, dz});
    };
    auto star = [&](bool x, bool y, bool z) {
        pts.push_back({0, 0, 0});
        if (x) pts.insert(pts.end(), {{-1, 0, 0}, {1, 0, 0}});
        if (y) pts.insert(pts.end(), {{0, -1, 0}, {0, 1, 0}});
        if (z) pts.insert(pts.end(), {{0, 0, -1}, {0, 0, 1}});
    };
    switch (in.op) {
    case Op::Shift: pts.push_back({in.offset[0], in.offset[1], in.offset[2]}); break;
    case Op::ShiftT: box(std::abs(in.offset[0]), std::abs(in.offset[1]), std::abs(in.offset[2])); break;
    case Op::Lap: case Op::Diffuse: case Op::Adv: case Op::Flux: star(true, true, true); break;
    case Op::Gx: case Op::GxT: star(true, false, false); break;
    case Op::Gy: case Op::GyT: star(false, true, false); break;
    case Op::Gz: case Op::GzT: case Op::Fall: star(false, false, true); break;
    case Op::Spread: box(1, 1, 0); break;
    default: {
        const Radius r = axis_radius(in);
        box(r.x, r.y, r.z);
    }
    }
}

bool supported_cell_op(Op op)
{
    switch (op) {
    case Op::Local:
        return false;
    default:
        return true;
    }
}

class Generator {
public:
    Generator(const ir::Module& m, const law::Law& law, int nx, int ny, int nz, double h, Plan& plan)
        : m_(m), law_(law), nx_(nx), ny_(ny), nz_(nz), h_(h), plan_(plan)
    {
    }

    bool run(std::string& why)
    {
        plan_.slot_of.assign(m_.insts.size(), -1);
        plan_.uniform_of.assign(m_.insts.size(), -1);
        plan_.aux_of.assign(m_.insts.size(), -1);
        plan_.pingpong.assign(law_.fields.size(), 0);
        if (!allocate(why)) return false;
        out_ << device_prelude() << "\n";
        out_ << "__constant__ float FE_P[1024];\n";
        out_ << "__device__ float FE_U[" << std::max(plan_.uniforms, 1) << "];\n";
        out_ << "constexpr int NX = " << nx_ << ", NY = " << ny_ << ", NZ = " << nz_ << ";\n";
        out_ << "constexpr float FE_H = " << literal(h_) << ";\n";
        {
            char hd[48];
            std::snprintf(hd, sizeof(hd), "%.17g", h_);
            out_ << "constexpr double FE_HD = " << hd << ";\n";
        }
        emit_nets();
        out_ << R"(__device__ __forceinline__ int fe_ex(int v) { return v < 0 ? 0 : (v >= NX ? NX - 1 : v); }
__device__ __forceinline__ int fe_ey(int v) { return v < 0 ? 0 : (v >= NY ? NY - 1 : v); }
__device__ __forceinline__ int fe_ez(int v) { return v < 0 ? 0 : (v >= NZ ? NZ - 1 : v); }
__device__ __forceinline__ bool fe_inside(int x, int y, int z) { return x >= 0 && y >= 0 && z >= 0 && x < NX && y < NY && z < NZ; }
// IN: the cell and every point its expressions read lie inside the lattice (the pass checked its reach), so clamps are
// the identity and edge tests are true; the same arithmetic, with the index work and the branches compiled away.
template <bool IN> __device__ __forceinline__ int fe_cx(int v) { return IN ? v : fe_ex(v); }
template <bool IN> __device__ __forceinline__ int fe_cy(int v) { return IN ? v : fe_ey(v); }
template <bool IN> __device__ __forceinline__ int fe_cz(int v) { return IN ? v : fe_ez(v); }
__device__ __forceinline__ int fe_imin(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int fe_imax(int a, int b) { return a > b ? a : b; }
__device__ __forceinline__ void fe_run_to(int j, int d, int n, int& lo, int& hi)
{
    lo = fe_imax(j == 0 ? 0 : j - d, 0); hi = fe_imin(j == n - 1 ? n - 1 : j - d, n - 1);
}
__device__ __forceinline__ float fe_dv(float a, float b) { return b == 0.f ? 0.f : a / b; }
__device__ __forceinline__ float fe_sat(float v) { return fminf(fmaxf(v, 0.f), 1.f); }
__device__ __forceinline__ float fe_face(float ka, float kb, float va, float vb)
{
    const float s = ka + kb;
    return (s > 0.f ? 2.f * ka * kb / s : 0.f) * (vb - va);
}
)";
        for (std::size_t t = 0; t < m_.terms.size(); ++t) {
            if (!program(m_.terms[t], "t" + std::to_string(t), false, plan_.terms.emplace_back(), why)) return false;
            if (!program(m_.learned[t], "l" + std::to_string(t), false, plan_.learned.emplace_back(), why)) return false;
        }
        for (std::size_t d = 0; d < m_.derives.size(); ++d) {
            if (!program(m_.derives[d], "d" + std::to_string(d), true, plan_.derives.emplace_back(), why)) return false;
        }
        plan_.source = out_.str();
        return true;
    }

private:
    [[nodiscard]] const Inst& at(int id) const { return m_.insts[static_cast<std::size_t>(id)]; }

    bool allocate(std::string& why)
    {
        std::set<int> used;
        auto take = [&](const ir::Program& p) {
            used.insert(p.stages.begin(), p.stages.end());
            used.insert(p.limit_stages.begin(), p.limit_stages.end());
        };
        for (const ir::Program& p : m_.terms) take(p);
        for (const ir::Program& p : m_.learned) take(p);
        for (const ir::Program& p : m_.derives) take(p);
        for (const int id : used) {
            const Inst& in = at(id);
            switch (in.op) {
            case Op::Tridiag:
                plan_.slot_of[static_cast<std::size_t>(id)] = plan_.slots;
                plan_.slots += 2; // the answer, and c' of the y/z recurrence
                break;
            case Op::MaxOf: case Op::MinOf: case Op::SumOf:
                plan_.uniform_of[static_cast<std::size_t>(id)] = plan_.uniforms++;
                break;
            case Op::Distance:
                // The answer, then seeds inside and outside, two scratch passes, squared distances to inside and
                // outside (CudaSolver.cpp:394-418). The seeds start unlike any seed, so the first look solves.
                plan_.slot_of[static_cast<std::size_t>(id)] = plan_.slots;
                plan_.aux_of[static_cast<std::size_t>(id)] = plan_.slots + 1;
                plan_.slot_fill.emplace_back(plan_.slots + 1, 0xffffffffu);
                plan_.slots += 7;
                flag_of_[id] = plan_.flags++;
                break;
            case Op::Poisson:
                // The answer (warm-started from zero), the source as last solved (starting unlike any source), and
                // the other half of the Jacobi ping-pong (CudaSolver.cpp:420-434).
                plan_.slot_of[static_cast<std::size_t>(id)] = plan_.slots;
                plan_.aux_of[static_cast<std::size_t>(id)] = plan_.slots + 1;
                plan_.slot_fill.emplace_back(plan_.slots, 0u);
                plan_.slot_fill.emplace_back(plan_.slots + 1, 0xffffffffu);
                plan_.slots += 3;
                flag_of_[id] = plan_.flags++;
                break;
            default:
                plan_.slot_of[static_cast<std::size_t>(id)] = plan_.slots++;
                break;
            }
        }
        for (const Inst& in : m_.insts) {
            if (!supported_cell_op(in.op)) {
                why = std::string("this backend does not run '") + law::op_name(in.op) + "' yet";
                return false;
            }
        }
        if (m_.insts.empty()) return true;
        return true;
    }

    // ---- one pass: its sources, their halos, and its device code ------------------------------------------------------

    struct PassBuild {
        std::vector<Source> sources;
        std::vector<Radius> reach;            // per source
        std::set<int> own_stages;             // stages whose bodies this pass computes
        std::set<std::pair<int, std::tuple<int, int, int>>> seen;
        // The plane carry: per source, whether it is read below the cell's plane, and whether any such read is other
        // than the cell's own column one plane down; cslot the carry slot of each source (-1: none).
        std::set<std::pair<int, std::tuple<int, int, int>>> seen_points;
        std::vector<char> below, below_off;
        std::vector<int> cslot;
        bool zcarry = false;
    };

    int source_index(PassBuild& pb, Buf buf)
    {
        for (std::size_t k = 0; k < pb.sources.size(); ++k) {
            if (pb.sources[k].buf == buf) return static_cast<int>(k);
        }
        pb.sources.push_back(Source{buf});
        pb.reach.push_back({});
        pb.below.push_back(0);
        pb.below_off.push_back(0);
        return static_cast<int>(pb.sources.size()) - 1;
    }

    // The same closure as walk(), with signed offsets: which sources are read below the cell's plane, and whether each
    // such read is the cell's own column one plane down (what the plane carry can serve).
    void walk_points(PassBuild& pb, int id, int dx, int dy, int dz, bool body)
    {
        const Inst& in = at(id);
        if (!pb.seen_points.insert({id * 2 + (body ? 1 : 0), {dx, dy, dz}}).second) return;
        const bool stored = m_.is_stage(id) || in.global;
        int k = -1;
        if (!body && stored) {
            if (in.shape == Shape::Scalar) return;
            k = source_index(pb, Buf{Buf::Slot, plan_.slot_of[static_cast<std::size_t>(id)]});
        } else if (in.op == Op::Field) {
            k = source_index(pb, Buf{Buf::FieldNow, in.index});
        }
        if (k >= 0) {
            if (dz < 0) {
                pb.below[static_cast<std::size_t>(k)] = 1;
                if (dz != -1 || dx != 0 || dy != 0) pb.below_off[static_cast<std::size_t>(k)] = 1;
            }
            return;
        }
        std::vector<std::array<int, 3>> pts;
        read_points(in, pts);
        for (const auto& p : pts) {
            for (const int arg : in.args) walk_points(pb, arg, dx + p[0], dy + p[1], dz + p[2], false);
        }
    }

    // The plane carry applies when the pass reads one plane each way (RZ = 1), every read below the plane is the cell's
    // own column, and at most two sources need carrying (their cells of one plane live in registers).
    void plan_carry(PassBuild& pb)
    {
        pb.cslot.assign(pb.sources.size(), -1);
        pb.zcarry = false;
        int rz = 0;
        for (const Radius& r : pb.reach) rz = std::max(rz, r.z);
        if (rz != 1) return;
        int n = 0;
        for (std::size_t k = 0; k < pb.sources.size(); ++k) {
            if (pb.below_off[k]) return;
            if (pb.below[k]) pb.cslot[k] = n++;
        }
        if (n == 0 || n > 2) {
            pb.cslot.assign(pb.sources.size(), -1);
            return;
        }
        pb.zcarry = true;
    }

    // Walks a value's inlined closure with the offset it is read at, growing the sources' reach. `body`: evaluate this
    // instruction itself even if it is a stage (the stage a pass stores); otherwise a stage is a read of its slot.
    void walk(PassBuild& pb, int id, Radius off, bool body)
    {
        const Inst& in = at(id);
        if (!pb.seen.insert({id * 2 + (body ? 1 : 0), {off.x, off.y, off.z}}).second) return;
        const bool stored = m_.is_stage(id) || in.global;
        if (!body && stored) {
            if (in.shape == Shape::Scalar) return; // a reduction's uniform
            const int k = source_index(pb, Buf{Buf::Slot, plan_.slot_of[static_cast<std::size_t>(id)]});
            Radius& r = pb.reach[static_cast<std::size_t>(k)];
            r.x = std::max(r.x, off.x);
            r.y = std::max(r.y, off.y);
            r.z = std::max(r.z, off.z);
            return;
        }
        if (in.op == Op::Field) {
            const int k = source_index(pb, Buf{Buf::FieldNow, in.index});
            Radius& r = pb.reach[static_cast<std::size_t>(k)];
            r.x = std::max(r.x, off.x);
            r.y = std::max(r.y, off.y);
            r.z = std::max(r.z, off.z);
            return;
        }
        const Radius a = axis_radius(in);
        const Radius next{off.x + a.x, off.y + a.y, off.z + a.z};
        for (const int arg : in.args) walk(pb, arg, next, false);
    }

    // The device functions of a pass: v<id>(c, x, y, z) for every instruction its outputs inline (stages it reads, and
    // fields, are loads of their source) and b<id> for the bodies of the stages it stores.
    void emit_functions(std::ostringstream& f, PassBuild& pb, const std::vector<int>& roots, bool bodies)
    {
        std::set<int> done;
        std::vector<std::pair<int, bool>> order;
        std::function<void(int, bool)> visit = [&](int id, bool body) {
            const int key = id * 2 + (body ? 1 : 0);
            if (done.count(key)) return;
            const Inst& in = at(id);
            const bool stored = (m_.is_stage(id) || in.global) && !body;
            if (!stored) {
                for (const int a : in.args) visit(a, false);
            }
            done.insert(key);
            order.emplace_back(id, body);
        };
        for (const int r : roots) visit(r, bodies);
        for (const auto& [id, body] : order) emit_inst(f, pb, id, body);
    }

    static std::string v(int id, const std::string& x = "x", const std::string& y = "y", const std::string& z = "z")
    {
        return "v" + std::to_string(id) + "<IN>(c, " + x + ", " + y + ", " + z + ")";
    }

    void emit_inst(std::ostringstream& f, PassBuild& pb, int id, bool body)
    {
        const Inst& in = at(id);
        const std::string name = (body ? "b" : "v") + std::to_string(id);
        f << "template <bool IN, class C> __device__ __forceinline__ float " << name << "(const C& c, int x, int y, int z)";
        auto a = [&](std::size_t k, const std::string& x = "x", const std::string& y = "y", const std::string& z = "z") {
            return v(in.args[k], x, y, z);
        };
        auto simple = [&](const std::string& e) { f << " { return " << e << "; }\n"; };
        const bool stored = (m_.is_stage(id) || in.global) && !body;
        if (stored) {
            if (in.shape == Shape::Scalar) {
                simple("FE_U[" + std::to_string(plan_.uniform_of[static_cast<std::size_t>(id)]) + "]");
            } else {
                const int k = source_index(pb, Buf{Buf::Slot, plan_.slot_of[static_cast<std::size_t>(id)]});
                simple("c.template ld<" + std::to_string(k) + ">(x, y, z)");
            }
            return;
        }
        switch (in.op) {
        case Op::Const: simple(literal(in.number)); break;
        case Op::Param: simple("FE_P[" + std::to_string(in.index) + "]"); break;
        case Op::Cell: simple("FE_H"); break;
        case Op::Dt: simple("c.dt"); break;
        case Op::Rim: simple("(x == 0 || y == 0 || z == 0 || x + 1 == NX || y + 1 == NY || z + 1 == NZ) ? 1.f : 0.f"); break;
        case Op::Local: simple("0.f"); break;
        case Op::Field: {
            const int k = source_index(pb, Buf{Buf::FieldNow, in.index});
            simple("c.template ld<" + std::to_string(k) + ">(x, y, z)");
            break;
        }
        case Op::Neg: simple("-" + a(0)); break;
        case Op::Abs: simple("fabsf(" + a(0) + ")"); break;
        case Op::Sqrt: simple("sqrtf(fmaxf(0.f, " + a(0) + "))"); break;
        case Op::Exp: simple("expf(fminf(" + a(0) + ", 80.f))"); break;
        case Op::Log: simple("logf(fmaxf(" + a(0) + ", 1e-30f))"); break;
        case Op::Step: simple(a(0) + " > 0.f ? 1.f : 0.f"); break;
        case Op::Pos: simple("fmaxf(" + a(0) + ", 0.f)"); break;
        case Op::Add: simple(a(0) + " + " + a(1)); break;
        case Op::Sub: simple(a(0) + " - " + a(1)); break;
        case Op::Mul: simple(a(0) + " * " + a(1)); break;
        case Op::Div: simple("fe_dv(" + a(0) + ", " + a(1) + ")"); break;
        case Op::Pow: simple("powf(" + a(0) + ", " + a(1) + ")"); break;
        case Op::Min: simple("fminf(" + a(0) + ", " + a(1) + ")"); break;
        case Op::Max: simple("fmaxf(" + a(0) + ", " + a(1) + ")"); break;
        case Op::Clamp:
            f << " { const float lo = " << a(1) << "; return fminf(fmaxf(" << a(0) << ", lo), fmaxf(lo, " << a(2) << ")); }\n";
            break;
        case Op::Shift:
            simple(a(0, "fe_cx<IN>(x + " + std::to_string(in.offset[0]) + ")", "fe_cy<IN>(y + " + std::to_string(in.offset[1]) + ")",
                "fe_cz<IN>(z + " + std::to_string(in.offset[2]) + ")"));
            break;
        case Op::ShiftT:
            f << " { int lx, hx, ly, hy, lz, hz; fe_run_to(x, " << in.offset[0] << ", NX, lx, hx); fe_run_to(y, " << in.offset[1]
              << ", NY, ly, hy); fe_run_to(z, " << in.offset[2] << ", NZ, lz, hz);\n"
              << "    float s = 0.f; for (int k = lz; k <= hz; ++k) for (int j = ly; j <= hy; ++j) for (int i = lx; i <= hx; ++i) s += "
              << a(0, "i", "j", "k") << ";\n    return s; }\n";
            break;
        case Op::GxT: case Op::GyT: case Op::GzT: {
            const int axis = in.op == Op::GxT ? 0 : (in.op == Op::GyT ? 1 : 2);
            const char* cc = axis == 0 ? "x" : (axis == 1 ? "y" : "z");
            const char* n = axis == 0 ? "NX" : (axis == 1 ? "NY" : "NZ");
            const std::string at_q = axis == 0 ? a(0, "q", "y", "z") : (axis == 1 ? a(0, "x", "q", "z") : a(0, "x", "y", "q"));
            f << " { float s = 0.f;\n"
              << "    for (int d = 1; d >= -1; d -= 2) { int lo, hi; fe_run_to(" << cc << ", d, " << n << ", lo, hi);\n"
              << "        for (int q = lo; q <= hi; ++q) { const int span = fe_imin(q + 1, " << n << " - 1) - fe_imax(q - 1, 0);\n"
              << "            const float w = span > 0 ? " << at_q << " / (FE_H * span) : 0.f; s += d > 0 ? w : -w; } }\n"
              << "    return s; }\n";
            break;
        }
        case Op::Lap:
            f << " { const float c0 = " << a(0) << "; return ((" << a(0, "fe_cx<IN>(x - 1)") << " - c0) + (" << a(0, "fe_cx<IN>(x + 1)")
              << " - c0) + (" << a(0, "x", "fe_cy<IN>(y - 1)") << " - c0) + (" << a(0, "x", "fe_cy<IN>(y + 1)") << " - c0) + ("
              << a(0, "x", "y", "fe_cz<IN>(z - 1)") << " - c0) + (" << a(0, "x", "y", "fe_cz<IN>(z + 1)") << " - c0)) / (FE_H * FE_H); }\n";
            break;
        case Op::Gx:
            f << " { const int hi = fe_cx<IN>(x + 1); const int lo = fe_cx<IN>(x - 1); const int span = hi - lo; return span > 0 ? ("
              << a(0, "hi") << " - " << a(0, "lo") << ") / (FE_H * span) : 0.f; }\n";
            break;
        case Op::Gy:
            f << " { const int hi = fe_cy<IN>(y + 1); const int lo = fe_cy<IN>(y - 1); const int span = hi - lo; return span > 0 ? ("
              << a(0, "x", "hi") << " - " << a(0, "x", "lo") << ") / (FE_H * span) : 0.f; }\n";
            break;
        case Op::Gz:
            f << " { const int hi = fe_cz<IN>(z + 1); const int lo = fe_cz<IN>(z - 1); const int span = hi - lo; return span > 0 ? ("
              << a(0, "x", "y", "hi") << " - " << a(0, "x", "y", "lo") << ") / (FE_H * span) : 0.f; }\n";
            break;
        case Op::Diffuse: {
            static const char* sides[6][4] = {{"IN || x > 0", "x - 1", "y", "z"}, {"IN || x + 1 < NX", "x + 1", "y", "z"},
                {"IN || y > 0", "x", "y - 1", "z"}, {"IN || y + 1 < NY", "x", "y + 1", "z"}, {"IN || z > 0", "x", "y", "z - 1"},
                {"IN || z + 1 < NZ", "x", "y", "z + 1"}};
            // A face's flux is antisymmetric to the bit: (b - a) = -(a - b) in IEEE arithmetic, and the harmonic mean is
            // symmetric in its two conductivities. So the lower face of a cell (-x, -y, -z) is written as its lower
            // neighbour's upper face, subtracted: acc - (c - nb) is acc + (nb - c) exactly (acc, a sum from +0, is never
            // -0). The cells a lane computes side by side along x and the rows it computes along y then name the same
            // difference twice, and the compiler computes it once (CudaCodegen.cpp:193-206 is the arithmetic kept).
            static const bool lower[6] = {true, false, true, false, true, false};
            if (at(in.args[0]).shape == Shape::Scalar) {
                // One k everywhere: the harmonic mean of a face is k itself.
                f << " { const float c0 = " << a(1) << "; float acc = 0.f;\n";
                for (int k = 0; k < 6; ++k) {
                    const auto& s = sides[k];
                    if (lower[k]) f << "    if (" << s[0] << ") acc -= c0 - " << a(1, s[1], s[2], s[3]) << ";\n";
                    else f << "    if (" << s[0] << ") acc += " << a(1, s[1], s[2], s[3]) << " - c0;\n";
                }
                f << "    return fmaxf(" << a(0) << ", 0.f) * acc / (FE_H * FE_H); }\n";
            } else {
                f << " { const float ka = " << a(0) << "; const float c0 = " << a(1) << "; float acc = 0.f;\n";
                for (int k = 0; k < 6; ++k) {
                    const auto& s = sides[k];
                    if (lower[k]) {
                        f << "    if (" << s[0] << ") acc -= fe_face(" << a(0, s[1], s[2], s[3]) << ", ka, " << a(1, s[1], s[2], s[3]) << ", c0);\n";
                    } else {
                        f << "    if (" << s[0] << ") acc += fe_face(ka, " << a(0, s[1], s[2], s[3]) << ", c0, " << a(1, s[1], s[2], s[3]) << ");\n";
                    }
                }
                f << "    return acc / (FE_H * FE_H); }\n";
            }
            break;
        }
        case Op::Adv: {
            auto up = [&](const std::string& speed, const char* pos, const char* count, const std::string& lo, const std::string& hi) {
                return "(" + speed + " > 0.f ? ((IN || " + pos + " > 0) ? " + speed + " * (c0 - " + lo + ") / FE_H : 0.f) : ((IN || " + pos +
                    " + 1 < " + count + ") ? " + speed + " * (" + hi + " - c0) / FE_H : 0.f))";
            };
            f << " { const float c0 = " << a(0) << "; const float u = " << a(1) << "; const float w = " << a(2) << "; const float s = " << a(3)
              << ";\n    return -(" << up("u", "x", "NX", a(0, "x - 1"), a(0, "x + 1")) << " + "
              << up("w", "y", "NY", a(0, "x", "y - 1"), a(0, "x", "y + 1")) << " + "
              << up("s", "z", "NZ", a(0, "x", "y", "z - 1"), a(0, "x", "y", "z + 1")) << "); }\n";
            break;
        }
        case Op::Fall: {
            const std::string n = std::to_string(id);
            f << ";\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float fall" << n << "(const C& c, int x, int y, int z) { if (!IN && z == 0) return 0.f;\n"
              << "    return fmaxf(0.f, " << a(2) << ") / FE_H * fmaxf(0.f, " << a(0) << ") * fe_sat(1.f - " << a(1, "x", "y", "z - 1")
              << " - " << a(0, "x", "y", "z - 1") << "); }\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float " << name << "(const C& c, int x, int y, int z)"
              << " { float o = -fall" << n << "<IN>(c, x, y, z); if (IN || z + 1 < NZ) o += fall" << n << "<IN>(c, x, y, z + 1); return o; }\n";
            break;
        }
        case Op::Spread: {
            const std::string n = std::to_string(id);
            f << ";\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float spread" << n << "(const C& c, int ax, int ay, int az, int bx, int by, int bz) {\n"
              << "    const float fa = " << a(0, "ax", "ay", "az") << "; const float fb = " << a(0, "bx", "by", "bz") << ";\n"
              << "    const bool to_b = fa > fb; const int rx = to_b ? bx : ax; const int ry = to_b ? by : ay; const int rz = to_b ? bz : az;\n"
              << "    return 0.5f * (fmaxf(0.f, " << a(2, "ax", "ay", "az") << ") + fmaxf(0.f, " << a(2, "bx", "by", "bz")
              << ")) / (FE_H * FE_H) * (fa - fb) * fe_sat(1.f - " << a(1, "rx", "ry", "rz") << " - " << a(0, "rx", "ry", "rz") << "); }\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float " << name << "(const C& c, int x, int y, int z)"
              << " { float o = 0.f;\n"
              << "    if (IN || y > 0) o += spread" << n << "<IN>(c, x, y - 1, z, x, y, z);\n"
              << "    if (IN || x > 0) o += spread" << n << "<IN>(c, x - 1, y, z, x, y, z);\n"
              << "    if (IN || x + 1 < NX) o -= spread" << n << "<IN>(c, x, y, z, x + 1, y, z);\n"
              << "    if (IN || y + 1 < NY) o -= spread" << n << "<IN>(c, x, y, z, x, y + 1, z);\n"
              << "    return o; }\n";
            break;
        }
        case Op::Topple: {
            const std::string n = std::to_string(id);
            f << ";\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float room" << n << "(const C& c, int x, int y, int z) { return fe_sat(1.f - " << a(1)
              << " - " << a(0) << "); }\n"
              << "template <bool IN, class C> __device__ __forceinline__ float send" << n << "(const C& c, int x, int y, int z, int sx, int sy) {\n"
              << "    const float here = " << a(0) << "; if (here <= 0.f || (!IN && z == 0)) return 0.f;\n"
              << "    if (room" << n << "<IN>(c, x, y, z - 1) > 0.01f) return 0.f;\n"
              << "    const int jx = x + sx; const int jy = y + sy; if (!IN && !fe_inside(jx, jy, z)) return 0.f;\n"
              << "    return 0.25f * fmaxf(0.f, " << a(2) << ") / FE_H * here * fminf(room" << n << "<IN>(c, jx, jy, z), room" << n << "<IN>(c, jx, jy, z - 1)); }\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float " << name << "(const C& c, int x, int y, int z)"
              << " { float o = 0.f;\n"
              << "    o -= send" << n << "<IN>(c, x, y, z, -1, 0); o -= send" << n << "<IN>(c, x, y, z, 1, 0); o -= send" << n << "<IN>(c, x, y, z, 0, -1); o -= send"
              << n << "<IN>(c, x, y, z, 0, 1);\n"
              << "    if (IN || z + 1 < NZ) {\n"
              << "        if (IN || x + 1 < NX) o += send" << n << "<IN>(c, x + 1, y, z + 1, -1, 0);\n"
              << "        if (IN || x > 0) o += send" << n << "<IN>(c, x - 1, y, z + 1, 1, 0);\n"
              << "        if (IN || y + 1 < NY) o += send" << n << "<IN>(c, x, y + 1, z + 1, 0, -1);\n"
              << "        if (IN || y > 0) o += send" << n << "<IN>(c, x, y - 1, z + 1, 0, 1);\n"
              << "    }\n    return o; }\n";
            break;
        }
        case Op::Mlp: {
            // mlp(NET, a...): the net at the cell, its first output (Law.cpp:1298-1333).
            const law::NetDecl& net = law_.nets[static_cast<std::size_t>(in.index)];
            f << " { float xin[" << in.args.size() << "];\n";
            for (std::size_t k = 0; k < in.args.size(); ++k) f << "    xin[" << k << "] = " << a(k) << ";\n";
            f << "    float yout[" << net.sizes.back() << "]; fe_net" << in.index << "(xin, yout); return yout[0]; }\n";
            break;
        }
        case Op::Flux: {
            // flux(NET, F, a..., lo, hi): across each face (i below, j above) the net sees both sides both ways round;
            // half the difference, limited, is what moves from i to j; a cell gains its lower faces' and loses its upper
            // faces', over h (Law.cpp:1335-1389, 691-706). Both cells of a face compute it the same way: antisymmetric.
            const law::NetDecl& net = law_.nets[static_cast<std::size_t>(in.index)];
            const std::size_t m = in.args.size() - 2;
            const double lo = at(in.args[m]).number;
            const double hi = at(in.args[m + 1]).number;
            const std::string n = std::to_string(id);
            char bounds[96];
            std::snprintf(bounds, sizeof(bounds), "%.17g, %.17g", lo, hi);
            f << ";\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float face" << n
              << "(const C& c, int ix, int iy, int iz, int jx, int jy, int jz) {\n    float xij[" << 2 * m << "], xji[" << 2 * m << "];\n";
            for (std::size_t k = 0; k < m; ++k) {
                f << "    { const float vi = " << a(k, "ix", "iy", "iz") << "; const float vj = " << a(k, "jx", "jy", "jz") << "; xij[" << k
                  << "] = vi; xij[" << m + k << "] = vj; xji[" << k << "] = vj; xji[" << m + k << "] = vi; }\n";
            }
            f << "    float y[" << net.sizes.back() << "]; fe_net" << in.index << "(xij, y); const float gij = y[0]; fe_net" << in.index
              << "(xji, y); const float gji = y[0];\n"
              << "    return fe_limit_face(0.5f * (gij - gji), xij[0], xij[" << m << "], " << bounds << ", c.dt); }\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float " << name << "(const C& c, int x, int y, int z)"
              << " { float o = 0.f;\n"
              << "    if (IN || x > 0) o += face" << n << "<IN>(c, x - 1, y, z, x, y, z);\n"
              << "    if (IN || x + 1 < NX) o -= face" << n << "<IN>(c, x, y, z, x + 1, y, z);\n"
              << "    if (IN || y > 0) o += face" << n << "<IN>(c, x, y - 1, z, x, y, z);\n"
              << "    if (IN || y + 1 < NY) o -= face" << n << "<IN>(c, x, y, z, x, y + 1, z);\n"
              << "    if (IN || z > 0) o += face" << n << "<IN>(c, x, y, z - 1, x, y, z);\n"
              << "    if (IN || z + 1 < NZ) o -= face" << n << "<IN>(c, x, y, z, x, y, z + 1);\n"
              << "    return o / FE_H; }\n";
            break;
        }
        case Op::LDiffuse: {
            // ldiffuse(NET, k, F): the flux through a face from the window F[i-1] F[i] | F[j] F[j+1] (edge cells repeat),
            // with weights the net gives around the classical [0 -1 1 0]; each way round, half the difference
            // (Law.cpp:1391-1438, 708-738). k's face value is the harmonic mean, in double like the reference.
            const std::string n = std::to_string(id);
            f << ";\n";
            f << "__device__ __forceinline__ float lraw" << n << "(const float* w, float kf, float dt) {\n"
              << "    const float centre = 0.5f * (w[1] + w[2]); float spread = 1e-6f;\n"
              << "#pragma unroll\n    for (int q = 0; q < 4; ++q) spread = fmaxf(spread, fabsf(w[q] - centre));\n"
              << "    float xin[5];\n#pragma unroll\n    for (int q = 0; q < 4; ++q) xin[q] = (w[q] - centre) / spread;\n"
              << "    xin[4] = kf * dt / (FE_H * FE_H);\n"
              << "    float yw[4]; fe_net" << in.index << "(xin, yw);\n"
              << "    const float mean = 0.25f * (yw[0] + yw[1] + yw[2] + yw[3]);\n"
              << "    const float base[4] = {0.f, -1.f, 1.f, 0.f}; float acc = 0.f;\n"
              << "#pragma unroll\n    for (int q = 0; q < 4; ++q) acc += (base[q] + (yw[q] - mean)) * w[q];\n"
              << "    return -kf / FE_H * acc; }\n";
            // The face between cell i = (x, y, z) and its +AX neighbour j.
            f << "template <bool IN, int AX, class C> __device__ __forceinline__ float ldface" << n << "(const C& c, int x, int y, int z) {\n"
              << "    const int jx = x + (AX == 0), jy = y + (AX == 1), jz = z + (AX == 2);\n"
              << "    const int q = AX == 0 ? x : (AX == 1 ? y : z); const int count = AX == 0 ? NX : (AX == 1 ? NY : NZ);\n"
              << "    const int mx = (IN || q > 0) ? x - (AX == 0) : x, my = (IN || q > 0) ? y - (AX == 1) : y, mz = (IN || q > 0) ? z - (AX == 2) : z;\n"
              << "    const int px = (IN || q + 2 < count) ? jx + (AX == 0) : jx, py = (IN || q + 2 < count) ? jy + (AX == 1) : jy,"
              << " pz = (IN || q + 2 < count) ? jz + (AX == 2) : jz;\n"
              << "    const float w[4] = {" << a(1, "mx", "my", "mz") << ", " << a(1, "x", "y", "z") << ", " << a(1, "jx", "jy", "jz") << ", "
              << a(1, "px", "py", "pz") << "};\n"
              << "    const double ka = " << a(0, "x", "y", "z") << ", kb = " << a(0, "jx", "jy", "jz") << ";\n"
              << "    const float kf = static_cast<float>((ka + kb) > 0.0 ? 2.0 * ka * kb / (ka + kb) : 0.0);\n"
              << "    const float mirror[4] = {w[3], w[2], w[1], w[0]};\n"
              << "    const float ij = lraw" << n << "(w, kf, c.dt); const float ji = lraw" << n << "(mirror, kf, c.dt);\n"
              << "    return 0.5f * (ij - ji); }\n";
            f << "template <bool IN, class C> __device__ __forceinline__ float " << name << "(const C& c, int x, int y, int z)"
              << " { float o = 0.f;\n"
              << "    if (IN || x > 0) o += ldface" << n << "<IN, 0>(c, x - 1, y, z);\n"
              << "    if (IN || x + 1 < NX) o -= ldface" << n << "<IN, 0>(c, x, y, z);\n"
              << "    if (IN || y > 0) o += ldface" << n << "<IN, 1>(c, x, y - 1, z);\n"
              << "    if (IN || y + 1 < NY) o -= ldface" << n << "<IN, 1>(c, x, y, z);\n"
              << "    if (IN || z > 0) o += ldface" << n << "<IN, 2>(c, x, y, z - 1);\n"
              << "    if (IN || z + 1 < NZ) o -= ldface" << n << "<IN, 2>(c, x, y, z);\n"
              << "    return o / FE_H; }\n";
            break;
        }
        case Op::Tridiag: case Op::MaxOf: case Op::MinOf: case Op::SumOf:
            // Only as a body: the stage kernels evaluate their arguments directly.
            simple("0.f");
            break;
        default:
            simple("0.f");
            break;
        }
    }

    // The law's nets: their parameters in one module array, FE_NET (the engine writes plan.net_blob there), and a
    // forward function a net, fe_net<k>(in, out), in the reference's order (Net.cpp:93-153): inputs shifted and scaled,
    // then per layer out[o] = bias[o] + sum_i W[o][i] x[i] in i order, the activation on every layer but the last, the
    // outputs times out_scale. fp32, no FMA contraction, like the reference's CPU nets.
    void emit_nets()
    {
        std::ostringstream f;
        for (std::size_t k = 0; k < law_.nets.size(); ++k) {
            const law::NetDecl& net = law_.nets[k];
            const std::size_t w0 = plan_.net_blob.size();
            plan_.net_blob.insert(plan_.net_blob.end(), net.weights.begin(), net.weights.end());
            const std::size_t sh = plan_.net_blob.size();
            plan_.net_blob.insert(plan_.net_blob.end(), net.in_shift.begin(), net.in_shift.end());
            const std::size_t sc = plan_.net_blob.size();
            plan_.net_blob.insert(plan_.net_blob.end(), net.in_scale.begin(), net.in_scale.end());
            const std::size_t os = plan_.net_blob.size();
            plan_.net_blob.push_back(net.out_scale);
            net_at_.push_back(NetAt{w0, sh, sc, os, pack_half(net)});
            const std::string act = net.act == "tanh" ? "tanhf(v)" : net.act == "relu" ? "(v > 0.f ? v : 0.f)" : net.act == "silu" ? "v / (1.f + expf(-v))" : "v";
            f << "__device__ __forceinline__ float fe_act" << k << "(float v) { return " << act << "; }\n";
            f << "__device__ __forceinline__ void fe_net" << k << "(const float* in, float* out) {\n";
            const int n0 = net.sizes.front();
            f << "    float h0[" << n0 << "];\n#pragma unroll\n    for (int i = 0; i < " << n0 << "; ++i) h0[i] = (in[i] - FE_NET[" << sh << " + i]) * FE_NET[" << sc
              << " + i];\n";
            for (int l = 0; l < net.layers(); ++l) {
                const int ni = net.sizes[static_cast<std::size_t>(l)];
                const int no = net.sizes[static_cast<std::size_t>(l) + 1];
                const std::size_t wl = w0 + net.weight_offset(l);
                const bool last = l + 1 == net.layers();
                f << "    float h" << l + 1 << "[" << no << "];\n#pragma unroll\n    for (int o = 0; o < " << no << "; ++o) {\n"
                  << "        float acc = FE_NET[" << wl + static_cast<std::size_t>(ni) * no << " + o];\n#pragma unroll\n        for (int i = 0; i < " << ni
                  << "; ++i) acc += FE_NET[" << wl << " + o * " << ni << " + i] * h" << l << "[i];\n"
                  << "        h" << l + 1 << "[o] = " << (last ? "acc" : "fe_act" + std::to_string(k) + "(acc)") << ";\n    }\n";
            }
            f << "#pragma unroll\n    for (int o = 0; o < " << net.sizes.back() << "; ++o) out[o] = h" << net.layers() << "[o] * FE_NET[" << os << "];\n}\n";
        }
        out_ << "__device__ float FE_NET[" << std::max<std::size_t>(1, plan_.net_blob.size()) << "];\n";
        out_ << "__device__ __align__(16) unsigned short FE_NETB[" << std::max<std::size_t>(8, plan_.net_bf16.size()) << "];\n";
        out_ << R"(// The flux limiter of flux(): the same on both sides of a face, so the flux stays antisymmetric; within one step of dt
// no cell goes below the moved field's least or above its most (Law.cpp:672-689).
__device__ __forceinline__ float fe_limit_face(float r, float fi, float fj, double lo, double hi, float dt)
{
    if (!(dt > 0.f)) return r;
    const float per = static_cast<float>(0.999 * FE_HD / (6.0 * static_cast<double>(dt)));
    const bool has_lo = lo > -1e29, has_hi = hi < 1e29;
    if (r > 0.f) {
        if (has_lo) r = fminf(r, fmaxf(0.f, (fi - static_cast<float>(lo)) * per));
        if (has_hi) r = fminf(r, fmaxf(0.f, (static_cast<float>(hi) - fj) * per));
    } else if (r < 0.f) {
        if (has_lo) r = fmaxf(r, -fmaxf(0.f, (fj - static_cast<float>(lo)) * per));
        if (has_hi) r = fmaxf(r, -fmaxf(0.f, (static_cast<float>(hi) - fi) * per));
    }
    return r;
}
)";
        out_ << f.str();
    }

    // The pass traits: lattice, tile, sources' layout, outputs' checks.
    void emit_traits(std::ostringstream& f, const PassBuild& pb, const Launch& L, int nout, const std::vector<char>& checked)
    {
        const int nsrc = static_cast<int>(pb.sources.size());
        f << "struct P {\n"
          << "    static constexpr int NX = ::NX, NY = ::NY, NZ = ::NZ;\n"
          << "    static constexpr int W = 8, R = " << L.ty / 8 << ", RZ = " << L.rz << ", NST = " << L.nst << ", NSRC = " << nsrc
          << ", NOUT = " << nout << ";\n";
        std::vector<int> ax, ry, px, pl, base;
        int off = 0;
        unsigned bytes = 0;
        for (const Source& s : pb.sources) {
            const int p_x = 128 + 2 * s.ax;
            const int p_y = L.ty + 2 * s.ry;
            const int plane = (p_x * p_y + 31) / 32 * 32;
            ax.push_back(s.ax);
            ry.push_back(s.ry);
            px.push_back(p_x);
            pl.push_back(plane);
            base.push_back(off);
            off += plane * L.nst;
            bytes += static_cast<unsigned>(p_x * p_y * 4);
        }
        auto fn = [&](const char* name, const std::vector<int>& v) {
            f << "    static __device__ __forceinline__ constexpr int " << name << "(int k) { ";
            for (std::size_t k = 0; k < v.size(); ++k) f << "if (k == " << k << ") return " << v[k] << "; ";
            f << "return 0; }\n";
        };
        fn("ax", ax);
        fn("ry", ry);
        fn("px", px);
        fn("pl", pl);
        fn("base", base);
        f << "    static constexpr unsigned BYTES = " << bytes << "u;\n";
        {
            int ncarry = 0;
            std::vector<int> cs;
            for (std::size_t k = 0; k < pb.sources.size(); ++k) {
                const int v = pb.zcarry && k < pb.cslot.size() ? pb.cslot[k] : -1;
                cs.push_back(v);
                ncarry = std::max(ncarry, v + 1);
            }
            f << "    static constexpr bool ZCARRY = " << (pb.zcarry ? "true" : "false") << ";\n"
              << "    static constexpr int NCARRY = " << ncarry << ";\n"
              << "    static __device__ __forceinline__ constexpr int cslot(int k) { ";
            for (std::size_t k = 0; k < cs.size(); ++k) f << "if (k == " << k << ") return " << cs[k] << "; ";
            f << "return -1; }\n";
        }
        // The pass's true reach along each axis (unrounded): a cell this far from every face is interior (IN).
        int rxt = 0, ryt = 0, rzt = 0;
        for (const Radius& r : pb.reach) {
            rxt = std::max(rxt, r.x);
            ryt = std::max(ryt, r.y);
            rzt = std::max(rzt, r.z);
        }
        f << "    static constexpr int RXT = " << rxt << ", RYT = " << ryt << ", RZT = " << rzt << ";\n";
        f << "    static __device__ __forceinline__ constexpr bool checked(int j) { ";
        for (int j = 0; j < nout; ++j) f << "if (j == " << j << ") return " << (checked[static_cast<std::size_t>(j)] ? "true" : "false") << "; ";
        f << "return false; }\n";
    }

    // Sizes a slab pass's tile and ring to the shared memory; false when no shape fits (the plain twin runs then).
    bool size_slab(PassBuild& pb, Launch& L)
    {
        int rz = 0;
        for (std::size_t k = 0; k < pb.sources.size(); ++k) {
            pb.sources[k].ax = (pb.reach[k].x + 3) / 4 * 4;
            pb.sources[k].ry = pb.reach[k].y;
            rz = std::max(rz, pb.reach[k].z);
        }
        L.rz = rz;
        // A slab tile is 128 cells wide: a lattice narrower than that would leave most of each tile's lanes idle and
        // stage a plane a CTA, so it takes the plain pass (a thread a cell, as many CTAs as the planes allow).
        if ((nx_ % 4) != 0 || nx_ < 128 || pb.sources.empty() || pb.sources.size() > FE_MAX_MAP_HOST) return false;
        for (const Source& s : pb.sources) {
            if (128 + 2 * s.ax > 256 || s.ry > 64) return false;
        }
        // The ring holds the 2 RZ + 1 planes a z reads and at least one being fetched. Measured on the 512^3 heat gather,
        // more CTAs an SM beat a deeper ring (16 rows: 4 stages 4.05 TB/s, 5 stages 3.98, 6 stages 3.69, 8 stages
        // 3.09; 8-row tiles 3.2 whatever the ring), so the shallowest ring of at least 4 stages comes first, 16-row
        // tiles before 8, under budgets that leave room for 3, then 2, then 1 CTA an SM. A pass that reads no other
        // plane (RZ = 0) starts at 2 stages: the explicit Heston gather (7 sources, 512 x 256) takes 0.39 ms a substep
        // on 128 planes with 2 stages against 0.65 with 4, which leave room for one CTA an SM only. With the plane carry
        // the ring holds planes z and z + 1, and its 4 stages keep two planes in flight: the 512^3 heat gather (32-row
        // tiles, 80 registers: 3 CTAs an SM whatever the ring) 5.24 TB/s with 4 stages, 5.08 with 3; the 43-term law at
        // 512^3 16.8 ms a step against 17.1. Forced to 64 registers for a fourth CTA an SM (3 stages) it spills: slower.
        // A carried pass that fits no budget with 4 stages tries 3.
        auto fit = [&](int shallowest) {
            // First, 32-row tiles when they leave room for 3 CTAs an SM (a warp then computes 4 rows of a plane, so the
            // per-plane waits, barrier and ring bookkeeping are shared by 16 cells a lane): the 512^3 heat gather,
            // 16-row tiles 4.15 TB/s (5 CTAs an SM), 24 rows 4.10, 32 rows 4.41 (3 CTAs), 32 rows with 5 stages 4.02,
            // 40 rows 3.34 (before the plane carry).
            {
                std::size_t floats = 0;
                for (const Source& s : pb.sources) floats += static_cast<std::size_t>(((128 + 2 * s.ax) * (32 + 2 * s.ry) + 31) / 32 * 32) * shallowest;
                if (floats * 4 <= 75u * 1024 && 32 + 2 * rz < 256) {
                    L.ty = 32;
                    L.nst = shallowest;
                    L.smem = static_cast<unsigned>(floats * 4);
                    return true;
                }
            }
            for (const std::size_t budget : {72u * 1024, 110u * 1024, 200u * 1024}) {
                for (const int ty : {16, 8}) {
                    for (int nst = shallowest; nst <= shallowest + 2; ++nst) {
                        std::size_t floats = 0;
                        for (const Source& s : pb.sources) {
                            const int plane = ((128 + 2 * s.ax) * (ty + 2 * s.ry) + 31) / 32 * 32;
                            floats += static_cast<std::size_t>(plane) * nst;
                        }
                        if (floats * 4 <= budget && ty + 2 * rz < 256) {
                            L.ty = ty;
                            L.nst = nst;
                            L.smem = static_cast<unsigned>(floats * 4);
                            return true;
                        }
                    }
                }
            }
            return false;
        };
        if (rz == 0) return fit(2);
        if (pb.zcarry) return fit(rz + 3) || fit(rz + 2);
        return fit(std::max(4, 2 * rz + 2));
    }

    // How far along x a value reads, everything it inlines included (a stage read by it is one load: 0).
    int xreach(int id, bool body, std::map<std::pair<int, bool>, int>& memo)
    {
        const auto key = std::make_pair(id, body);
        const auto found = memo.find(key);
        if (found != memo.end()) return found->second;
        const Inst& in = at(id);
        int r = 0;
        if ((body || !(m_.is_stage(id) || in.global)) && in.op != Op::Field) {
            const int own = axis_radius(in).x;
            for (const int a : in.args) r = std::max(r, own + xreach(a, false, memo));
        }
        memo.emplace(key, r);
        return r;
    }

    // Whether the lattice's x edge can be met by filling the staged x halo with the edge cell (what a clamped read
    // returns) and reading without clamps: true when every op that reads along x gives the same arithmetic either way
    // (shift, lap, diffuse, adv: a face past the edge reads the cell itself, a difference of +-0) and reads only values
    // with no x reach of their own (a nested x stencil evaluated past the edge would not be the clamped one).
    bool xfill_safe(const std::vector<int>& roots, bool bodies)
    {
        std::map<std::pair<int, bool>, int> memo;
        std::set<std::pair<int, bool>> seen;
        bool safe = true;
        std::function<void(int, bool)> visit = [&](int id, bool body) {
            if (!safe || !seen.insert({id, body}).second) return;
            const Inst& in = at(id);
            if (!body && (m_.is_stage(id) || in.global)) return;
            if (axis_radius(in).x > 0) {
                const bool kind_ok = in.op == Op::Shift || in.op == Op::Lap || in.op == Op::Diffuse || in.op == Op::Adv;
                if (!kind_ok) safe = false;
                for (const int a : in.args) {
                    if (xreach(a, false, memo) != 0) safe = false;
                }
            }
            for (const int a : in.args) visit(a, false);
        };
        for (const int r : roots) visit(r, bodies);
        return safe;
    }

    static constexpr std::size_t FE_MAX_SRC_HOST = 32;   // FE_MAX_SRC
    static constexpr std::size_t FE_MAX_MAP_HOST = 12;   // FE_MAX_MAP: a slab pass stages at most this many sources
    static constexpr std::size_t FE_MAX_OUT_HOST = 8;

    // A pass: computes `outs` (stage bodies, or the gather's targets) at every cell.
    struct PassOut {
        enum Kind { StageBody, Gather, Derive } kind = StageBody;
        int stage = -1;            // StageBody
        int target = -1;           // Gather / Derive: the field
        std::vector<int> values;   // Gather: the rates of the equations on the target, in order
        bool accumulate = false;   // Derive
        Buf dest;
    };

    bool emit_pass(const std::string& tag, std::vector<PassOut> outs, Launch& L, std::string& why)
    {
        PassBuild pb;
        std::vector<int> roots;
        for (const PassOut& o : outs) {
            if (o.kind == PassOut::StageBody) {
                pb.own_stages.insert(o.stage);
                roots.push_back(o.stage);
            } else {
                roots.insert(roots.end(), o.values.begin(), o.values.end());
                // The target's current value at its own cell.
                source_index(pb, Buf{Buf::FieldNow, o.target});
            }
        }
        const bool bodies = outs.front().kind == PassOut::StageBody;
        for (const int r : roots) walk(pb, r, Radius{}, bodies);
        for (const int r : roots) walk_points(pb, r, 0, 0, 0, bodies);
        plan_carry(pb);
        std::ostringstream f;
        const std::string ns = "fe_" + tag;
        f << "namespace " << ns << " {\n";
        emit_functions(f, pb, roots, bodies);
        if (pb.sources.size() > FE_MAX_SRC_HOST || outs.size() > FE_MAX_OUT_HOST) {
            why = "a pass of '" + tag + "' reads " + std::to_string(pb.sources.size()) + " buffers and writes " + std::to_string(outs.size()) +
                " (at most 32 and 8)";
            return false;
        }
        L.kind = Launch::Pass;
        L.sources = pb.sources;
        L.slab = size_slab(pb, L);
        L.sources = pb.sources;
        std::vector<char> checked;
        for (const PassOut& o : outs) {
            L.outs.push_back(o.dest);
            const bool c = o.kind != PassOut::StageBody;
            checked.push_back(c ? 1 : 0);
            L.checked_fields.push_back(c ? o.target : -1);
        }
        if (!L.slab) {
            L.ty = 16;
            L.nst = 4;
            pb.zcarry = false;
        }
        emit_traits(f, pb, L, static_cast<int>(outs.size()), checked);
        f << "    static constexpr bool XFILL = " << (xfill_safe(roots, bodies) ? "true" : "false") << ";\n";
        // The cell: every output's value, and the value it replaces (for the contracts).
        f << "    template <bool IN, class C> static __device__ __forceinline__ void cell(const C& c, int x, int y, int z, float* o, float* b) {\n";
        for (std::size_t j = 0; j < outs.size(); ++j) {
            const PassOut& o = outs[j];
            if (o.kind == PassOut::StageBody) {
                f << "        o[" << j << "] = b" << o.stage << "<IN>(c, x, y, z); b[" << j << "] = 0.f;\n";
                continue;
            }
            const int k = source_index(pb, Buf{Buf::FieldNow, o.target});
            if (o.kind == PassOut::Derive) {
                f << "        { const float v = " << v(o.values[0]) << "; const float old = c.template ld<" << k << ">(x, y, z); b[" << j
                  << "] = old; o[" << j << "] = " << (o.accumulate ? "old" : "0.f") << " + v; }\n";
                continue;
            }
            f << "        { float n = c.template ld<" << k << ">(x, y, z); b[" << j << "] = n; float d;\n";
            for (const int val : o.values) {
                f << "          d = " << v(val) << " * c.dt; if (d != 0.f) n += d;\n";
            }
            f << "          o[" << j << "] = n; }\n";
        }
        f << "    }\n};\n}\n";
        L.kernel = "fe_pass_" + tag;
        L.plain_kernel = "fe_pass_" + tag + "_plain";
        if (L.slab) {
            f << "extern \"C\" __global__ void __launch_bounds__(256) " << L.kernel << "(const __grid_constant__ FePassArgs a) { fe_slab_pass<"
              << ns << "::P>(a); }\n";
        }
        f << "extern \"C\" __global__ void __launch_bounds__(256) " << L.plain_kernel << "(const __grid_constant__ FePassArgs a) { fe_plain_pass<"
          << ns << "::P>(a); }\n";
        // A pass with contracts also comes in a variant for a slab of a split lattice (halo planes left out of them).
        if (std::any_of(L.checked_fields.begin(), L.checked_fields.end(), [](int f) { return f >= 0; })) {
            if (L.slab) {
                f << "extern \"C\" __global__ void __launch_bounds__(256) " << L.kernel << "_halo(const __grid_constant__ FePassArgs a) { fe_slab_pass<"
                  << ns << "::P, true>(a); }\n";
            }
            f << "extern \"C\" __global__ void __launch_bounds__(256) " << L.plain_kernel << "_halo(const __grid_constant__ FePassArgs a) { fe_plain_pass<"
              << ns << "::P, true>(a); }\n";
        }
        out_ << f.str();
        return true;
    }

    bool emit_tridiag(const std::string& tag, int id, Launch& L, std::string& why)
    {
        const Inst& in = at(id);
        PassBuild pb;
        for (const int a : in.args) walk(pb, a, Radius{}, false);
        for (const Radius& r : pb.reach) {
            if (r.x || r.y || r.z) {
                why = "a tridiag's coefficients must be read at its own cell";
                return false;
            }
        }
        std::ostringstream f;
        const std::string ns = "fe_" + tag;
        f << "namespace " << ns << " {\n";
        std::vector<int> roots(in.args.begin(), in.args.end());
        emit_functions(f, pb, roots, false);
        const int axis = in.index % 3;
        const bool transposed = in.index >= 3;
        L.kind = axis == 0 ? Launch::TridiagX : Launch::TridiagYZ;
        L.axis = axis;
        L.sources = pb.sources;
        L.slab = false;
        L.ty = 16;
        L.nst = 4;
        const int slot = plan_.slot_of[static_cast<std::size_t>(id)];
        L.outs = {Buf{Buf::Slot, slot}, Buf{Buf::Slot, slot + 1}};
        L.checked_fields = {-1, -1};
        emit_traits(f, pb, L, 2, {0, 0});
        f << "    template <class C> static __device__ __forceinline__ void coef(const C& c, int x, int y, int z, float& lo, float& di, float& up, float& rhs) {\n"
          << "        constexpr bool IN = false;\n";
        if (!transposed) {
            f << "        lo = " << v(in.args[0]) << "; up = " << v(in.args[2]) << "; di = " << v(in.args[1]) << "; rhs = " << v(in.args[3]) << ";\n    }\n";
        } else {
            // The transpose of the edge-repeating matrix: below the diagonal the previous cell's `up`, above it the next
            // cell's `lo`, the folded edge terms on the diagonal (so the pass's own folding adds zeros).
            const char* q = axis == 0 ? "x" : (axis == 1 ? "y" : "z");
            const char* n = axis == 0 ? "NX" : (axis == 1 ? "NY" : "NZ");
            auto at = [&](int arg, int d) {
                const std::string s = std::string(q) + (d < 0 ? " - 1" : " + 1");
                return axis == 0 ? v(in.args[arg], s) : (axis == 1 ? v(in.args[arg], "x", s) : v(in.args[arg], "x", "y", s));
            };
            f << "        const float l0 = " << v(in.args[0]) << ", u0 = " << v(in.args[2]) << ";\n"
              << "        lo = " << q << " > 0 ? " << at(2, -1) << " : 0.f;\n"
              << "        up = " << q << " + 1 < P::" << n << " ? " << at(0, +1) << " : 0.f;\n"
              << "        di = " << v(in.args[1]) << ";\n"
              << "        if (" << q << " == 0) di += l0;\n"
              << "        if (" << q << " + 1 == P::" << n << ") di += u0;\n"
              << "        rhs = " << v(in.args[3]) << ";\n    }\n";
        }
        f << "    template <bool IN, class C> static __device__ __forceinline__ void cell(const C&, int, int, int, float*, float*) {}\n";
        f << "};\n}\n";
        L.kernel = "fe_tri_" + tag;
        if (axis == 0) {
            const int m = (nx_ + 31) / 32;
            if (m >= 2 && m <= kTriLaneRows) {
                // A warp a line, M rows a lane (the partition method): lines of 33 .. 32 kTriLaneRows cells.
                L.tri_rows = m;
                L.smem = static_cast<unsigned>(kTriWarps * 4 * (33 * m) * 4);
                f << "extern \"C\" __global__ void __launch_bounds__(" << 32 * kTriWarps << ") " << L.kernel
                  << "(const __grid_constant__ FePassArgs a) { fe_tridiag_x_warp<" << ns << "::P, " << m << ", " << kTriWarps << ">(a); }\n";
            } else {
                if (nx_ > 640) {
                    why = "tridiag_x keeps a line in shared memory: nx up to 640";
                    return false;
                }
                L.tri_rows = 0;
                L.smem = static_cast<unsigned>(2 * nx_ * 33 * 4);
                f << "extern \"C\" __global__ void __launch_bounds__(32) " << L.kernel << "(const __grid_constant__ FePassArgs a) { fe_tridiag_x_pass<" << ns
                  << "::P>(a); }\n";
            }
        } else {
            const int n = axis == 1 ? ny_ : nz_;
            const int other = axis == 1 ? nz_ : ny_;
            // Segments of M rows, K of them a line (at most 16: a block of 32 K threads holds 32 lines and keeps 4 M
            // floats a thread in registers, so 512 threads at most).
            const int m = n >= 128 ? 16 : 8;
            const int k = (n + m - 1) / m;
            if (n >= 2 * m && k <= 16 && other <= 65535) {
                L.tri_rows = m;
                L.tri_segs = k;
                f << "extern \"C\" __global__ void __launch_bounds__(" << 32 * k << ") " << L.kernel
                  << "(const __grid_constant__ FePassArgs a) { fe_tridiag_yz_seg<" << ns << "::P, " << axis << ", " << m << ", " << k << ">(a); }\n";
            } else {
                L.tri_rows = 0;
                f << "extern \"C\" __global__ void __launch_bounds__(128) " << L.kernel << "(const __grid_constant__ FePassArgs a) { fe_tridiag_yz_pass<"
                  << ns << "::P, " << axis << ">(a); }\n";
            }
        }
        out_ << f.str();
        return true;
    }

    // A distance or poisson op: the seed pass (its argument at every cell, clamped reads) against what was last
    // solved; the engine runs the fixed solve kernels after it.
    void emit_solve(const std::string& tag, int id, Launch& L)
    {
        const Inst& in = at(id);
        PassBuild pb;
        walk(pb, in.args[0], Radius{}, false);
        std::ostringstream f;
        const std::string ns = "fe_" + tag;
        f << "namespace " << ns << " {\n";
        emit_functions(f, pb, {in.args[0]}, false);
        L.kind = in.op == Op::Distance ? Launch::Distance : Launch::Poisson;
        L.sources = pb.sources;
        L.slab = false;
        const int slot = plan_.slot_of[static_cast<std::size_t>(id)];
        L.aux = plan_.aux_of[static_cast<std::size_t>(id)];
        L.flag = flag_of_.at(id);
        L.iterations = in.iterations;
        L.outs = {Buf{Buf::Slot, slot}};
        L.checked_fields = {-1};
        emit_traits(f, pb, L, 0, {});
        f << "    template <class C> static __device__ __forceinline__ float value(const C& c, int x, int y, int z) { constexpr bool IN = false; return "
          << v(in.args[0]) << "; }\n"
          << "    template <bool IN, class C> static __device__ __forceinline__ void cell(const C&, int, int, int, float*, float*) {}\n"
          << "};\n}\n";
        L.kernel = "fe_seed_" + tag;
        f << "extern \"C\" __global__ void __launch_bounds__(256) " << L.kernel << "(const __grid_constant__ FePassArgs a) { fe_seed_pass<" << ns
          << "::P, " << (in.op == Op::Distance ? 1 : 0) << ">(a); }\n";
        out_ << f.str();
    }

    bool emit_reduce(const std::string& tag, int id, Launch& L)
    {
        const Inst& in = at(id);
        PassBuild pb;
        walk(pb, in.args[0], Radius{}, false);
        std::ostringstream f;
        const std::string ns = "fe_" + tag;
        f << "namespace " << ns << " {\n";
        emit_functions(f, pb, {in.args[0]}, false);
        L.kind = Launch::Reduce;
        L.sources = pb.sources;
        L.slab = false;
        L.uniform = plan_.uniform_of[static_cast<std::size_t>(id)];
        emit_traits(f, pb, L, 0, {});
        f << "    static constexpr int KIND = " << (in.op == Op::SumOf ? 0 : (in.op == Op::MaxOf ? 1 : 2)) << ";\n"
          << "    template <class C> static __device__ __forceinline__ float value(const C& c, int x, int y, int z) { constexpr bool IN = false; return "
          << v(in.args[0]) << "; }\n"
          << "    template <bool IN, class C> static __device__ __forceinline__ void cell(const C&, int, int, int, float*, float*) {}\n"
          << "};\n}\n";
        L.kernel = "fe_red_" + tag;
        f << "extern \"C\" __global__ void __launch_bounds__(256) " << L.kernel << "(const __grid_constant__ FePassArgs a) { fe_reduce_pass<" << ns
          << "::P>(a, &FE_U[" << L.uniform << "]); }\n";
        out_ << f.str();
        return true;
    }

    static int pad16(int v) { return (v + 15) / 16 * 16; }

    // BF16, round to nearest even (NaN kept a NaN).
    static unsigned short to_bf16(float v)
    {
        std::uint32_t u = 0;
        std::memcpy(&u, &v, sizeof(u));
        if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu) != 0u) return static_cast<unsigned short>((u >> 16) | 0x40u);
        u += 0x7FFFu + ((u >> 16) & 1u);
        return static_cast<unsigned short>(u >> 16);
    }

    // A `half` net's weights into FE_NETB: per layer the K x N matrix (K = inputs, N = outputs, each padded to 16 with
    // zeros) in BF16, in the no-swizzle core-matrix layout with K rows, element (k, n) = W[n][k]; returns the net's byte
    // offset (every layer starts on a 512-byte boundary). A net without `half` packs nothing.
    std::size_t pack_half(const law::NetDecl& net)
    {
        const std::size_t start = plan_.net_bf16.size() * 2;
        if (!net.half) return start;
        for (int l = 0; l < net.layers(); ++l) {
            const int ni = net.sizes[static_cast<std::size_t>(l)];
            const int no = net.sizes[static_cast<std::size_t>(l) + 1];
            const int K = pad16(ni), N = pad16(no);
            const std::size_t base = plan_.net_bf16.size();
            plan_.net_bf16.resize(base + static_cast<std::size_t>(K) * N, 0);
            const std::size_t off = net.weight_offset(l);
            for (int k = 0; k < ni; ++k) {
                for (int n = 0; n < no; ++n) {
                    const unsigned byte = static_cast<unsigned>(((n >> 3) * (K >> 3) + (k >> 3)) * 128 + (k & 7) * 16 + (n & 7) * 2);
                    plan_.net_bf16[base + byte / 2] = to_bf16(net.weights[off + static_cast<std::size_t>(n) * ni + static_cast<std::size_t>(k)]);
                }
            }
        }
        return start;
    }

    // A net op whose net is declared `half` (the reference's tensor-core nets): one stage kernel on tcgen05
    // (fe_device.cuh's fe_net_pass) that stores the op's value at every cell in the stage's slot. The P traits give the
    // net's padded shapes, its parameters' places, the inputs of each of a cell's evaluations (mlp: its arguments at
    // the cell; flux: the moved field and its companions on both sides of each of the six faces, both ways round;
    // ldiffuse: each face's normalised window of four cells and k's face value times dt / h^2, both ways round) and the
    // op's own FP32 arithmetic around the net (Law.cpp:1298-1438; CudaCodegen.cpp:718-840).
    bool emit_net(const std::string& tag, int id, Launch& L, std::string& why)
    {
        const Inst& in = at(id);
        const law::NetDecl& net = law_.nets[static_cast<std::size_t>(in.index)];
        const NetAt& na = net_at_[static_cast<std::size_t>(in.index)];
        const int layers = net.layers();
        std::vector<int> kp, np, no, wb;
        int wbytes = 0, nmax = 16, kmax = 16;
        for (int l = 0; l < layers; ++l) {
            const int ni = net.sizes[static_cast<std::size_t>(l)];
            const int o = net.sizes[static_cast<std::size_t>(l) + 1];
            if (o > 256 || ni > 256) {
                why = "net '" + net.name + "' is declared half, and the tensor-core form takes layers at most 256 wide";
                return false;
            }
            kp.push_back(pad16(ni));
            np.push_back(pad16(o));
            no.push_back(o);
            wb.push_back(wbytes);
            wbytes += pad16(ni) * pad16(o) * 2;
            nmax = std::max(nmax, pad16(o));
            kmax = std::max(kmax, pad16(ni));
        }
        int e = 1, nin = static_cast<int>(in.args.size());
        const std::size_t m = in.op == Op::Flux ? in.args.size() - 2 : 0;
        if (in.op == Op::Flux) {
            e = 12;
            nin = 2 * static_cast<int>(m);
        } else if (in.op == Op::LDiffuse) {
            e = 12;
            nin = 5;
        }
        const int nout = net.sizes.back();
        if (nin != net.sizes.front() || (in.op == Op::LDiffuse && nout != 4)) {
            why = "net '" + net.name + "' does not fit its op";
            return false;
        }
        // Evaluations a chunk: whole faces (pairs), as many as 64 accumulator columns hold (at least one face), so that
        // eight CTAs an SM find tensor memory when the net is at most 32 wide.
        const int pair = e == 1 ? 1 : 2;
        int ec = e == 1 ? 1 : std::max(2, (64 / nmax) / 2 * 2);
        while (e % ec != 0) ec -= pair;
        int tcols = 32;
        while (tcols < ec * nmax) tcols *= 2;
        const int per_sm = std::min(8, 512 / tcols);
        const unsigned a_bytes = static_cast<unsigned>(128 * kmax * 2);
        const unsigned need = static_cast<unsigned>(ec) * a_bytes + static_cast<unsigned>(wbytes) + 16;
        // Enough shared memory that no more than per_sm CTAs fit on an SM (228 KB, 1 KB reserved a CTA): each holds
        // tcols tensor-memory columns, and an SM has 512.
        const unsigned cap = static_cast<unsigned>(233472 / (per_sm + 1) - 1024 + 128) / 128 * 128;
        const unsigned smem = std::max(need, cap);
        if (smem > 227u * 1024u) {
            why = "net '" + net.name + "' is declared half, and its tensor-core tiles need more shared memory than a CTA has";
            return false;
        }

        PassBuild pb;
        const Radius r = axis_radius(in);
        for (const int arg : in.args) walk(pb, arg, r, false);
        std::ostringstream f;
        const std::string ns = "fe_" + tag;
        f << "namespace " << ns << " {\n";
        std::vector<int> roots(in.args.begin(), in.args.end());
        emit_functions(f, pb, roots, false);
        auto arg = [&](std::size_t k, const std::string& x, const std::string& y, const std::string& z) {
            return "v" + std::to_string(in.args[k]) + "<false>(c, " + x + ", " + y + ", " + z + ")";
        };
        auto fn = [&](const char* type, const char* name, const std::vector<int>& v) {
            f << "    static __device__ __forceinline__ constexpr " << type << " " << name << "(int l) { ";
            for (std::size_t k = 0; k < v.size(); ++k) f << "if (l == " << k << ") return " << v[k] << "; ";
            f << "return 0; }\n";
        };
        auto table = [&](const std::vector<float>& v, std::size_t size) {
            std::string t = "{";
            for (std::size_t k = 0; k < size; ++k) t += (k ? ", " : "") + literal(k < v.size() ? v[k] : 0.0f);
            return t + "}";
        };
        // The face f (0..5: -x, +x, -y, +y, -z, +z) of a cell: its lower cell i and upper cell j (clamped: a face past
        // the lattice's edge is never used), and whether it is open.
        f << "__device__ __forceinline__ void face_cells(int f, int x, int y, int z, int& ix, int& iy, int& iz, int& jx, int& jy, int& jz) {\n"
          << "    const int ax = f >> 1; ix = x; iy = y; iz = z;\n"
          << "    if ((f & 1) == 0) { ix = fe_ex(x - (ax == 0)); iy = fe_ey(y - (ax == 1)); iz = fe_ez(z - (ax == 2)); }\n"
          << "    jx = fe_ex(ix + (ax == 0)); jy = fe_ey(iy + (ax == 1)); jz = fe_ez(iz + (ax == 2)); }\n"
          << "__device__ __forceinline__ unsigned faces_open(int x, int y, int z) {\n"
          << "    return (x > 0 ? 1u : 0u) | (x + 1 < NX ? 2u : 0u) | (y > 0 ? 4u : 0u) | (y + 1 < NY ? 8u : 0u) | (z > 0 ? 16u : 0u) | (z + 1 < NZ ? 32u : 0u); }\n";
        if (in.op == Op::LDiffuse) {
            // The window F[i-1] F[i] | F[j] F[j+1] of the face between i = (x, y, z) and its +AX neighbour j (edge
            // cells repeat), and k's face value (the harmonic mean, in double): the fp32 form's arithmetic.
            f << "template <int AX, class C> __device__ __forceinline__ void window(const C& c, int x, int y, int z, float* w, float& kf) {\n"
              << "    const int jx = fe_ex(x + (AX == 0)), jy = fe_ey(y + (AX == 1)), jz = fe_ez(z + (AX == 2));\n"
              << "    const int q = AX == 0 ? x : (AX == 1 ? y : z); const int count = AX == 0 ? NX : (AX == 1 ? NY : NZ);\n"
              << "    const int mx = q > 0 ? x - (AX == 0) : x, my = q > 0 ? y - (AX == 1) : y, mz = q > 0 ? z - (AX == 2) : z;\n"
              << "    const int px = q + 2 < count ? jx + (AX == 0) : jx, py = q + 2 < count ? jy + (AX == 1) : jy, pz = q + 2 < count ? jz + (AX == 2) : jz;\n"
              << "    w[0] = " << arg(1, "mx", "my", "mz") << "; w[1] = " << arg(1, "x", "y", "z") << "; w[2] = " << arg(1, "jx", "jy", "jz")
              << "; w[3] = " << arg(1, "px", "py", "pz") << ";\n"
              << "    const double ka = " << arg(0, "x", "y", "z") << ", kb = " << arg(0, "jx", "jy", "jz") << ";\n"
              << "    kf = static_cast<float>((ka + kb) > 0.0 ? 2.0 * ka * kb / (ka + kb) : 0.0); }\n"
              << "__device__ __forceinline__ float after_net(const float* yw, const float* w, float kf) {\n"
              << "    const float mean = 0.25f * (yw[0] + yw[1] + yw[2] + yw[3]);\n"
              << "    const float base[4] = {0.f, -1.f, 1.f, 0.f}; float acc = 0.f;\n"
              << "#pragma unroll\n    for (int q = 0; q < 4; ++q) acc += (base[q] + (yw[q] - mean)) * w[q];\n"
              << "    return -kf / FE_H * acc; }\n";
        }
        f << "struct P {\n"
          << "    static constexpr int NX = ::NX, NY = ::NY, NZ = ::NZ;\n"
          << "    static constexpr int E = " << e << ", EC = " << ec << ", PAIR = " << pair << ", NIN = " << nin << ", NOUT = " << nout
          << ", L = " << layers << ", NMAX = " << nmax << ", KP0 = " << kp[0] << ";\n"
          << "    static constexpr unsigned TCOLS = " << tcols << "u, A_BYTES = " << a_bytes << "u, W_BYTES = " << wbytes << "u, WOFF = " << na.bf16_bytes
          << "u;\n"
          << "    static constexpr bool ROLL = " << (e * layers > 24 ? "true" : "false") << ";\n"
          << "    static constexpr float OSCALE = " << literal(net.out_scale) << ";\n";
        fn("int", "kp", kp);
        fn("int", "np", np);
        fn("int", "no", no);
        fn("unsigned", "wb", wb);
        // The net's FP32 parameters as literals (fixed when the law is created): the inputs' shift and scale, the biases.
        f << "    static __device__ __forceinline__ float shift(int i) { constexpr float v[] = " << table(net.in_shift, static_cast<std::size_t>(kp[0]))
          << "; return v[i]; }\n"
          << "    static __device__ __forceinline__ float scale(int i) { constexpr float v[] = " << table(net.in_scale, static_cast<std::size_t>(kp[0]))
          << "; return v[i]; }\n"
          << "    static __device__ __forceinline__ float bias(int l, int o) {\n";
        for (int l = 0; l < layers; ++l) {
            const std::size_t off = net.weight_offset(l) + static_cast<std::size_t>(net.sizes[static_cast<std::size_t>(l)]) * no[static_cast<std::size_t>(l)];
            std::vector<float> b(net.weights.begin() + static_cast<std::ptrdiff_t>(off),
                net.weights.begin() + static_cast<std::ptrdiff_t>(off) + no[static_cast<std::size_t>(l)]);
            f << "        if (l == " << l << ") { constexpr float v[] = " << table(b, static_cast<std::size_t>(np[static_cast<std::size_t>(l)])) << "; return v[o]; }\n";
        }
        f << "        return 0.f; }\n";
        const std::string act = net.act == "tanh" ? "fe_tanh_approx(v)" : net.act == "relu" ? "(v > 0.f ? v : 0.f)" : net.act == "silu" ? "fe_silu_approx(v)" : "v";
        f << "    static __device__ __forceinline__ float act(float v) { return " << act << "; }\n";
        if (in.op == Op::Mlp) {
            f << "    struct Keep { float x[" << nin << "]; };\n"
              << "    template <class C> static __device__ __forceinline__ void prepare(const C& c, int x, int y, int z, Keep& k) {\n";
            for (std::size_t q = 0; q < in.args.size(); ++q) f << "        k.x[" << q << "] = " << arg(q, "x", "y", "z") << ";\n";
            f << "    }\n"
              << "    static __device__ __forceinline__ void input(const Keep& k, int, float* xin) {\n"
              << "#pragma unroll\n        for (int i = 0; i < NIN; ++i) xin[i] = k.x[i]; }\n"
              << "    static __device__ __forceinline__ void take(const Keep&, int, const float* y0, const float*, float& o) { o = y0[0]; }\n"
              << "    static __device__ __forceinline__ float result(float o) { return o; }\n";
        } else if (in.op == Op::Flux) {
            char bounds[96];
            std::snprintf(bounds, sizeof(bounds), "%.17g, %.17g", at(in.args[m]).number, at(in.args[m + 1]).number);
            // The cell's own values and its six neighbours' (a closed face's neighbour is the cell itself).
            f << "    struct Keep { float cen[" << m << "]; float nb[6][" << m << "]; unsigned open; float dt; };\n"
              << "    template <class C> static __device__ __forceinline__ void prepare(const C& c, int x, int y, int z, Keep& k) {\n";
            for (std::size_t q = 0; q < m; ++q) f << "        k.cen[" << q << "] = " << arg(q, "x", "y", "z") << ";\n";
            f << "#pragma unroll\n        for (int f = 0; f < 6; ++f) {\n"
              << "            int ix, iy, iz, jx, jy, jz; face_cells(f, x, y, z, ix, iy, iz, jx, jy, jz);\n"
              << "            const int nx = (f & 1) ? jx : ix, ny = (f & 1) ? jy : iy, nz = (f & 1) ? jz : iz;\n";
            for (std::size_t q = 0; q < m; ++q) f << "            k.nb[f][" << q << "] = " << arg(q, "nx", "ny", "nz") << ";\n";
            f << "        }\n"
              << "        k.open = faces_open(x, y, z); k.dt = c.dt; }\n"
              // Way 0 sees (i, j), way 1 (j, i); i is the face's lower cell.
              << "    static __device__ __forceinline__ void input(const Keep& k, int e, float* xin) {\n"
              << "        const int f = e >> 1; const bool up = (f & 1) != 0; const bool way = (e & 1) != 0;\n"
              << "        const float* i = up ? k.cen : k.nb[f]; const float* j = up ? k.nb[f] : k.cen;\n"
              << "#pragma unroll\n        for (int q = 0; q < " << m << "; ++q) { xin[q] = way ? j[q] : i[q]; xin[" << m << " + q] = way ? i[q] : j[q]; } }\n"
              << "    static __device__ __forceinline__ void take(const Keep& k, int e, const float* y0, const float* y1, float& o) {\n"
              << "        const int f = e >> 1; const bool up = (f & 1) != 0;\n"
              << "        if (((k.open >> f) & 1u) == 0u) return;\n"
              << "        const float fi = up ? k.cen[0] : k.nb[f][0], fj = up ? k.nb[f][0] : k.cen[0];\n"
              << "        const float g = fe_limit_face(0.5f * (y0[0] - y1[0]), fi, fj, " << bounds << ", k.dt);\n"
              << "        if (up) o -= g; else o += g; }\n"
              << "    static __device__ __forceinline__ float result(float o) { return o / FE_H; }\n";
        } else {
            f << "    struct Keep { float w[6][4]; float kf[6]; unsigned open; float dt; };\n"
              << "    template <class C> static __device__ __forceinline__ void prepare(const C& c, int x, int y, int z, Keep& k) {\n"
              << "#pragma unroll\n        for (int f = 0; f < 6; ++f) {\n"
              << "            int ix, iy, iz, jx, jy, jz; face_cells(f, x, y, z, ix, iy, iz, jx, jy, jz);\n"
              << "            if ((f >> 1) == 0) window<0>(c, ix, iy, iz, k.w[f], k.kf[f]);\n"
              << "            else if ((f >> 1) == 1) window<1>(c, ix, iy, iz, k.w[f], k.kf[f]);\n"
              << "            else window<2>(c, ix, iy, iz, k.w[f], k.kf[f]);\n"
              << "        }\n"
              << "        k.open = faces_open(x, y, z); k.dt = c.dt; }\n"
              // Way 1 is the mirrored window: the same centre and spread, so its inputs are way 0's reversed.
              << "    static __device__ __forceinline__ void input(const Keep& k, int e, float* xin) {\n"
              << "        const int f = e >> 1; const float* w = k.w[f];\n"
              << "        const float centre = 0.5f * (w[1] + w[2]); float spread = 1e-6f;\n"
              << "#pragma unroll\n        for (int q = 0; q < 4; ++q) spread = fmaxf(spread, fabsf(w[q] - centre));\n"
              << "#pragma unroll\n        for (int q = 0; q < 4; ++q) xin[(e & 1) ? 3 - q : q] = (w[q] - centre) / spread;\n"
              << "        xin[4] = k.kf[f] * k.dt / (FE_H * FE_H); }\n"
              << "    static __device__ __forceinline__ void take(const Keep& k, int e, const float* y0, const float* y1, float& o) {\n"
              << "        const int f = e >> 1; const bool up = (f & 1) != 0;\n"
              << "        if (((k.open >> f) & 1u) == 0u) return;\n"
              << "        const float* w = k.w[f]; const float mirror[4] = {w[3], w[2], w[1], w[0]};\n"
              << "        const float g = 0.5f * (after_net(y0, w, k.kf[f]) - after_net(y1, mirror, k.kf[f]));\n"
              << "        if (up) o -= g; else o += g; }\n"
              << "    static __device__ __forceinline__ float result(float o) { return o / FE_H; }\n";
        }
        f << "};\n}\n";
        L.kind = Launch::Net;
        L.sources = pb.sources;
        L.slab = false;
        int rz = 0;
        for (const Radius& q : pb.reach) rz = std::max(rz, q.z);
        L.rz = rz;
        L.outs = {Buf{Buf::Slot, plan_.slot_of[static_cast<std::size_t>(id)]}};
        L.checked_fields = {-1};
        L.smem = smem;
        L.per_sm = per_sm;
        L.kernel = "fe_net_" + tag;
        f << "extern \"C\" __global__ void __launch_bounds__(128) " << L.kernel << "(const __grid_constant__ FePassArgs a) { fe_net_pass<" << ns
          << "::P>(a, FE_NETB); }\n";
        out_ << f.str();
        return true;
    }

    // Stages in order; consecutive stored stages that do not read one another share a pass.
    bool emit_stages(const std::string& tag, const std::vector<int>& stages, std::vector<Launch>& launches, std::string& why)
    {
        std::vector<int> group;
        int n = 0;
        auto flush = [&]() -> bool {
            if (group.empty()) return true;
            std::vector<PassOut> outs;
            for (const int s : group) {
                PassOut o;
                o.kind = PassOut::StageBody;
                o.stage = s;
                o.dest = Buf{Buf::Slot, plan_.slot_of[static_cast<std::size_t>(s)]};
                outs.push_back(o);
            }
            Launch L;
            if (!emit_pass(tag + "s" + std::to_string(n++), outs, L, why)) return false;
            launches.push_back(L);
            group.clear();
            return true;
        };
        for (const int s : stages) {
            const Inst& in = at(s);
            if (in.net && law_.nets[static_cast<std::size_t>(in.index)].half) {
                if (!flush()) return false;
                Launch L;
                if (!emit_net(tag + "n" + std::to_string(n++), s, L, why)) return false;
                launches.push_back(L);
                continue;
            }
            if (in.op == Op::Tridiag || in.global) {
                if (!flush()) return false;
                Launch L;
                if (in.op == Op::Tridiag) {
                    if (!emit_tridiag(tag + "x" + std::to_string(n++), s, L, why)) return false;
                } else if (in.op == Op::Distance || in.op == Op::Poisson) {
                    emit_solve(tag + "d" + std::to_string(n++), s, L);
                } else {
                    if (!emit_reduce(tag + "r" + std::to_string(n++), s, L)) return false;
                }
                launches.push_back(L);
                continue;
            }
            // Does s read (through what it inlines) a stage already in the group?
            PassBuild probe;
            probe.own_stages.insert(s);
            walk(probe, s, Radius{}, true);
            bool depends = false;
            for (const Source& src : probe.sources) {
                for (const int g : group) {
                    if (src.buf.kind == Buf::Slot && src.buf.id == plan_.slot_of[static_cast<std::size_t>(g)]) depends = true;
                }
            }
            if (depends || group.size() >= FE_MAX_OUT_HOST) {
                if (!flush()) return false;
            }
            group.push_back(s);
        }
        return flush();
    }

    bool program(const ir::Program& p, const std::string& tag, bool derive, ProgramPlan& pp, std::string& why)
    {
        pp.empty = p.equations.empty();
        if (pp.empty) return true;
        if (!emit_stages(tag, p.stages, pp.stages, why)) return false;
        if (!emit_stages(tag + "m", p.limit_stages, pp.limit, why)) return false;
        std::vector<PassOut> outs;
        if (derive) {
            const ir::Equation& eq = p.equations[0];
            const bool reads_itself = std::find(p.reads.begin(), p.reads.end(), eq.target) != p.reads.end();
            pp.in_place = !reads_itself;
            PassOut o;
            o.kind = PassOut::Derive;
            o.target = eq.target;
            o.values = {eq.value};
            o.accumulate = p.accumulate;
            if (pp.in_place) {
                o.dest = Buf{Buf::FieldNow, eq.target};
            } else {
                o.dest = Buf{Buf::FieldNext, eq.target};
                pp.swaps.push_back(eq.target);
                plan_.pingpong[static_cast<std::size_t>(eq.target)] = 1;
            }
            outs.push_back(o);
        } else {
            pp.in_place = p.in_place;
            std::vector<int> targets;
            for (const ir::Equation& eq : p.equations) {
                if (std::find(targets.begin(), targets.end(), eq.target) == targets.end()) targets.push_back(eq.target);
            }
            for (const int t : targets) {
                PassOut o;
                o.kind = PassOut::Gather;
                o.target = t;
                for (const ir::Equation& eq : p.equations) {
                    if (eq.target == t) o.values.push_back(eq.value);
                }
                if (pp.in_place) {
                    o.dest = Buf{Buf::FieldNow, t};
                } else {
                    o.dest = Buf{Buf::FieldNext, t};
                    pp.swaps.push_back(t);
                    plan_.pingpong[static_cast<std::size_t>(t)] = 1;
                }
                outs.push_back(o);
            }
        }
        return emit_pass(tag + "g", outs, pp.gather, why);
    }

    const ir::Module& m_;
    const law::Law& law_;
    int nx_, ny_, nz_;
    double h_;
    Plan& plan_;
    std::map<int, int> flag_of_; // distance / poisson inst -> its change flag
    // Per net: where its parameters sit in FE_NET (weights, input shift, input scale, output scale) and, for a `half`
    // net, its BF16 weights' byte offset in FE_NETB.
    struct NetAt {
        std::size_t w0, shift, scale, oscale, bf16_bytes;
    };
    std::vector<NetAt> net_at_;
    std::ostringstream out_;
};

} // namespace

bool generate(const ir::Module& m, const law::Law& law, int nx, int ny, int nz, double h, Plan& plan, std::string& why)
{
    plan = Plan{};
    // Wider staging pays once a pass has enough cells to hide its own cost: the FHN law (one RK4 stage read at five
    // points) goes 5.75 -> 3.02 ms a frame at 128 x 128 x 1000 and 0.49 -> 0.39 at 64 x 64 x 1000, bit-identical, but
    // 0.134 -> 0.142 at 32 x 32 x 1000, where the extra pass costs more than the recomputation it saves.
    ir::Module staged = m;
    if (static_cast<long long>(nx) * ny * nz >= (2LL << 20)) ir::widen_stages(staged);
    Generator g(staged, law, nx, ny, nz, h, plan);
    return g.run(why);
}

} // namespace fe::gen
