// Lowering a compiled law to the SSA module, and the module's JSON and text listings.
//
// Design. Everything the lowering needs to know about an operation sits in one table of traits (OpInfo): how its shape
// follows from its arguments, how far from its cell it reads, how many points of an argument one of its points reads,
// whether it is plain arithmetic on numbers, a whole-lattice op or a net, and which argument makes it vanish when that
// argument is one number everywhere. The algebraic shortcuts are rows of a rule table. The law's expression graph is
// walked with an explicit stack (no recursion, so deep laws cannot overflow), leaves first, each node once; values are
// hash-consed on a key of their own (InstKey). Because every instruction's arguments are created before it, ids are a
// topological order: the passes after lowering (stage costs, what a program reaches, how far it reads each field) are
// sweeps over the ids, forward or backward, instead of walks of the graph.
//
// The rules are the reference's, so a law gives the same instructions in the same order and the same programs
// (src/field/ir/LawIR.cpp:140-526: folding with the CPU's scalar semantics 162-250, shapes and radii 254-288, the
// stage cost model with the inline budget 314-338, stage sets, reads and the in-place decision 340-433) and the same
// JSON (LawIR.cpp:528-593); tests/test_ir_cpu.py holds every test law, the reference's benchmark laws and its world
// law to the reference's own lawc --ir-json output.
#include "ir.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <set>
#include <sstream>
#include <unordered_map>

namespace fe::ir {

namespace {

// ---- operation traits --------------------------------------------------------------------------------------------------

enum class ShapeRule : unsigned char { Scalar, Cell, FromArgs };
// What an op becomes when its `vanish_arg` is one number everywhere: zero (nothing varies, so no gradient, flux or
// spread), or that argument itself (a shift of a constant).
enum class Vanish : unsigned char { Never, ToZero, ToOperand };

using Eval = double (*)(const double*);

struct OpInfo {
    ShapeRule shape = ShapeRule::FromArgs;
    int radius = 0;          // cells from its own it reads; -1: the largest |offset| (shifts)
    int points = 1;          // points of each argument one point reads (the stage cost model's weight)
    bool global = false;     // needs the whole lattice before any cell (reductions, solves): always a stage
    bool net = false;        // a net evaluation: always a stage
    int vanish_arg = -1;
    Vanish vanish = Vanish::Never;
    Eval eval = nullptr;     // plain arithmetic: the value on numbers, in double, as the CPU's scalar path computes it
};

constexpr std::size_t kOps = static_cast<std::size_t>(Op::GzT) + 1;

const std::array<OpInfo, kOps>& op_table()
{
    static const std::array<OpInfo, kOps> table = [] {
        std::array<OpInfo, kOps> t{};
        auto at = [&t](Op op) -> OpInfo& { return t[static_cast<std::size_t>(op)]; };
        for (Op op : {Op::Const, Op::Param, Op::Cell, Op::Dt, Op::Local, Op::MaxOf, Op::MinOf, Op::SumOf}) at(op).shape = ShapeRule::Scalar;
        for (Op op : {Op::Field, Op::Rim, Op::Distance, Op::Poisson, Op::Fall, Op::Spread, Op::Topple, Op::Flux, Op::LDiffuse,
                      Op::Lap, Op::Gx, Op::Gy, Op::Gz, Op::Diffuse, Op::Adv, Op::Tridiag, Op::ShiftT, Op::GxT, Op::GyT, Op::GzT}) {
            at(op).shape = ShapeRule::Cell;
        }
        for (Op op : {Op::Lap, Op::Gx, Op::Gy, Op::Gz, Op::Diffuse, Op::Adv, Op::Fall, Op::Spread, Op::Topple, Op::Flux, Op::GxT,
                      Op::GyT, Op::GzT}) {
            at(op).radius = 1;
        }
        at(Op::LDiffuse).radius = 2;
        at(Op::Shift).radius = -1;
        at(Op::ShiftT).radius = -1;
        at(Op::Lap).points = at(Op::Diffuse).points = at(Op::Adv).points = 7;
        at(Op::Gx).points = at(Op::Gy).points = at(Op::Gz).points = 2;
        at(Op::Fall).points = 3;
        at(Op::Spread).points = 5;
        at(Op::Topple).points = 13;
        for (Op op : {Op::Distance, Op::Poisson, Op::MaxOf, Op::MinOf, Op::SumOf, Op::Tridiag}) at(op).global = true;
        for (Op op : {Op::Mlp, Op::Flux, Op::LDiffuse}) at(op).net = true;
        for (Op op : {Op::Lap, Op::Gx, Op::Gy, Op::Gz, Op::Adv, Op::Fall, Op::Spread, Op::Topple}) {
            at(op).vanish_arg = 0;
            at(op).vanish = Vanish::ToZero;
        }
        for (Op op : {Op::Diffuse, Op::LDiffuse}) {  // the conductivity may be a number; the field may not
            at(op).vanish_arg = 1;
            at(op).vanish = Vanish::ToZero;
        }
        at(Op::Shift).vanish_arg = 0;
        at(Op::Shift).vanish = Vanish::ToOperand;
        // The CPU's scalar semantics (src/field/Law.cpp:757-860): guarded division, clamped exp/log/sqrt.
        at(Op::Neg).eval = [](const double* a) { return -a[0]; };
        at(Op::Abs).eval = [](const double* a) { return std::fabs(a[0]); };
        // (std::min/std::max with these argument orders: a NaN argument passes through exp, log and pos, not sqrt.)
        at(Op::Sqrt).eval = [](const double* a) { return std::sqrt(std::max(0.0, a[0])); };
        at(Op::Exp).eval = [](const double* a) { return std::exp(std::min(a[0], 80.0)); };
        at(Op::Log).eval = [](const double* a) { return std::log(std::max(a[0], 1e-30)); };
        at(Op::Step).eval = [](const double* a) { return a[0] > 0.0 ? 1.0 : 0.0; };
        at(Op::Pos).eval = [](const double* a) { return std::max(a[0], 0.0); };
        at(Op::Add).eval = [](const double* a) { return a[0] + a[1]; };
        at(Op::Sub).eval = [](const double* a) { return a[0] - a[1]; };
        at(Op::Mul).eval = [](const double* a) { return a[0] * a[1]; };
        at(Op::Div).eval = [](const double* a) { return a[1] == 0.0 ? 0.0 : a[0] / a[1]; };
        at(Op::Pow).eval = [](const double* a) { return std::pow(a[0], a[1]); };
        at(Op::Min).eval = [](const double* a) { return std::min(a[0], a[1]); };
        at(Op::Max).eval = [](const double* a) { return std::max(a[0], a[1]); };
        at(Op::Clamp).eval = [](const double* a) { return std::clamp(a[0], a[1], std::max(a[1], a[2])); };
        return t;
    }();
    return table;
}

const OpInfo& info(Op op) { return op_table()[static_cast<std::size_t>(op)]; }

// ---- algebraic shortcuts ----------------------------------------------------------------------------------------------
// One row: when argument `arg` of `op` is the constant `value`, the instruction is zero, or another of its arguments.
// Rows of one op are tried in table order. (Zero times anything is zero on the CPU, which never looks at the anything.)

enum class Gives : unsigned char { Zero, Arg0, Arg1 };

struct Shortcut {
    Op op;
    int arg;
    double value;
    Gives gives;
};

constexpr Shortcut kShortcuts[] = {
    {Op::Mul, 0, 0.0, Gives::Zero}, {Op::Mul, 1, 0.0, Gives::Zero}, {Op::Mul, 0, 1.0, Gives::Arg1}, {Op::Mul, 1, 1.0, Gives::Arg0},
    {Op::Add, 0, 0.0, Gives::Arg1}, {Op::Add, 1, 0.0, Gives::Arg0},
    {Op::Sub, 1, 0.0, Gives::Arg0},
    {Op::Div, 1, 1.0, Gives::Arg0}, {Op::Div, 0, 0.0, Gives::Zero},
};

// ---- hash-consing --------------------------------------------------------------------------------------------------------

struct InstKey {
    Op op;
    std::uint64_t number_bits;
    int index, iterations;
    std::array<int, 3> offset;
    std::vector<int> args;

    bool operator==(const InstKey& o) const
    {
        return op == o.op && number_bits == o.number_bits && index == o.index && iterations == o.iterations && offset == o.offset &&
            args == o.args;
    }
};

struct InstKeyHash {
    std::size_t operator()(const InstKey& k) const
    {
        // FNV-1a over the fields, then the arguments.
        std::uint64_t h = 1469598103934665603ull;
        auto mix = [&h](std::uint64_t v) {
            for (int i = 0; i < 8; ++i) {
                h ^= (v >> (8 * i)) & 0xffu;
                h *= 1099511628211ull;
            }
        };
        mix(static_cast<std::uint64_t>(k.op));
        mix(k.number_bits);
        mix(static_cast<std::uint64_t>(static_cast<std::uint32_t>(k.index)) << 32 | static_cast<std::uint32_t>(k.iterations));
        for (const int o : k.offset) mix(static_cast<std::uint32_t>(o));
        for (const int a : k.args) mix(static_cast<std::uint32_t>(a));
        return static_cast<std::size_t>(h);
    }
};

std::uint64_t double_bits(double v)
{
    std::uint64_t b = 0;
    std::memcpy(&b, &v, sizeof(b));
    return b;
}

// ---- lowering ----------------------------------------------------------------------------------------------------------

class Builder {
public:
    Builder(Module& m, const law::Law& law) : m_(m), law_(law), done_(law.nodes.size(), -1) {}

    // The instruction of a law node: its argument nodes first, left to right (each fully before the next), then the
    // node itself; a node met again gives the instruction it gave the first time.
    int value_of(int root)
    {
        struct Frame {
            int node;
            bool expanded;
        };
        std::vector<Frame> stack{{root, false}};
        while (!stack.empty()) {
            const Frame f = stack.back();
            stack.pop_back();
            if (done_[static_cast<std::size_t>(f.node)] >= 0) continue;
            const law::Node& n = law_.nodes[static_cast<std::size_t>(f.node)];
            const std::size_t lowered = is_shift(n.op) ? 1 : n.args.size(); // a shift's offsets are numbers, not values
            if (!f.expanded) {
                stack.push_back({f.node, true});
                for (std::size_t i = lowered; i-- > 0;) stack.push_back({n.args[i], false});
                continue;
            }
            Inst in;
            in.op = n.op;
            in.number = n.number;
            in.index = n.index;
            in.iterations = n.iterations;
            for (std::size_t i = 0; i < lowered; ++i) in.args.push_back(done_[static_cast<std::size_t>(n.args[i])]);
            if (is_shift(n.op)) {
                for (int a = 0; a < 3; ++a) in.offset[a] = static_cast<int>(law_.nodes[static_cast<std::size_t>(n.args[1 + a])].number);
            }
            done_[static_cast<std::size_t>(f.node)] = reduce(std::move(in));
        }
        return done_[static_cast<std::size_t>(root)];
    }

private:
    static bool is_shift(Op op) { return op == Op::Shift || op == Op::ShiftT; }
    [[nodiscard]] const Inst& inst(int id) const { return m_.insts[static_cast<std::size_t>(id)]; }
    [[nodiscard]] bool holds(int id, double v) const { return inst(id).op == Op::Const && inst(id).number == v; }

    int number(double v)
    {
        Inst c;
        c.op = Op::Const;
        c.number = v;
        return intern(std::move(c));
    }

    // What the instruction simplifies to, or the instruction itself (interned).
    int reduce(Inst in)
    {
        const OpInfo& oi = info(in.op);
        auto folded = [&](int id) {
            ++m_.folded;
            return id;
        };
        if (oi.eval != nullptr) {
            std::array<double, 3> v{};
            bool numbers = true;
            for (std::size_t i = 0; i < in.args.size() && numbers; ++i) {
                numbers = inst(in.args[i]).op == Op::Const;
                if (numbers) v[i] = inst(in.args[i]).number;
            }
            if (numbers) {
                ++m_.folded;
                return number(oi.eval(v.data()));
            }
        }
        for (const Shortcut& s : kShortcuts) {
            if (s.op != in.op || !holds(in.args[static_cast<std::size_t>(s.arg)], s.value)) continue;
            switch (s.gives) {
            case Gives::Zero: ++m_.folded; return number(0.0);
            case Gives::Arg0: return folded(in.args[0]);
            case Gives::Arg1: return folded(in.args[1]);
            }
        }
        if (in.op == Op::Neg && inst(in.args[0]).op == Op::Neg) return folded(inst(in.args[0]).args[0]);
        if (oi.vanish != Vanish::Never) {
            const int a = in.args[static_cast<std::size_t>(oi.vanish_arg)];
            const bool still = in.op == Op::Shift && in.offset[0] == 0 && in.offset[1] == 0 && in.offset[2] == 0;
            if (inst(a).shape == Shape::Scalar || still) {
                if (oi.vanish == Vanish::ToOperand) return folded(a);
                ++m_.folded;
                return number(0.0);
            }
        }
        return intern(std::move(in));
    }

    // Fills in what follows from the op and the arguments, then finds the equal instruction or appends this one.
    int intern(Inst in)
    {
        const OpInfo& oi = info(in.op);
        switch (oi.shape) {
        case ShapeRule::Scalar: in.shape = Shape::Scalar; break;
        case ShapeRule::Cell: in.shape = Shape::Cell; break;
        case ShapeRule::FromArgs: {
            bool cell = false;
            for (const int a : in.args) cell = cell || inst(a).shape == Shape::Cell;
            in.shape = cell ? Shape::Cell : Shape::Scalar;
            break;
        }
        }
        in.radius = oi.radius >= 0 ? oi.radius : std::max({std::abs(in.offset[0]), std::abs(in.offset[1]), std::abs(in.offset[2])});
        in.global = oi.global;
        in.net = oi.net;
        InstKey key{in.op, double_bits(in.number), in.index, in.iterations, {in.offset[0], in.offset[1], in.offset[2]}, in.args};
        const int next = static_cast<int>(m_.insts.size());
        const auto [it, fresh] = interned_.try_emplace(std::move(key), next);
        if (!fresh) {
            ++m_.shared;
            return it->second;
        }
        m_.insts.push_back(std::move(in));
        return next;
    }

    Module& m_;
    const law::Law& law_;
    std::vector<int> done_;
    std::unordered_map<InstKey, int, InstKeyHash> interned_;
};

// ---- stages --------------------------------------------------------------------------------------------------------------

// The cost of one point of every instruction with everything that is not a stage inlined, and which values become
// stages: a stencil that would inline a per-cell argument at more than the budget's cost stores it instead, and a
// tridiagonal solve stores every per-cell argument that is not a field (its line walk only loads; the values are
// computed over the lattice first). One forward sweep: an argument's cost is final before its readers are priced.
void price_and_stage(Module& m)
{
    m.materialized.assign(m.insts.size(), 0);
    for (std::size_t id = 0; id < m.insts.size(); ++id) {
        Inst& reader = m.insts[id];
        const int weight = info(reader.op).points;
        long long cost = 1;
        for (const int a : reader.args) {
            Inst& arg = m.insts[static_cast<std::size_t>(a)];
            ++arg.uses;
            int inline_cost = m.is_stage(a) ? 1 : arg.cost;
            const bool storable = !m.is_stage(a) && arg.shape == Shape::Cell && arg.op != Op::Field;
            const bool too_dear = reader.radius > 0 && inline_cost * weight > kInlineBudget;
            if (storable && (reader.op == Op::Tridiag || too_dear)) {
                m.materialized[static_cast<std::size_t>(a)] = 1;
                inline_cost = 1;
            }
            cost += static_cast<long long>(inline_cost) * weight;
        }
        reader.cost = static_cast<int>(std::min<long long>(cost, 1 << 20));
    }
}

// Which instructions the roots depend on (arguments have lower ids than their readers: one backward sweep).
std::vector<char> reachable(const Module& m, const std::vector<int>& roots)
{
    std::vector<char> on(m.insts.size(), 0);
    int top = -1;
    for (const int r : roots) {
        if (r < 0) continue;
        on[static_cast<std::size_t>(r)] = 1;
        top = std::max(top, r);
    }
    for (int id = top; id >= 0; --id) {
        if (!on[static_cast<std::size_t>(id)]) continue;
        for (const int a : m.insts[static_cast<std::size_t>(id)].args) on[static_cast<std::size_t>(a)] = 1;
    }
    return on;
}

// The stages a set of roots needs before its kernel: per-cell stages and every whole-lattice op they depend on.
std::vector<int> stages_of(const Module& m, const std::vector<int>& roots)
{
    const std::vector<char> on = reachable(m, roots);
    std::vector<int> out;
    for (std::size_t id = 0; id < on.size(); ++id) {
        const Inst& in = m.insts[id];
        if (on[id] && ((m.is_stage(static_cast<int>(id)) && in.shape == Shape::Cell) || in.global)) out.push_back(static_cast<int>(id));
    }
    return out;
}

// How far from a cell the program's kernel reads each field: the largest sum of radii along a path from an equation's
// value to the field that runs through inlined instructions only (a stage, a net or a whole-lattice op is read at the
// cell, so the path ends there; an equation's own value is computed by the kernel even when it is a stage, unless it is
// a net or whole-lattice op). Backward sweep: an instruction's distance is final before its arguments are reached.
std::vector<int> field_reach(const Module& m, const Program& p, std::size_t fields)
{
    constexpr int kNone = -1;
    std::vector<int> dist(m.insts.size(), kNone);    // distance at which a non-root path arrives
    std::vector<char> root(m.insts.size(), 0);
    int top = -1;
    for (const Equation& eq : p.equations) {
        root[static_cast<std::size_t>(eq.value)] = 1;
        top = std::max(top, eq.value);
    }
    std::vector<int> out(fields, kNone);
    for (int id = top; id >= 0; --id) {
        const Inst& in = m.insts[static_cast<std::size_t>(id)];
        const bool is_root = root[static_cast<std::size_t>(id)] != 0;
        int d = kNone;
        if (is_root) d = m.is_stage(id) ? 0 : std::max(0, dist[static_cast<std::size_t>(id)]);
        else if (!m.is_stage(id)) d = dist[static_cast<std::size_t>(id)];
        if (in.op == Op::Field) {
            const int arrived = is_root ? std::max(0, dist[static_cast<std::size_t>(id)]) : dist[static_cast<std::size_t>(id)];
            if (arrived != kNone) out[static_cast<std::size_t>(in.index)] = std::max(out[static_cast<std::size_t>(in.index)], arrived);
            continue;
        }
        if (d == kNone || in.net || in.global) continue;
        for (const int a : in.args) dist[static_cast<std::size_t>(a)] = std::max(dist[static_cast<std::size_t>(a)], d + in.radius);
    }
    return out;
}

void finish(const Module& m, const law::Law& law, Program& p)
{
    std::vector<int> roots;
    for (const Equation& eq : p.equations) roots.push_back(eq.value);
    p.stages = stages_of(m, roots);
    p.limit_stages = p.max_dt >= 0 ? stages_of(m, {p.max_dt}) : std::vector<int>{};
    const std::vector<char> on = reachable(m, roots);
    std::set<int> reads;
    for (std::size_t id = 0; id < on.size(); ++id) {
        if (on[id] && m.insts[id].op == Op::Field) reads.insert(m.insts[id].index);
    }
    p.reads.assign(reads.begin(), reads.end());
    // A program whose kernel reads a field it writes at another cell must not overwrite it in place (ping-pong).
    const std::vector<int> reach = field_reach(m, p, law.fields.size());
    p.in_place = std::none_of(p.writes.begin(), p.writes.end(), [&](int f) { return reach[static_cast<std::size_t>(f)] > 0; });
}

Program start_program(Builder& b, std::string name, const std::vector<law::Equation>& equations, int max_dt)
{
    Program p;
    p.name = std::move(name);
    std::set<int> targets;
    for (const law::Equation& eq : equations) {
        p.equations.push_back(Equation{eq.target, b.value_of(eq.rhs)});
        targets.insert(eq.target);
    }
    if (max_dt >= 0) p.max_dt = b.value_of(max_dt);
    p.writes.assign(targets.begin(), targets.end());
    return p;
}

// ---- JSON ------------------------------------------------------------------------------------------------------------------

class Json {
public:
    Json& raw(const char* s)
    {
        out_ << s;
        return *this;
    }
    Json& num(double v)
    {
        if (!std::isfinite(v)) return raw(v > 0 ? "1e300" : (v < 0 ? "-1e300" : "0"));
        char text[40];
        std::snprintf(text, sizeof(text), "%.17g", v);
        out_ << text;
        return *this;
    }
    Json& integer(long long v)
    {
        out_ << v;
        return *this;
    }
    Json& boolean(bool v) { return raw(v ? "true" : "false"); }
    Json& str(const std::string& s)
    {
        out_ << '"';
        for (const char c : s) {
            if (c == '"' || c == '\\') out_ << '\\' << c;
            else out_ << (static_cast<unsigned char>(c) < 0x20 ? ' ' : c);
        }
        out_ << '"';
        return *this;
    }
    Json& ints(const std::vector<int>& v)
    {
        out_ << '[';
        const char* sep = "";
        for (const int x : v) {
            out_ << sep << x;
            sep = ",";
        }
        out_ << ']';
        return *this;
    }
    // "key": (a key with its quote and colon, after a comma unless it opens the object)
    Json& key(const char* k, bool first = false)
    {
        out_ << (first ? "" : ",") << '"' << k << "\":";
        return *this;
    }
    std::string text() const { return out_.str(); }

private:
    std::ostringstream out_;
};

void program_json(Json& j, const Program& p)
{
    j.raw("{").key("name", true).str(p.name).key("equations").raw("[");
    for (std::size_t e = 0; e < p.equations.size(); ++e) {
        j.raw(e ? ",[" : "[").integer(p.equations[e].target).raw(",").integer(p.equations[e].value).raw("]");
    }
    j.raw("]").key("stages").ints(p.stages).key("limit_stages").ints(p.limit_stages).key("in_place").boolean(p.in_place);
    j.key("max_dt").integer(p.max_dt).key("reads").ints(p.reads).key("writes").ints(p.writes).key("conserves").raw("[");
    for (std::size_t g = 0; g < p.conserves.size(); ++g) {
        if (g) j.raw(",");
        j.ints(p.conserves[g]);
    }
    j.raw("]").key("accumulate").boolean(p.accumulate).raw("}");
}

} // namespace

Module lower(const law::Law& law, int prelower)
{
    Module m;
    Builder b(m, law);
    for (int n = 0; n < prelower; ++n) b.value_of(n);
    for (const law::Term& term : law.terms) {
        m.terms.push_back(start_program(b, term.name, term.equations, term.max_dt));
        m.terms.back().conserves = term.conserves;
        m.learned.push_back(start_program(b, term.name + "~learned", term.learned, term.learned_max_dt));
        m.learned.back().conserves = term.conserves;
    }
    // A derive that adds into a field an earlier derive of the same field already started accumulates.
    std::vector<char> started(law.fields.size(), 0);
    for (const law::Derive& d : law.derives) {
        Program p = start_program(b, "derive " + law.fields[static_cast<std::size_t>(d.target)].name, {law::Equation{d.target, d.rhs}}, -1);
        p.accumulate = d.accumulate && started[static_cast<std::size_t>(d.target)] != 0;
        started[static_cast<std::size_t>(d.target)] = 1;
        m.derives.push_back(std::move(p));
    }
    price_and_stage(m);
    for (auto* programs : {&m.terms, &m.learned}) {
        for (Program& p : *programs) finish(m, law, p);
    }
    for (Program& p : m.derives) {
        finish(m, law, p);
        p.in_place = false; // a derive writes its own buffer, never a field it reads
    }
    return m;
}

void widen_stages(Module& m)
{
    // Points of each value that stencils read (nets and whole-lattice ops read at the cell).
    std::vector<long long> points_read(m.insts.size(), 0);
    for (const Inst& in : m.insts) {
        if (in.radius == 0 || in.global || in.net) continue;
        for (const int a : in.args) points_read[static_cast<std::size_t>(a)] += info(in.op).points;
    }
    bool changed = false;
    for (std::size_t id = 0; id < m.insts.size(); ++id) {
        const Inst& in = m.insts[id];
        const bool candidate = !m.is_stage(static_cast<int>(id)) && in.shape == Shape::Cell && in.op != Op::Field && points_read[id] >= 2;
        if (candidate && in.cost * points_read[id] > kInlineBudget) {
            m.materialized[id] = 1;
            changed = true;
        }
    }
    if (!changed) return;
    for (auto* programs : {&m.terms, &m.learned, &m.derives}) {
        for (Program& p : *programs) {
            std::vector<int> roots;
            for (const Equation& eq : p.equations) roots.push_back(eq.value);
            p.stages = stages_of(m, roots);
            p.limit_stages = p.max_dt >= 0 ? stages_of(m, {p.max_dt}) : std::vector<int>{};
        }
    }
}

std::string to_json(const Module& m, const law::Law& law)
{
    Json j;
    j.raw("{").key("version", true).integer(1).key("fields").raw("[");
    for (std::size_t f = 0; f < law.fields.size(); ++f) {
        const law::FieldDecl& d = law.fields[f];
        j.raw(f ? ",{" : "{").key("name", true).str(d.name).key("init").num(d.init).key("lo").num(d.lo).key("hi").num(d.hi);
        j.key("clamp").boolean(d.clamp).key("static").boolean(d.is_static).key("derived").boolean(d.derived).raw("}");
    }
    j.raw("]").key("params").raw("[");
    for (std::size_t p = 0; p < law.param_names.size(); ++p) {
        j.raw(p ? ",{" : "{").key("name", true).str(law.param_names[p]).key("value").num(law.param_values[p]).raw("}");
    }
    j.raw("]").key("nets").raw("[");
    for (std::size_t n = 0; n < law.nets.size(); ++n) {
        const law::NetDecl& net = law.nets[n];
        j.raw(n ? ",{" : "{").key("name", true).str(net.name).key("file").str(net.file).key("sizes").ints(net.sizes);
        j.key("act").str(net.act).key("half").boolean(net.half).key("loaded").boolean(net.loaded).raw("}");
    }
    j.raw("]").key("insts").raw("[");
    for (std::size_t i = 0; i < m.insts.size(); ++i) {
        const Inst& in = m.insts[i];
        j.raw(i ? ",\n{" : "\n{").key("op", true).str(law::op_name(in.op)).key("shape").str(in.shape == Shape::Cell ? "cell" : "scalar");
        j.key("number").num(in.number).key("index").integer(in.index).key("iterations").integer(in.iterations);
        j.key("offset").ints({in.offset[0], in.offset[1], in.offset[2]}).key("args").ints(in.args).key("radius").integer(in.radius);
        j.key("stage").boolean(m.is_stage(static_cast<int>(i))).raw("}");
    }
    j.raw("],\n");
    const std::pair<const char*, const std::vector<Program>*> lists[] = {{"terms", &m.terms}, {"learned", &m.learned}, {"derives", &m.derives}};
    for (std::size_t l = 0; l < 3; ++l) {
        j.raw(l ? "],\n" : "").key(lists[l].first, true).raw("[");
        const std::vector<Program>& progs = *lists[l].second;
        for (std::size_t p = 0; p < progs.size(); ++p) {
            j.raw(p ? ",\n" : "\n");
            program_json(j, progs[p]);
        }
    }
    j.raw("]}\n");
    return j.text();
}

std::string describe(const Module& m, const law::Law& law)
{
    std::ostringstream out;
    out << m.insts.size() << " instructions (" << m.shared << " found twice and kept once, " << m.folded << " folded away)\n";
    for (std::size_t i = 0; i < m.insts.size(); ++i) {
        const Inst& in = m.insts[i];
        out << "  %" << i << " = " << law::op_name(in.op);
        switch (in.op) {
        case Op::Const: out << ' ' << in.number; break;
        case Op::Field: out << ' ' << law.fields[static_cast<std::size_t>(in.index)].name; break;
        case Op::Param: out << ' ' << law.param_names[static_cast<std::size_t>(in.index)]; break;
        default: break;
        }
        for (const int a : in.args) out << " %" << a;
        if (in.op == Op::Shift) out << " (" << in.offset[0] << ',' << in.offset[1] << ',' << in.offset[2] << ')';
        if (in.op == Op::Tridiag) out << (in.index >= 3 ? " transposed" : "") << " along " << "xyz"[in.index % 3];
        out << "   [" << (in.shape == Shape::Cell ? "cell" : "scalar");
        if (in.radius > 0) out << ", reads " << in.radius << " away";
        if (m.is_stage(static_cast<int>(i))) out << (in.global ? ", global" : in.net ? ", net" : ", stored");
        out << ", cost " << in.cost << "]\n";
    }
    for (const auto* programs : {&m.terms, &m.learned, &m.derives}) {
        for (const Program& p : *programs) {
            if (p.equations.empty()) continue;
            out << p.name << ": " << p.equations.size() << " equation(s), " << p.stages.size() << " stage(s), "
                << (p.in_place ? "one kernel (in place)" : "one kernel (ping-pong buffers)") << "\n";
            for (const int s : p.stages) out << "    stage %" << s << " " << law::op_name(m.insts[static_cast<std::size_t>(s)].op) << "\n";
            for (const Equation& eq : p.equations) {
                out << "    d " << law.fields[static_cast<std::size_t>(eq.target)].name << " = %" << eq.value << "\n";
            }
            if (p.max_dt >= 0) out << "    max_dt = %" << p.max_dt << "\n";
        }
    }
    return out.str();
}

} // namespace fe::ir
