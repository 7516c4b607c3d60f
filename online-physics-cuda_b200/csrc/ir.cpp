#include "ir.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <functional>
#include <map>
#include <set>
#include <sstream>
#include <tuple>

namespace fe::ir {

namespace {

bool pure_arithmetic(Op op)
{
    switch (op) {
    case Op::Neg: case Op::Add: case Op::Sub: case Op::Mul: case Op::Div: case Op::Pow: case Op::Min: case Op::Max:
    case Op::Abs: case Op::Sqrt: case Op::Exp: case Op::Log: case Op::Step: case Op::Pos: case Op::Clamp:
        return true;
    default:
        return false;
    }
}

// Folding computes what the CPU's scalar path computes, in double (Law.cpp:757-860).
double fold(Op op, const std::vector<double>& a)
{
    switch (op) {
    case Op::Neg: return -a[0];
    case Op::Abs: return std::abs(a[0]);
    case Op::Sqrt: return std::sqrt(std::max(0.0, a[0]));
    case Op::Exp: return std::exp(std::min(a[0], 80.0));
    case Op::Log: return std::log(std::max(a[0], 1e-30));
    case Op::Step: return a[0] > 0.0 ? 1.0 : 0.0;
    case Op::Pos: return std::max(a[0], 0.0);
    case Op::Add: return a[0] + a[1];
    case Op::Sub: return a[0] - a[1];
    case Op::Mul: return a[0] * a[1];
    case Op::Div: return a[1] == 0.0 ? 0.0 : a[0] / a[1];
    case Op::Pow: return std::pow(a[0], a[1]);
    case Op::Min: return std::min(a[0], a[1]);
    case Op::Max: return std::max(a[0], a[1]);
    case Op::Clamp: return std::clamp(a[0], a[1], std::max(a[1], a[2]));
    default: return 0.0;
    }
}

// Points of each argument one point of the op reads (the cost model's weight).
int points(Op op)
{
    switch (op) {
    case Op::Lap: case Op::Diffuse: case Op::Adv: return 7;
    case Op::Gx: case Op::Gy: case Op::Gz: return 2;
    case Op::Fall: return 3;
    case Op::Spread: return 5;
    case Op::Topple: return 13;
    default: return 1;
    }
}

// The structural identity of an instruction: two with equal keys are one value.
using Key = std::tuple<int, std::uint64_t, int, int, int, int, int, std::vector<int>>;

std::uint64_t bits(double v)
{
    std::uint64_t b = 0;
    static_assert(sizeof(b) == sizeof(v), "double is 64-bit");
    __builtin_memcpy(&b, &v, sizeof(b));
    return b;
}

class Lowering {
public:
    Lowering(Module& m, const law::Law& law) : m_(m), law_(law) {}

    int lower(int node_id)
    {
        const auto found = memo_.find(node_id);
        if (found != memo_.end()) return found->second;
        const law::Node& n = law_.nodes[static_cast<std::size_t>(node_id)];
        Inst in;
        in.op = n.op;
        in.number = n.number;
        in.index = n.index;
        in.iterations = n.iterations;
        if (n.op == Op::Shift || n.op == Op::ShiftT) {
            in.args.push_back(lower(n.args[0]));
            for (int a = 0; a < 3; ++a) {
                in.offset[a] = static_cast<int>(law_.nodes[static_cast<std::size_t>(n.args[static_cast<std::size_t>(a) + 1])].number);
            }
        } else {
            for (const int a : n.args) in.args.push_back(lower(a));
        }
        const int id = simplify(in);
        memo_.emplace(node_id, id);
        return id;
    }

private:
    [[nodiscard]] const Inst& at(int id) const { return m_.insts[static_cast<std::size_t>(id)]; }
    [[nodiscard]] bool is_const(int id, double v) const { return at(id).op == Op::Const && at(id).number == v; }

    int constant(double v)
    {
        Inst c;
        c.op = Op::Const;
        c.number = v;
        return add(c);
    }

    int simplify(Inst in)
    {
        if (pure_arithmetic(in.op) && std::all_of(in.args.begin(), in.args.end(), [&](int a) { return at(a).op == Op::Const; })) {
            std::vector<double> v;
            for (const int a : in.args) v.push_back(at(a).number);
            ++m_.folded;
            return constant(fold(in.op, v));
        }
        switch (in.op) {
        case Op::Mul:
            if (is_const(in.args[0], 0.0) || is_const(in.args[1], 0.0)) { ++m_.folded; return constant(0.0); }
            if (is_const(in.args[0], 1.0)) { ++m_.folded; return in.args[1]; }
            if (is_const(in.args[1], 1.0)) { ++m_.folded; return in.args[0]; }
            break;
        case Op::Add:
            if (is_const(in.args[0], 0.0)) { ++m_.folded; return in.args[1]; }
            if (is_const(in.args[1], 0.0)) { ++m_.folded; return in.args[0]; }
            break;
        case Op::Sub:
            if (is_const(in.args[1], 0.0)) { ++m_.folded; return in.args[0]; }
            break;
        case Op::Div:
            if (is_const(in.args[1], 1.0)) { ++m_.folded; return in.args[0]; }
            if (is_const(in.args[0], 0.0)) { ++m_.folded; return constant(0.0); }
            break;
        case Op::Neg:
            if (at(in.args[0]).op == Op::Neg) { ++m_.folded; return at(in.args[0]).args[0]; }
            break;
        case Op::Shift:
            if (at(in.args[0]).shape == Shape::Scalar || (in.offset[0] == 0 && in.offset[1] == 0 && in.offset[2] == 0)) {
                ++m_.folded;
                return in.args[0];
            }
            break;
        case Op::Lap: case Op::Gx: case Op::Gy: case Op::Gz:
            if (at(in.args[0]).shape == Shape::Scalar) { ++m_.folded; return constant(0.0); }
            break;
        case Op::Diffuse: case Op::LDiffuse:
            if (at(in.args[1]).shape == Shape::Scalar) { ++m_.folded; return constant(0.0); }
            break;
        case Op::Adv: case Op::Fall: case Op::Spread: case Op::Topple:
            if (at(in.args[0]).shape == Shape::Scalar) { ++m_.folded; return constant(0.0); }
            break;
        default:
            break;
        }
        return add(in);
    }

    int add(Inst in)
    {
        switch (in.op) {
        case Op::Const: case Op::Param: case Op::Cell: case Op::Dt: case Op::Local: case Op::MaxOf: case Op::MinOf: case Op::SumOf:
            in.shape = Shape::Scalar;
            break;
        case Op::Field: case Op::Rim: case Op::Distance: case Op::Poisson: case Op::Fall: case Op::Spread: case Op::Topple:
        case Op::Flux: case Op::LDiffuse: case Op::Lap: case Op::Gx: case Op::Gy: case Op::Gz: case Op::Diffuse: case Op::Adv:
        case Op::Tridiag: case Op::ShiftT: case Op::GxT: case Op::GyT: case Op::GzT:
            in.shape = Shape::Cell;
            break;
        default:
            in.shape = std::any_of(in.args.begin(), in.args.end(), [&](int a) { return at(a).shape == Shape::Cell; }) ? Shape::Cell : Shape::Scalar;
            break;
        }
        switch (in.op) {
        case Op::Lap: case Op::Gx: case Op::Gy: case Op::Gz: case Op::Diffuse: case Op::Adv: case Op::Fall: case Op::Spread:
        case Op::Topple: case Op::Flux: case Op::GxT: case Op::GyT: case Op::GzT:
            in.radius = 1;
            break;
        case Op::LDiffuse:
            in.radius = 2;
            break;
        case Op::Shift: case Op::ShiftT:
            in.radius = std::max({std::abs(in.offset[0]), std::abs(in.offset[1]), std::abs(in.offset[2])});
            break;
        default:
            break;
        }
        in.global = in.op == Op::Distance || in.op == Op::Poisson || in.op == Op::MaxOf || in.op == Op::MinOf || in.op == Op::SumOf ||
            in.op == Op::Tridiag;
        in.net = in.op == Op::Mlp || in.op == Op::Flux || in.op == Op::LDiffuse;
        const Key key{static_cast<int>(in.op), bits(in.number), in.index, in.iterations, in.offset[0], in.offset[1], in.offset[2], in.args};
        const auto [where, inserted] = table_.emplace(key, static_cast<int>(m_.insts.size()));
        if (!inserted) {
            ++m_.shared;
            return where->second;
        }
        m_.insts.push_back(std::move(in));
        return where->second;
    }

    Module& m_;
    const law::Law& law_;
    std::map<int, int> memo_;
    std::map<Key, int> table_;
};

void plan_stages(Module& m)
{
    m.materialized.assign(m.insts.size(), 0);
    for (std::size_t id = 0; id < m.insts.size(); ++id) {
        Inst& in = m.insts[id];
        const int per = points(in.op);
        int cost = 1;
        for (const int a : in.args) {
            Inst& arg = m.insts[static_cast<std::size_t>(a)];
            const bool stored = m.is_stage(a);
            int c = stored ? 1 : arg.cost;
            const bool walked = in.op == Op::Tridiag && arg.op != Op::Field;
            if (!stored && arg.shape == Shape::Cell && arg.op != Op::Field && (walked || (in.radius > 0 && c * per > kInlineBudget))) {
                m.materialized[static_cast<std::size_t>(a)] = 1;
                c = 1;
            }
            cost += c * per;
            ++arg.uses;
        }
        in.cost = std::min(cost, 1 << 20);
    }
}

void collect_stages(const Module& m, int id, std::set<int>& out, std::set<int>& seen)
{
    if (!seen.insert(id).second) return;
    for (const int a : m.insts[static_cast<std::size_t>(id)].args) collect_stages(m, a, out, seen);
    if (m.is_stage(id) && m.insts[static_cast<std::size_t>(id)].shape == Shape::Cell) out.insert(id);
    if (m.insts[static_cast<std::size_t>(id)].global) out.insert(id);
}

void reach(const Module& m, int id, int offset, bool root, std::map<int, int>& out)
{
    const Inst& in = m.insts[static_cast<std::size_t>(id)];
    if (!root && m.is_stage(id)) return;
    if (in.op == Op::Field) {
        int& r = out[in.index];
        r = std::max(r, offset);
        return;
    }
    if (in.net || in.global) return;
    for (const int a : in.args) reach(m, a, offset + in.radius, false, out);
}

Program make_program(Lowering& low, const std::string& name, const std::vector<law::Equation>& equations, int max_dt)
{
    Program p;
    p.name = name;
    std::set<int> writes;
    for (const law::Equation& eq : equations) {
        p.equations.push_back(Equation{eq.target, low.lower(eq.rhs)});
        writes.insert(eq.target);
    }
    if (max_dt >= 0) p.max_dt = low.lower(max_dt);
    p.writes.assign(writes.begin(), writes.end());
    return p;
}

void finish_program(const Module& m, Program& p)
{
    std::set<int> stages, seen;
    for (const Equation& eq : p.equations) collect_stages(m, eq.value, stages, seen);
    p.stages.assign(stages.begin(), stages.end());
    if (p.max_dt >= 0) {
        std::set<int> limit, seen_limit;
        collect_stages(m, p.max_dt, limit, seen_limit);
        p.limit_stages.assign(limit.begin(), limit.end());
    }
    std::set<int> reads;
    std::function<void(int)> walk = [&](int id) {
        const Inst& in = m.insts[static_cast<std::size_t>(id)];
        if (in.op == Op::Field) reads.insert(in.index);
        for (const int a : in.args) walk(a);
    };
    for (const Equation& eq : p.equations) walk(eq.value);
    p.reads.assign(reads.begin(), reads.end());
    std::map<int, int> offsets;
    for (const Equation& eq : p.equations) reach(m, eq.value, 0, true, offsets);
    p.in_place = true;
    for (const int t : p.writes) {
        const auto f = offsets.find(t);
        if (f != offsets.end() && f->second > 0) p.in_place = false;
    }
}

void json_number(std::ostream& out, double v)
{
    if (!std::isfinite(v)) {
        out << (v > 0 ? "1e300" : (v < 0 ? "-1e300" : "0"));
        return;
    }
    char text[40];
    std::snprintf(text, sizeof(text), "%.17g", v);
    out << text;
}

void json_string(std::ostream& out, const std::string& s)
{
    out << '"';
    for (const char c : s) {
        if (c == '"' || c == '\\') out << '\\' << c;
        else if (static_cast<unsigned char>(c) < 0x20) out << ' ';
        else out << c;
    }
    out << '"';
}

void json_ints(std::ostream& out, const std::vector<int>& v)
{
    out << '[';
    for (std::size_t i = 0; i < v.size(); ++i) out << (i ? "," : "") << v[i];
    out << ']';
}

void json_program(std::ostream& out, const Program& p)
{
    out << "{\"name\":";
    json_string(out, p.name);
    out << ",\"equations\":[";
    for (std::size_t e = 0; e < p.equations.size(); ++e) out << (e ? "," : "") << '[' << p.equations[e].target << ',' << p.equations[e].value << ']';
    out << "],\"stages\":";
    json_ints(out, p.stages);
    out << ",\"limit_stages\":";
    json_ints(out, p.limit_stages);
    out << ",\"in_place\":" << (p.in_place ? "true" : "false") << ",\"max_dt\":" << p.max_dt << ",\"reads\":";
    json_ints(out, p.reads);
    out << ",\"writes\":";
    json_ints(out, p.writes);
    out << ",\"conserves\":[";
    for (std::size_t g = 0; g < p.conserves.size(); ++g) {
        out << (g ? "," : "");
        json_ints(out, p.conserves[g]);
    }
    out << "],\"accumulate\":" << (p.accumulate ? "true" : "false") << '}';
}

} // namespace

void widen_stages(Module& m)
{
    std::vector<int> reads(m.insts.size(), 0);
    for (const Inst& in : m.insts) {
        if (in.radius == 0 || in.global || in.net) continue;
        for (const int a : in.args) reads[static_cast<std::size_t>(a)] += points(in.op);
    }
    bool any = false;
    for (std::size_t id = 0; id < m.insts.size(); ++id) {
        const Inst& in = m.insts[id];
        if (m.is_stage(static_cast<int>(id)) || in.shape != Shape::Cell || in.op == Op::Field || reads[id] < 2) continue;
        if (static_cast<long long>(in.cost) * reads[id] > kInlineBudget) {
            m.materialized[id] = 1;
            any = true;
        }
    }
    if (!any) return;
    for (auto* programs : {&m.terms, &m.learned, &m.derives}) {
        for (Program& p : *programs) {
            std::set<int> stages, seen;
            for (const Equation& eq : p.equations) collect_stages(m, eq.value, stages, seen);
            p.stages.assign(stages.begin(), stages.end());
            if (p.max_dt >= 0) {
                std::set<int> limit, seen_limit;
                collect_stages(m, p.max_dt, limit, seen_limit);
                p.limit_stages.assign(limit.begin(), limit.end());
            }
        }
    }
}

Module lower(const law::Law& law)
{
    Module m;
    Lowering low(m, law);
    for (const law::Term& term : law.terms) {
        m.terms.push_back(make_program(low, term.name, term.equations, term.max_dt));
        m.terms.back().conserves = term.conserves;
        m.learned.push_back(make_program(low, term.name + "~learned", term.learned, term.learned_max_dt));
        m.learned.back().conserves = term.conserves;
    }
    std::set<int> started;
    for (const law::Derive& d : law.derives) {
        Program p = make_program(low, "derive " + law.fields[static_cast<std::size_t>(d.target)].name, {law::Equation{d.target, d.rhs}}, -1);
        p.accumulate = d.accumulate && started.count(d.target) != 0;
        started.insert(d.target);
        m.derives.push_back(std::move(p));
    }
    plan_stages(m);
    for (Program& p : m.terms) finish_program(m, p);
    for (Program& p : m.learned) finish_program(m, p);
    for (Program& p : m.derives) {
        finish_program(m, p);
        p.in_place = false;
    }
    return m;
}

std::string to_json(const Module& m, const law::Law& law)
{
    std::ostringstream out;
    out << "{\"version\":1,\"fields\":[";
    for (std::size_t f = 0; f < law.fields.size(); ++f) {
        const law::FieldDecl& d = law.fields[f];
        out << (f ? "," : "") << "{\"name\":";
        json_string(out, d.name);
        out << ",\"init\":";
        json_number(out, d.init);
        out << ",\"lo\":";
        json_number(out, d.lo);
        out << ",\"hi\":";
        json_number(out, d.hi);
        out << ",\"clamp\":" << (d.clamp ? "true" : "false") << ",\"static\":" << (d.is_static ? "true" : "false")
            << ",\"derived\":" << (d.derived ? "true" : "false") << '}';
    }
    out << "],\"params\":[";
    for (std::size_t p = 0; p < law.param_names.size(); ++p) {
        out << (p ? "," : "") << "{\"name\":";
        json_string(out, law.param_names[p]);
        out << ",\"value\":";
        json_number(out, law.param_values[p]);
        out << '}';
    }
    out << "],\"nets\":[";
    for (std::size_t n = 0; n < law.nets.size(); ++n) {
        const law::NetDecl& net = law.nets[n];
        out << (n ? "," : "") << "{\"name\":";
        json_string(out, net.name);
        out << ",\"file\":";
        json_string(out, net.file);
        out << ",\"sizes\":";
        json_ints(out, net.sizes);
        out << ",\"act\":\"" << net.act << "\",\"half\":" << (net.half ? "true" : "false") << ",\"loaded\":" << (net.loaded ? "true" : "false") << "}";
    }
    out << "],\"insts\":[";
    for (std::size_t i = 0; i < m.insts.size(); ++i) {
        const Inst& in = m.insts[i];
        out << (i ? ",\n" : "\n") << "{\"op\":\"" << law::op_name(in.op) << "\",\"shape\":\"" << (in.shape == Shape::Cell ? "cell" : "scalar")
            << "\",\"number\":";
        json_number(out, in.number);
        out << ",\"index\":" << in.index << ",\"iterations\":" << in.iterations << ",\"offset\":[" << in.offset[0] << ','
            << in.offset[1] << ',' << in.offset[2] << "],\"args\":";
        json_ints(out, in.args);
        out << ",\"radius\":" << in.radius << ",\"stage\":" << (m.is_stage(static_cast<int>(i)) ? "true" : "false") << '}';
    }
    out << "],\n\"terms\":[";
    for (std::size_t t = 0; t < m.terms.size(); ++t) {
        out << (t ? ",\n" : "\n");
        json_program(out, m.terms[t]);
    }
    out << "],\n\"learned\":[";
    for (std::size_t t = 0; t < m.learned.size(); ++t) {
        out << (t ? ",\n" : "\n");
        json_program(out, m.learned[t]);
    }
    out << "],\n\"derives\":[";
    for (std::size_t d = 0; d < m.derives.size(); ++d) {
        out << (d ? ",\n" : "\n");
        json_program(out, m.derives[d]);
    }
    out << "]}\n";
    return out.str();
}

std::string describe(const Module& m, const law::Law& law)
{
    std::ostringstream out;
    out << m.insts.size() << " instructions (" << m.shared << " found twice and kept once, " << m.folded << " folded away)\n";
    for (std::size_t i = 0; i < m.insts.size(); ++i) {
        const Inst& in = m.insts[i];
        out << "  %" << i << " = " << law::op_name(in.op);
        if (in.op == Op::Const) out << ' ' << in.number;
        else if (in.op == Op::Field) out << ' ' << law.fields[static_cast<std::size_t>(in.index)].name;
        else if (in.op == Op::Param) out << ' ' << law.param_names[static_cast<std::size_t>(in.index)];
        for (const int a : in.args) out << " %" << a;
        if (in.op == Op::Shift) out << " (" << in.offset[0] << ',' << in.offset[1] << ',' << in.offset[2] << ')';
        if (in.op == Op::Tridiag) out << (in.index >= 3 ? " transposed" : "") << " along " << "xyz"[in.index % 3];
        out << "   [" << (in.shape == Shape::Cell ? "cell" : "scalar");
        if (in.radius > 0) out << ", reads " << in.radius << " away";
        if (m.is_stage(static_cast<int>(i))) out << (in.global ? ", global" : in.net ? ", net" : ", stored");
        out << ", cost " << in.cost << "]\n";
    }
    auto program = [&](const Program& p) {
        if (p.equations.empty()) return;
        out << p.name << ": " << p.equations.size() << " equation(s), " << p.stages.size() << " stage(s), "
            << (p.in_place ? "one kernel (in place)" : "one kernel (ping-pong buffers)") << "\n";
        for (const int s : p.stages) out << "    stage %" << s << " " << law::op_name(m.insts[static_cast<std::size_t>(s)].op) << "\n";
        for (const Equation& eq : p.equations) out << "    d " << law.fields[static_cast<std::size_t>(eq.target)].name << " = %" << eq.value << "\n";
        if (p.max_dt >= 0) out << "    max_dt = %" << p.max_dt << "\n";
    };
    for (const Program& p : m.terms) program(p);
    for (const Program& p : m.learned) program(p);
    for (const Program& p : m.derives) program(p);
    return out.str();
}

} // namespace fe::ir
