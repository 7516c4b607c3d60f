#include "adjoint.hpp"

#include "ir.hpp"

#include <cmath>
#include <cstdio>
#include <map>
#include <set>
#include <sstream>
#include <vector>

namespace fe::adjoint {

using ir::Inst;
using ir::Shape;
using law::Op;

namespace {

std::string number(double v)
{
    char text[40];
    std::snprintf(text, sizeof(text), "%.17g", std::abs(v));
    const std::string s = text;
    return v < 0.0 ? "(0 - " + s + ")" : s;
}

// A number in a declaration (field init, param value): a plain signed literal.
std::string literal(double v)
{
    char text[40];
    std::snprintf(text, sizeof(text), "%.17g", v);
    return text;
}

std::string offsets(const int* d)
{
    return std::to_string(d[0]) + ", " + std::to_string(d[1]) + ", " + std::to_string(d[2]);
}

class Builder {
public:
    Builder(const law::Law& law, const ir::Module& m) : law_(law), m_(m) {}

    std::string build(std::size_t t, std::string& error)
    {
        const ir::Program& p = m_.terms[t];
        if (p.equations.empty()) {
            error = "term '" + p.name + "' has no equations";
            return {};
        }
        // What the equations reach, and which of it depends on a field or a param (only that carries an adjoint).
        std::vector<int> stack;
        for (const ir::Equation& eq : p.equations) stack.push_back(eq.value);
        while (!stack.empty()) {
            const int id = stack.back();
            stack.pop_back();
            if (!reached_.insert(id).second) continue;
            for (const int a : at(id).args) stack.push_back(a);
        }
        live_.assign(m_.insts.size(), 0);
        for (std::size_t id = 0; id < m_.insts.size(); ++id) {
            const Inst& in = at(static_cast<int>(id));
            bool live = in.op == Op::Field || in.op == Op::Param;
            for (const int a : in.args) live = live || live_[static_cast<std::size_t>(a)];
            live_[id] = live;
        }
        std::ostringstream lets;
        for (const int id : reached_) {
            const Inst& in = at(id);
            if (leaf(in)) continue;
            std::string e;
            if (!primal(id, e, error)) return {};
            lets << "  let pv__" << id << " = " << e << "\n";
        }
        // Seeds: the cotangent of each written field is its adjoint field.
        std::set<int> written;
        for (const ir::Equation& eq : p.equations) {
            give(eq.value, law_.fields[static_cast<std::size_t>(eq.target)].name + "__adj");
            written.insert(eq.target);
        }
        std::map<int, std::string> field_rate, param_rate;
        for (auto it = reached_.rbegin(); it != reached_.rend(); ++it) {
            const int id = *it;
            if (!live_[static_cast<std::size_t>(id)]) continue;
            auto found = adj_.find(id);
            if (found == adj_.end() || found->second.empty()) continue;
            std::string sum;
            for (const std::string& term : found->second) sum += (sum.empty() ? "" : " + ") + term;
            const std::string A = "av__" + std::to_string(id);
            lets << "  let " << A << " = " << sum << "\n";
            const Inst& in = at(id);
            if (in.op == Op::Field) {
                field_rate[in.index] = A;
                continue;
            }
            if (in.op == Op::Param) {
                param_rate[in.index] = A;
                continue;
            }
            if (!backward(id, A, lets, error)) return {};
        }
        // The law.
        std::ostringstream out;
        out << "# The adjoint of term '" << p.name << "' (reverse mode over its SSA instructions). The primal fields are static\n"
            << "# inputs written by the driver each step; X__adj is the cotangent of X, a param's adjoint field sums to its gradient.\n";
        std::set<int> fields;
        for (const int id : reached_) {
            if (at(id).op == Op::Field) fields.insert(at(id).index);
        }
        for (const int f : written) fields.insert(f);
        for (const int f : fields) {
            const law::FieldDecl& d = law_.fields[static_cast<std::size_t>(f)];
            out << "field " << d.name << " init " << literal(d.init) << " range -1e30 1e30 static\n";
        }
        std::set<int> adj_fields(written.begin(), written.end());
        for (const auto& [f, _] : field_rate) adj_fields.insert(f);
        for (const int f : adj_fields) {
            out << "field " << law_.fields[static_cast<std::size_t>(f)].name << "__adj init 0 range -1e30 1e30\n";
        }
        for (const auto& [q, _] : param_rate) {
            out << "field " << law_.param_names[static_cast<std::size_t>(q)] << "__adj init 0 range -1e30 1e30\n";
        }
        for (std::size_t q = 0; q < law_.param_names.size(); ++q) {
            out << "param " << law_.param_names[q] << " = " << literal(law_.param_values[q]) << "\n";
        }
        out << "term " << p.name << "__adj\n" << lets.str();
        bool any = false;
        for (const auto& [f, rate] : field_rate) {
            out << "  d " << law_.fields[static_cast<std::size_t>(f)].name << "__adj = " << rate << "\n";
            any = true;
        }
        for (const auto& [q, rate] : param_rate) {
            out << "  d " << law_.param_names[static_cast<std::size_t>(q)] << "__adj = " << rate << "\n";
            any = true;
        }
        if (!any) {
            // Nothing depends on the state: the cotangent passes through unchanged.
            const int f = *written.begin();
            out << "  d " << law_.fields[static_cast<std::size_t>(f)].name << "__adj = 0\n";
        }
        return out.str();
    }

private:
    const Inst& at(int id) const { return m_.insts[static_cast<std::size_t>(id)]; }

    static bool leaf(const Inst& in)
    {
        return in.op == Op::Const || in.op == Op::Param || in.op == Op::Field || in.op == Op::Cell || in.op == Op::Dt;
    }

    // A value as the adjoint law writes it: leaves by name, the rest by their let.
    std::string name(int id) const
    {
        const Inst& in = at(id);
        switch (in.op) {
        case Op::Const: return number(in.number);
        case Op::Param: return law_.param_names[static_cast<std::size_t>(in.index)];
        case Op::Field: return law_.fields[static_cast<std::size_t>(in.index)].name;
        case Op::Cell: return "h";
        case Op::Dt: return "dt";
        default: return "pv__" + std::to_string(id);
        }
    }

    bool primal(int id, std::string& e, std::string& error) const
    {
        const Inst& in = at(id);
        auto a = [&](std::size_t k) { return name(in.args[k]); };
        switch (in.op) {
        case Op::Neg: e = "(0 - " + a(0) + ")"; return true;
        case Op::Add: e = "(" + a(0) + " + " + a(1) + ")"; return true;
        case Op::Sub: e = "(" + a(0) + " - " + a(1) + ")"; return true;
        case Op::Mul: e = "(" + a(0) + " * " + a(1) + ")"; return true;
        case Op::Div: e = "(" + a(0) + " / " + a(1) + ")"; return true;
        case Op::Pow: e = "(" + a(0) + " ^ " + a(1) + ")"; return true;
        case Op::Min: case Op::Max: e = std::string(law::op_name(in.op)) + "(" + a(0) + ", " + a(1) + ")"; return true;
        case Op::Abs: case Op::Sqrt: case Op::Exp: case Op::Log: case Op::Step: case Op::Pos: case Op::Lap: case Op::Gx: case Op::Gy:
        case Op::Gz: case Op::GxT: case Op::GyT: case Op::GzT:
            e = std::string(law::op_name(in.op)) + "(" + a(0) + ")";
            return true;
        case Op::Clamp: e = "clamp(" + a(0) + ", " + a(1) + ", " + a(2) + ")"; return true;
        case Op::Diffuse: e = "diffuse(" + a(0) + ", " + a(1) + ")"; return true;
        case Op::Shift: e = "shift(" + a(0) + ", " + offsets(in.offset) + ")"; return true;
        case Op::ShiftT: e = "shift_t(" + a(0) + ", " + offsets(in.offset) + ")"; return true;
        case Op::Rim: e = "rim"; return true;
        case Op::Tridiag:
            e = std::string("tridiag_") + "xyz"[in.index % 3] + (in.index >= 3 ? "_t(" : "(") + a(0) + ", " + a(1) + ", " + a(2) + ", " +
                a(3) + ")";
            return true;
        default:
            error = std::string("no adjoint for '") + law::op_name(in.op) + "'";
            return false;
        }
    }

    void give(int id, const std::string& term)
    {
        if (live_[static_cast<std::size_t>(id)] && at(id).op != Op::Const) adj_[id].push_back(term);
    }

    bool backward(int id, const std::string& A, std::ostringstream& lets, std::string& error)
    {
        const Inst& in = at(id);
        const std::string P = name(id);
        auto x = [&](std::size_t k) { return name(in.args[k]); };
        auto arg = [&](std::size_t k) { return in.args[k]; };
        switch (in.op) {
        case Op::Add: give(arg(0), A); give(arg(1), A); return true;
        case Op::Sub: give(arg(0), A); give(arg(1), "(0 - " + A + ")"); return true;
        case Op::Neg: give(arg(0), "(0 - " + A + ")"); return true;
        case Op::Mul: give(arg(0), "(" + A + " * " + x(1) + ")"); give(arg(1), "(" + A + " * " + x(0) + ")"); return true;
        case Op::Div:
            // Guarded division (0 where the divisor is 0), and so are its adjoints.
            give(arg(0), "(" + A + " / " + x(1) + ")");
            give(arg(1), "(0 - " + A + " * " + P + " / " + x(1) + ")");
            return true;
        case Op::Pow:
            give(arg(0), "(" + A + " * " + x(1) + " * (" + x(0) + " ^ (" + x(1) + " - 1)))");
            give(arg(1), "(" + A + " * " + P + " * log(" + x(0) + "))");
            return true;
        case Op::Min:
            give(arg(0), "(" + A + " * (1 - step(" + x(0) + " - " + x(1) + ")))");
            give(arg(1), "(" + A + " * step(" + x(0) + " - " + x(1) + "))");
            return true;
        case Op::Max:
            give(arg(0), "(" + A + " * (1 - step(" + x(1) + " - " + x(0) + ")))");
            give(arg(1), "(" + A + " * step(" + x(1) + " - " + x(0) + "))");
            return true;
        case Op::Abs: give(arg(0), "(" + A + " * (step(" + x(0) + ") - step(0 - " + x(0) + ")))"); return true;
        case Op::Sqrt: give(arg(0), "(" + A + " * 0.5 / " + P + ")"); return true;
        case Op::Exp: give(arg(0), "(" + A + " * " + P + " * (1 - step(" + x(0) + " - 80)))"); return true;
        case Op::Log: give(arg(0), "(" + A + " * step(" + x(0) + " - 1e-30) / " + x(0) + ")"); return true;
        case Op::Step: return true;
        case Op::Pos: give(arg(0), "(" + A + " * step(" + x(0) + "))"); return true;
        case Op::Clamp:
            if (live_[static_cast<std::size_t>(arg(1))] || live_[static_cast<std::size_t>(arg(2))]) {
                error = "no adjoint for clamp with bounds that depend on fields or params";
                return false;
            }
            give(arg(0), "(" + A + " * step(" + x(0) + " - " + x(1) + ") * step(" + x(2) + " - " + x(0) + "))");
            return true;
        case Op::Lap: give(arg(0), "lap(" + A + ")"); return true;
        case Op::Gx: give(arg(0), "gx_t(" + A + ")"); return true;
        case Op::Gy: give(arg(0), "gy_t(" + A + ")"); return true;
        case Op::Gz: give(arg(0), "gz_t(" + A + ")"); return true;
        case Op::GxT: give(arg(0), "gx(" + A + ")"); return true;
        case Op::GyT: give(arg(0), "gy(" + A + ")"); return true;
        case Op::GzT: give(arg(0), "gz(" + A + ")"); return true;
        case Op::Shift: give(arg(0), "shift_t(" + A + ", " + offsets(in.offset) + ")"); return true;
        case Op::ShiftT: give(arg(0), "shift(" + A + ", " + offsets(in.offset) + ")"); return true;
        case Op::Diffuse:
            if (at(arg(0)).shape != Shape::Scalar) {
                error = "no adjoint for diffuse whose k is a field";
                return false;
            }
            give(arg(1), "diffuse(" + x(0) + ", " + A + ")");
            give(arg(0), "(" + A + " * diffuse(1, " + x(1) + ") * step(" + x(0) + "))");
            return true;
        case Op::Tridiag: {
            if (in.index >= 3) {
                error = "no adjoint for a transposed tridiagonal solve";
                return false;
            }
            const char ax = "xyz"[in.index];
            const std::string Y = "yv__" + std::to_string(id);
            lets << "  let " << Y << " = tridiag_" << ax << "_t(" << x(0) << ", " << x(1) << ", " << x(2) << ", " << A << ")\n";
            int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
            lo[in.index] = -1;
            hi[in.index] = 1;
            give(arg(3), Y);
            give(arg(0), "(0 - " + Y + " * shift(" + P + ", " + offsets(lo) + "))");
            give(arg(1), "(0 - " + Y + " * " + P + ")");
            give(arg(2), "(0 - " + Y + " * shift(" + P + ", " + offsets(hi) + "))");
            return true;
        }
        case Op::Rim: case Op::Cell: case Op::Dt: case Op::Const:
            return true;
        default:
            error = std::string("no adjoint for '") + law::op_name(in.op) + "'";
            return false;
        }
    }

    const law::Law& law_;
    const ir::Module& m_;
    std::set<int> reached_;
    std::vector<char> live_;
    std::map<int, std::vector<std::string>> adj_;
};

} // namespace

std::string adjoint_law(const law::Law& law, const std::string& term, std::string& error)
{
    const ir::Module m = ir::lower(law);
    std::size_t t = 0;
    if (!term.empty()) {
        while (t < m.terms.size() && m.terms[t].name != term) ++t;
    }
    if (t >= m.terms.size()) {
        error = "no term '" + term + "'";
        return {};
    }
    Builder b(law, m);
    return b.build(t, error);
}

} // namespace fe::adjoint
