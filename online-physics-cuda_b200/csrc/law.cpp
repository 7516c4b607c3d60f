#include "law.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <map>
#include <set>
#include <sstream>

namespace fe::law {

const char* op_name(Op op)
{
    static const char* names[] = {"const", "param", "h", "rim", "field", "neg", "add", "sub", "mul", "div", "pow", "min",
        "max", "abs", "sqrt", "exp", "log", "step", "pos", "clamp", "lap", "gx", "gy", "gz", "diffuse", "adv", "distance",
        "poisson", "maxof", "minof", "sumof", "fall", "spread", "topple", "shift", "local", "mlp", "flux", "ldiffuse", "dt",
        "tridiag", "shift_t", "gx_t", "gy_t", "gz_t"};
    const auto i = static_cast<std::size_t>(op);
    return i < sizeof(names) / sizeof(names[0]) ? names[i] : "?";
}

int Law::field_id(const std::string& name) const
{
    for (std::size_t i = 0; i < fields.size(); ++i) {
        if (fields[i].name == name) return static_cast<int>(i);
    }
    return -1;
}

int Law::param_id(const std::string& name) const
{
    for (std::size_t i = 0; i < param_names.size(); ++i) {
        if (param_names[i] == name) return static_cast<int>(i);
    }
    return -1;
}

int Law::net_id(const std::string& name) const
{
    for (std::size_t i = 0; i < nets.size(); ++i) {
        if (nets[i].name == name) return static_cast<int>(i);
    }
    return -1;
}

namespace {

// ---- tokens (the reference's lexical rules, Law.cpp:47-122) -----------------------------------------------------------

struct Token {
    enum Kind { Number, Name, Symbol, End } kind = End;
    std::string text;
    double number = 0.0;
};

bool is_digit(char c) { return std::isdigit(static_cast<unsigned char>(c)) != 0; }
bool is_alpha(char c) { return std::isalpha(static_cast<unsigned char>(c)) != 0; }
bool is_alnum(char c) { return std::isalnum(static_cast<unsigned char>(c)) != 0; }

std::vector<Token> tokenize(const std::string& line, std::string& error)
{
    std::vector<Token> out;
    std::size_t i = 0;
    while (i < line.size()) {
        const char c = line[i];
        if (c == '#') break;
        if (std::isspace(static_cast<unsigned char>(c))) {
            ++i;
            continue;
        }
        if (is_digit(c) || (c == '.' && i + 1 < line.size() && is_digit(line[i + 1]))) {
            std::size_t j = i;
            while (j < line.size() && (is_digit(line[j]) || line[j] == '.')) ++j;
            if (j < line.size() && (line[j] == 'e' || line[j] == 'E')) {
                std::size_t k = j + 1;
                if (k < line.size() && (line[k] == '+' || line[k] == '-')) ++k;
                if (k < line.size() && is_digit(line[k])) {
                    j = k;
                    while (j < line.size() && is_digit(line[j])) ++j;
                }
            }
            Token t;
            t.kind = Token::Number;
            t.text = line.substr(i, j - i);
            try {
                std::size_t used = 0;
                t.number = std::stod(t.text, &used);
            } catch (...) {
                error = "bad number '" + t.text + "'";
                return {};
            }
            out.push_back(t);
            i = j;
            continue;
        }
        if (is_alpha(c) || c == '_') {
            std::size_t j = i;
            while (j < line.size() && (is_alnum(line[j]) || line[j] == '_')) ++j;
            Token t;
            t.kind = Token::Name;
            t.text = line.substr(i, j - i);
            out.push_back(t);
            i = j;
            continue;
        }
        if (std::string("+-*/^(),=").find(c) != std::string::npos) {
            Token t;
            t.kind = Token::Symbol;
            t.text = std::string(1, c);
            out.push_back(t);
            ++i;
            continue;
        }
        error = std::string("unexpected character '") + c + "'";
        return {};
    }
    out.push_back(Token{});
    return out;
}

struct FunctionSpec {
    Op op;
    int min_args;
    int max_args;
};

// The function table (Law.cpp:126-144).
const std::map<std::string, FunctionSpec>& functions()
{
    static const std::map<std::string, FunctionSpec> table = {
        {"abs", {Op::Abs, 1, 1}}, {"sqrt", {Op::Sqrt, 1, 1}}, {"exp", {Op::Exp, 1, 1}}, {"log", {Op::Log, 1, 1}},
        {"step", {Op::Step, 1, 1}}, {"pos", {Op::Pos, 1, 1}}, {"min", {Op::Min, 2, 2}}, {"max", {Op::Max, 2, 2}},
        {"clamp", {Op::Clamp, 3, 3}}, {"lap", {Op::Lap, 1, 1}}, {"gx", {Op::Gx, 1, 1}}, {"gy", {Op::Gy, 1, 1}},
        {"gz", {Op::Gz, 1, 1}}, {"diffuse", {Op::Diffuse, 2, 2}}, {"adv", {Op::Adv, 4, 4}}, {"distance", {Op::Distance, 1, 1}},
        {"poisson", {Op::Poisson, 1, 2}}, {"maxof", {Op::MaxOf, 1, 1}}, {"minof", {Op::MinOf, 1, 1}},
        {"sumof", {Op::SumOf, 1, 1}}, {"fall", {Op::Fall, 3, 3}}, {"spread", {Op::Spread, 3, 3}},
        {"topple", {Op::Topple, 3, 3}}, {"shift", {Op::Shift, 4, 4}}, {"shift_t", {Op::ShiftT, 4, 4}},
        {"gx_t", {Op::GxT, 1, 1}}, {"gy_t", {Op::GyT, 1, 1}}, {"gz_t", {Op::GzT, 1, 1}},
        {"tridiag_x", {Op::Tridiag, 4, 4}}, {"tridiag_y", {Op::Tridiag, 4, 4}}, {"tridiag_z", {Op::Tridiag, 4, 4}},
        {"tridiag_x_t", {Op::Tridiag, 4, 4}}, {"tridiag_y_t", {Op::Tridiag, 4, 4}}, {"tridiag_z_t", {Op::Tridiag, 4, 4}},
        {"mlp", {Op::Mlp, 2, 33}}, {"flux", {Op::Flux, 2, 9}}, {"ldiffuse", {Op::LDiffuse, 3, 3}},
    };
    return table;
}

bool is_reserved(const std::string& name)
{
    static const std::set<std::string> reserved = {"field", "param", "term", "derive", "creature", "show", "d", "conserves",
        "max_dt", "h", "dt", "pi", "inf", "init", "range", "unit", "static", "clamp", "net", "learned", "plan", "observe", "let"};
    return reserved.count(name) != 0 || functions().count(name) != 0;
}

int net_inputs(const NetDecl& n) { return n.sizes.empty() ? 0 : n.sizes.front(); }
int net_outputs(const NetDecl& n) { return n.sizes.empty() ? 0 : n.sizes.back(); }

// ---- expressions (precedence climbing, Law.cpp:148-410) ----------------------------------------------------------------

class Parser {
public:
    Parser(Law& law, const std::vector<Token>& tokens, std::size_t start, const std::map<std::string, int>* lets)
        : law_(law), t_(tokens), pos_(start), lets_(lets)
    {
    }

    int expression()
    {
        int left = product();
        while (ok() && (peek("+") || peek("-"))) {
            const bool add = take().text == "+";
            const int right = product();
            left = make(add ? Op::Add : Op::Sub, {left, right});
        }
        return left;
    }

    [[nodiscard]] bool ok() const { return error_.empty(); }
    [[nodiscard]] bool at_end() const { return t_[pos_].kind == Token::End; }
    [[nodiscard]] const std::string& error() const { return error_; }

private:
    int make(Op op, std::vector<int> args = {})
    {
        Node n;
        n.op = op;
        n.args = std::move(args);
        law_.nodes.push_back(std::move(n));
        return static_cast<int>(law_.nodes.size()) - 1;
    }

    int constant(double v)
    {
        const int id = make(Op::Const);
        law_.nodes[static_cast<std::size_t>(id)].number = v;
        return id;
    }

    int product()
    {
        int left = unary();
        while (ok() && (peek("*") || peek("/"))) {
            const bool mul = take().text == "*";
            const int right = unary();
            left = make(mul ? Op::Mul : Op::Div, {left, right});
        }
        return left;
    }

    int unary()
    {
        if (peek("-")) {
            take();
            return make(Op::Neg, {unary()});
        }
        if (peek("+")) {
            take();
            return unary();
        }
        return power();
    }

    int power()
    {
        const int base = primary();
        if (ok() && peek("^")) {
            take();
            const int exponent = unary(); // right-associative
            return make(Op::Pow, {base, exponent});
        }
        return base;
    }

    int primary()
    {
        const Token& tok = t_[pos_];
        if (tok.kind == Token::Number) {
            ++pos_;
            return constant(tok.number);
        }
        if (tok.kind == Token::Symbol && tok.text == "(") {
            ++pos_;
            const int inner = expression();
            expect(")");
            return inner;
        }
        if (tok.kind == Token::Name) {
            ++pos_;
            if (peek("(")) return call(tok.text);
            return name(tok.text);
        }
        fail(tok.kind == Token::End ? "expression ends too early" : "unexpected '" + tok.text + "'");
        return constant(0.0);
    }

    int call(const std::string& function)
    {
        take(); // (
        std::vector<int> args;
        int net = -1;
        const bool net_op = function == "mlp" || function == "flux" || function == "ldiffuse";
        if (net_op) {
            const Token& nm = t_[pos_];
            net = nm.kind == Token::Name ? law_.net_id(nm.text) : -1;
            if (net < 0) {
                fail("'" + function + "' takes the name of a declared net first");
                return constant(0.0);
            }
            ++pos_;
            if (!peek(",")) {
                fail("expected ',' after the net's name");
                return constant(0.0);
            }
            take();
        }
        if (!peek(")")) {
            args.push_back(expression());
            while (ok() && peek(",")) {
                take();
                args.push_back(expression());
            }
        }
        expect(")");
        const auto found = functions().find(function);
        if (found == functions().end()) {
            fail("unknown function '" + function + "'");
            return constant(0.0);
        }
        const FunctionSpec& spec = found->second;
        // The reference counts the net's place as an argument (Law.cpp:262-275).
        const int count = static_cast<int>(args.size()) + (net_op ? 1 : 0);
        if (count < spec.min_args || count > spec.max_args) {
            fail("'" + function + "' takes " + std::to_string(spec.min_args) +
                (spec.max_args != spec.min_args ? "-" + std::to_string(spec.max_args) : "") + " argument(s), got " +
                std::to_string(count));
            return constant(0.0);
        }
        const int id = make(spec.op);
        Node& node = law_.nodes[static_cast<std::size_t>(id)];
        if (spec.op == Op::Tridiag) {
            // tridiag_x/_y/_z: axis 0/1/2; the transposed solves tridiag_x_t/_y_t/_z_t (adjoints; not in the
            // reference's language): 3 + axis.
            node.index = function[8] - 'x' + (function.size() > 9 ? 3 : 0);
        }
        if (net >= 0) {
            node.index = net;
            const NetDecl& decl = law_.nets[static_cast<std::size_t>(net)];
            const int given = static_cast<int>(args.size());
            const int wanted = spec.op == Op::Mlp ? given : (spec.op == Op::Flux ? 2 * given : 5);
            if (net_inputs(decl) != wanted) {
                fail("net '" + decl.name + "' takes " + std::to_string(net_inputs(decl)) + " inputs; " + function +
                    " here gives it " + std::to_string(wanted));
                return constant(0.0);
            }
            if (spec.op == Op::LDiffuse && net_outputs(decl) != 4) {
                fail("ldiffuse's net gives 4 weights, '" + decl.name + "' gives " + std::to_string(net_outputs(decl)));
                return constant(0.0);
            }
            const std::size_t moved = spec.op == Op::LDiffuse ? 1 : 0;
            if ((spec.op == Op::Flux || spec.op == Op::LDiffuse) &&
                law_.nodes[static_cast<std::size_t>(args[moved])].op != Op::Field) {
                fail(function + " moves a field: its " + (moved == 0 ? "first" : "second") + " argument after the net is a field's name");
                return constant(0.0);
            }
            if (spec.op == Op::Flux) {
                const FieldDecl& f = law_.fields[static_cast<std::size_t>(law_.nodes[static_cast<std::size_t>(args[0])].index)];
                args.push_back(constant(f.lo));
                args.push_back(constant(f.hi));
            }
            law_.nodes[static_cast<std::size_t>(id)].args = args;
            return id;
        }
        if (spec.op == Op::Poisson) {
            int iterations = 24;
            if (args.size() == 2) {
                const Node& a = law_.nodes[static_cast<std::size_t>(args[1])];
                if (a.op != Op::Const || a.number < 1.0) {
                    fail("poisson's iteration count must be a positive number");
                } else {
                    iterations = static_cast<int>(a.number);
                }
            }
            Node& n = law_.nodes[static_cast<std::size_t>(id)];
            n.iterations = iterations;
            n.args = {args[0]};
            return id;
        }
        if (spec.op == Op::Shift || spec.op == Op::ShiftT) {
            // Offsets are whole cells fixed when the law is written, at most 8 (Law.cpp:329-345).
            for (std::size_t a = 1; a < 4; ++a) {
                double sign = 1.0;
                const Node* arg = &law_.nodes[static_cast<std::size_t>(args[a])];
                if (arg->op == Op::Neg) {
                    sign = -1.0;
                    arg = &law_.nodes[static_cast<std::size_t>(arg->args[0])];
                }
                if (arg->op != Op::Const || arg->number != std::floor(arg->number) || std::abs(arg->number) > 8.0) {
                    fail("shift's offsets must be whole numbers of cells (at most 8)");
                    return constant(0.0);
                }
                args[a] = constant(sign * arg->number);
            }
        }
        law_.nodes[static_cast<std::size_t>(id)].args = args;
        return id;
    }

    int name(const std::string& text)
    {
        if (text == "h") return make(Op::Cell);
        if (text == "dt") return make(Op::Dt);
        if (text == "rim") return make(Op::Rim);
        if (text == "pi") return constant(3.14159265358979323846);
        if (lets_ != nullptr) {
            const auto found = lets_->find(text);
            if (found != lets_->end()) return found->second;
        }
        if (const int p = law_.param_id(text); p >= 0) {
            const int id = make(Op::Param);
            law_.nodes[static_cast<std::size_t>(id)].index = p;
            return id;
        }
        if (const int f = law_.field_id(text); f >= 0) {
            const int id = make(Op::Field);
            law_.nodes[static_cast<std::size_t>(id)].index = f;
            return id;
        }
        fail("unknown name '" + text + "' (not a field, param, h or pi)");
        return constant(0.0);
    }

    [[nodiscard]] bool peek(const char* s) const { return t_[pos_].kind == Token::Symbol && t_[pos_].text == s; }
    const Token& take() { return t_[pos_++]; }
    void expect(const char* s)
    {
        if (!peek(s)) {
            fail(std::string("expected '") + s + "'");
            return;
        }
        ++pos_;
    }
    void fail(const std::string& m)
    {
        if (error_.empty()) error_ = m;
    }

    Law& law_;
    const std::vector<Token>& t_;
    std::size_t pos_;
    const std::map<std::string, int>* lets_;
    std::string error_;
};

bool parse_bound(const std::vector<Token>& t, std::size_t& i, double& out)
{
    double sign = 1.0;
    if (t[i].kind == Token::Symbol && t[i].text == "-") {
        sign = -1.0;
        ++i;
    }
    if (t[i].kind == Token::Number) {
        out = sign * t[i].number;
        ++i;
        return true;
    }
    if (t[i].kind == Token::Name && t[i].text == "inf") {
        out = sign * 1e30;
        ++i;
        return true;
    }
    return false;
}

void collect_reads(const Law& law, int id, std::set<int>& out)
{
    const Node& n = law.nodes[static_cast<std::size_t>(id)];
    if (n.op == Op::Field) out.insert(n.index);
    for (const int a : n.args) collect_reads(law, a, out);
}

bool reads_dt(const Law& law, int id)
{
    const Node& n = law.nodes[static_cast<std::size_t>(id)];
    if (n.op == Op::Dt) return true;
    for (const int a : n.args) {
        if (reads_dt(law, a)) return true;
    }
    return false;
}

// Whether a node is one number whatever the fields hold (LawNode.hpp:87-123).
bool always_scalar(const Law& law, int id)
{
    const Node& n = law.nodes[static_cast<std::size_t>(id)];
    switch (n.op) {
    case Op::Const: case Op::Param: case Op::Cell: case Op::MaxOf: case Op::MinOf: case Op::SumOf:
        return true;
    case Op::Flux: case Op::LDiffuse: case Op::Field: case Op::Distance: case Op::Poisson: case Op::Fall: case Op::Spread:
    case Op::Topple: case Op::Tridiag: case Op::ShiftT: case Op::GxT: case Op::GyT: case Op::GzT:
        return false;
    default:
        for (const int a : n.args) {
            if (!always_scalar(law, a)) return false;
        }
        return true;
    }
}

struct Line {
    std::string where;
    std::vector<Token> tokens;
};

} // namespace

bool evaluate_scalar(const Law& law, int id, double h, double dt, double& out)
{
    const Node& n = law.nodes[static_cast<std::size_t>(id)];
    double a = 0.0, b = 0.0, c = 0.0;
    auto arg = [&](std::size_t k, double& v) { return evaluate_scalar(law, n.args[k], h, dt, v); };
    switch (n.op) {
    case Op::Const: out = n.number; return true;
    case Op::Param: out = law.param_values[static_cast<std::size_t>(n.index)]; return true;
    case Op::Cell: out = h; return true;
    case Op::Dt: out = dt; return true;
    case Op::Neg: if (!arg(0, a)) return false; out = -a; return true;
    case Op::Abs: if (!arg(0, a)) return false; out = std::abs(a); return true;
    case Op::Sqrt: if (!arg(0, a)) return false; out = std::sqrt(std::max(0.0, a)); return true;
    case Op::Exp: if (!arg(0, a)) return false; out = std::exp(std::min(a, 80.0)); return true;
    case Op::Log: if (!arg(0, a)) return false; out = std::log(std::max(a, 1e-30)); return true;
    case Op::Step: if (!arg(0, a)) return false; out = a > 0.0 ? 1.0 : 0.0; return true;
    case Op::Pos: if (!arg(0, a)) return false; out = std::max(a, 0.0); return true;
    case Op::Add: if (!arg(0, a) || !arg(1, b)) return false; out = a + b; return true;
    case Op::Sub: if (!arg(0, a) || !arg(1, b)) return false; out = a - b; return true;
    case Op::Mul:
        // Zero times anything is zero without looking at the anything (Law.cpp:818-830).
        if (!arg(0, a)) return false;
        if (a == 0.0) { out = 0.0; return true; }
        if (!arg(1, b)) return false;
        out = b == 0.0 ? 0.0 : a * b;
        return true;
    case Op::Div: if (!arg(0, a) || !arg(1, b)) return false; out = b == 0.0 ? 0.0 : a / b; return true;
    case Op::Pow: if (!arg(0, a) || !arg(1, b)) return false; out = std::pow(a, b); return true;
    case Op::Min: if (!arg(0, a) || !arg(1, b)) return false; out = std::min(a, b); return true;
    case Op::Max: if (!arg(0, a) || !arg(1, b)) return false; out = std::max(a, b); return true;
    case Op::Clamp:
        if (!arg(0, a) || !arg(1, b) || !arg(2, c)) return false;
        out = std::clamp(a, b, std::max(b, c));
        return true;
    case Op::Shift: case Op::MaxOf: case Op::MinOf: return arg(0, out);
    case Op::Lap: case Op::Gx: case Op::Gy: case Op::Gz:
        if (!arg(0, a)) return false;
        out = 0.0;
        return true;
    default:
        return false;
    }
}

Law compile(const std::vector<Source>& sources, std::vector<std::string>& errors)
{
    Law law;
    std::vector<Line> lines;
    for (const Source& src : sources) {
        std::istringstream stream(src.text);
        std::string raw;
        int number = 0;
        while (std::getline(stream, raw)) {
            ++number;
            if (!raw.empty() && raw.back() == '\r') raw.pop_back();
            const std::string where = src.name + ":" + std::to_string(number);
            std::string error;
            std::vector<Token> tokens = tokenize(raw, error);
            if (!error.empty()) {
                errors.push_back(where + ": " + error);
                continue;
            }
            if (tokens.size() > 1) lines.push_back(Line{where, std::move(tokens)});
        }
    }

    auto top_level = [](const std::string& k) {
        return k == "field" || k == "param" || k == "term" || k == "derive" || k == "show" || k == "net";
    };

    // Pass 1: declarations (Law.cpp:1690-1870): nets, fields, and fields first named by a derive.
    bool creature = false;
    for (const Line& line : lines) {
        const std::vector<Token>& t = line.tokens;
        if (t[0].kind != Token::Name) continue;
        const std::string& k = t[0].text;
        if (top_level(k)) creature = false;
        if (k == "creature") {
            creature = true;
            continue;
        }
        if (creature) continue;
        if (k == "net") {
            if (t[1].kind != Token::Name || is_reserved(t[1].text) || law.net_id(t[1].text) >= 0) {
                errors.push_back(line.where + ": expected 'net NAME in N hidden H... out M act tanh|relu|silu [half] [file PATH]'");
                continue;
            }
            NetDecl net;
            net.name = t[1].text;
            net.file = "assets/nets/" + net.name + ".net";
            int in = 0, out = 0;
            std::vector<int> hidden;
            bool bad = false;
            std::string section;
            std::size_t i = 2;
            while (t[i].kind != Token::End && !bad) {
                const Token& tok = t[i++];
                if (tok.kind == Token::Number) {
                    if (section == "in") in = static_cast<int>(tok.number);
                    else if (section == "hidden") hidden.push_back(static_cast<int>(tok.number));
                    else if (section == "out") out = static_cast<int>(tok.number);
                    else bad = true;
                    continue;
                }
                section = tok.text;
                if (section == "act") {
                    bad = t[i].kind != Token::Name ||
                        !(t[i].text == "tanh" || t[i].text == "relu" || t[i].text == "silu" || t[i].text == "linear");
                    net.act = t[i].text;
                    ++i;
                } else if (section == "half") {
                    net.half = true;
                } else if (section == "file") {
                    std::string path;
                    while (t[i].kind != Token::End && !(t[i].kind == Token::Name && (t[i].text == "half" || t[i].text == "act"))) {
                        path += t[i].kind == Token::Number ? std::to_string(static_cast<long long>(t[i].number)) : t[i].text;
                        ++i;
                    }
                    bad = path.empty();
                    net.file = path;
                } else if (section != "in" && section != "hidden" && section != "out") {
                    bad = true;
                }
            }
            if (bad || in < 1 || out < 1 || in > 64 || out > 64 || hidden.size() > 6 ||
                std::any_of(hidden.begin(), hidden.end(), [](int h) { return h < 1 || h > 128; })) {
                errors.push_back(line.where + ": malformed net (in 1..64, hidden up to 6 layers of 1..128, out 1..64)");
                continue;
            }
            net.sizes.push_back(in);
            net.sizes.insert(net.sizes.end(), hidden.begin(), hidden.end());
            net.sizes.push_back(out);
            // Untrained unless its file is there (a missing file is not an error: the net starts at 0).
            init_net(net);
            std::string why;
            if (!load_net(net, why) && why.rfind("no weights at", 0) != 0) {
                errors.push_back(line.where + ": " + why);
                continue;
            }
            law.nets.push_back(net);
            continue;
        }
        if (k == "field") {
            if (t[1].kind != Token::Name || is_reserved(t[1].text)) {
                errors.push_back(line.where + ": 'field' needs a name that is not a keyword");
                continue;
            }
            if (law.field_id(t[1].text) >= 0) {
                errors.push_back(line.where + ": field '" + t[1].text + "' declared twice");
                continue;
            }
            FieldDecl decl;
            decl.name = t[1].text;
            std::size_t i = 2;
            bool bad = false;
            while (t[i].kind != Token::End && !bad) {
                const std::string key = t[i].text;
                ++i;
                if (key == "init") bad = !parse_bound(t, i, decl.init);
                else if (key == "range") bad = !parse_bound(t, i, decl.lo) || !parse_bound(t, i, decl.hi) || decl.lo > decl.hi;
                else if (key == "unit") {
                    bad = t[i].kind != Token::Name;
                    decl.unit = t[i].text;
                    ++i;
                } else if (key == "static") decl.is_static = true;
                else if (key == "clamp") decl.clamp = true;
                else bad = true;
            }
            if (bad) {
                errors.push_back(line.where + ": malformed field declaration (expected init N, range LO HI, unit U, static, clamp)");
                continue;
            }
            law.fields.push_back(decl);
        } else if (k == "derive" && t[1].kind == Token::Name && law.field_id(t[1].text) < 0 && !is_reserved(t[1].text)) {
            FieldDecl decl;
            decl.name = t[1].text;
            decl.derived = true;
            law.fields.push_back(decl);
        }
    }

    // Pass 2: params in order, terms, lets, equations, contracts, derives (Law.cpp:1872-2310).
    int current = -1;
    std::map<std::string, int> lets;
    std::set<int> derived_targets;
    creature = false;
    for (const Line& line : lines) {
        const std::vector<Token>& t = line.tokens;
        auto fail = [&](const std::string& m) { errors.push_back(line.where + ": " + m); };
        if (t[0].kind != Token::Name) {
            fail("a line starts with a keyword (field, param, term, let, derive, creature, d, conserves, max_dt)");
            continue;
        }
        const std::string& k = t[0].text;
        if (top_level(k)) creature = false;
        if (k == "creature") {
            creature = true;
            current = -1;
            continue;
        }
        if (creature || k == "net" || k == "show") continue; // creatures and looks are not the law step's
        if (k == "field") {
            current = -1;
            continue;
        }
        if (k == "param") {
            current = -1;
            if (t[1].kind != Token::Name || is_reserved(t[1].text) || !(t[2].kind == Token::Symbol && t[2].text == "=")) {
                fail("expected 'param NAME = expression'");
                continue;
            }
            if (law.param_id(t[1].text) >= 0 || law.field_id(t[1].text) >= 0) {
                fail("'" + t[1].text + "' is already a param or a field");
                continue;
            }
            Parser p(law, t, 3, nullptr);
            const int e = p.expression();
            if (!p.ok() || !p.at_end()) {
                fail(p.ok() ? "trailing tokens after the expression" : p.error());
                continue;
            }
            if (!always_scalar(law, e)) {
                fail("a param cannot read a field");
                continue;
            }
            double v = 0.0;
            if (!evaluate_scalar(law, e, 1.0, 0.0, v)) v = 0.0; // a one-cell lattice at h = 1 (Law.cpp:2132-2141)
            law.param_names.push_back(t[1].text);
            law.param_values.push_back(v);
            continue;
        }
        if (k == "term") {
            if (t[1].kind != Token::Name || t[2].kind != Token::End) {
                fail("expected 'term NAME'");
                current = -1;
                continue;
            }
            for (const Term& existing : law.terms) {
                if (existing.name == t[1].text) fail("term '" + t[1].text + "' declared twice");
            }
            Term term;
            term.name = t[1].text;
            term.where = line.where;
            law.terms.push_back(term);
            current = static_cast<int>(law.terms.size()) - 1;
            lets.clear();
            continue;
        }
        if (k == "let") {
            if (current < 0) {
                fail("'let' outside a term");
                continue;
            }
            if (t[1].kind != Token::Name || !(t[2].kind == Token::Symbol && t[2].text == "=")) {
                fail("expected 'let NAME = expression'");
                continue;
            }
            const std::string& nm = t[1].text;
            if (is_reserved(nm) || law.field_id(nm) >= 0 || law.param_id(nm) >= 0 || lets.count(nm)) {
                fail("'" + nm + "' is already a keyword, field, param or let");
                continue;
            }
            Parser p(law, t, 3, &lets);
            const int e = p.expression();
            if (!p.ok() || !p.at_end()) {
                fail(p.ok() ? "trailing tokens after the expression" : p.error());
                continue;
            }
            lets.emplace(nm, e);
            continue;
        }
        if (k == "derive") {
            current = -1;
            const int target = t[1].kind == Token::Name ? law.field_id(t[1].text) : -1;
            const bool accumulate = t[2].kind == Token::Symbol && t[2].text == "+" && t[3].kind == Token::Symbol && t[3].text == "=";
            if (target < 0 || !(accumulate || (t[2].kind == Token::Symbol && t[2].text == "="))) {
                fail("expected 'derive FIELD = expression' or 'derive FIELD += expression'");
                continue;
            }
            if (!accumulate && derived_targets.count(target)) {
                fail("field '" + t[1].text + "' is derived twice with '=' (use '+=' to add to it)");
                continue;
            }
            Parser p(law, t, accumulate ? 4 : 3, nullptr);
            const int e = p.expression();
            if (!p.ok() || !p.at_end()) {
                fail(p.ok() ? "trailing tokens after the expression" : p.error());
                continue;
            }
            law.fields[static_cast<std::size_t>(target)].derived = true;
            if (!accumulate) derived_targets.insert(target);
            Derive d;
            d.target = target;
            d.accumulate = accumulate;
            d.where = line.where;
            d.rhs = e;
            law.derives.push_back(d);
            continue;
        }
        if (k == "learned") {
            if (current < 0) {
                fail("'learned' outside a term");
                continue;
            }
            Term& term = law.terms[static_cast<std::size_t>(current)];
            if (t[1].kind == Token::Name && t[1].text == "d") {
                const int target = t[2].kind == Token::Name ? law.field_id(t[2].text) : -1;
                if (target < 0 || !(t[3].kind == Token::Symbol && t[3].text == "=")) {
                    fail("expected 'learned d FIELD = expression'");
                    continue;
                }
                Parser p(law, t, 4, &lets);
                const int e = p.expression();
                if (!p.ok() || !p.at_end()) {
                    fail(p.ok() ? "trailing tokens after the expression" : p.error());
                    continue;
                }
                term.learned.push_back(Equation{target, e});
            } else if (t[1].kind == Token::Name && t[1].text == "max_dt" && t[2].kind == Token::Symbol && t[2].text == "=") {
                Parser p(law, t, 3, nullptr);
                const int e = p.expression();
                if (!p.ok() || !p.at_end() || !always_scalar(law, e) || reads_dt(law, e)) {
                    fail(p.ok() ? "learned max_dt must be a number that does not read dt" : p.error());
                    continue;
                }
                term.learned_max_dt = e;
            } else {
                fail("expected 'learned d FIELD = expression' or 'learned max_dt = expression'");
            }
            continue;
        }
        if (k == "d" || k == "conserves" || k == "max_dt") {
            if (current < 0) {
                fail("'" + k + "' outside a term");
                continue;
            }
            Term& term = law.terms[static_cast<std::size_t>(current)];
            if (k == "d") {
                const int target = t[1].kind == Token::Name ? law.field_id(t[1].text) : -1;
                if (target < 0 || !(t[2].kind == Token::Symbol && t[2].text == "=")) {
                    fail("expected 'd FIELD = expression' with a declared field");
                    continue;
                }
                Parser p(law, t, 3, &lets);
                const int e = p.expression();
                if (!p.ok() || !p.at_end()) {
                    fail(p.ok() ? "trailing tokens after the expression" : p.error());
                    continue;
                }
                term.equations.push_back(Equation{target, e});
            } else if (k == "conserves") {
                bool join = false;
                for (std::size_t i = 1; t[i].kind != Token::End; ++i) {
                    if (t[i].kind == Token::Symbol && t[i].text == "+") {
                        join = true;
                        continue;
                    }
                    const int f = t[i].kind == Token::Name ? law.field_id(t[i].text) : -1;
                    if (f < 0) {
                        fail("conserves: '" + t[i].text + "' is not a field");
                        continue;
                    }
                    if (join && !term.conserves.empty()) term.conserves.back().push_back(f);
                    else term.conserves.push_back({f});
                    join = false;
                }
            } else {
                if (!(t[1].kind == Token::Symbol && t[1].text == "=")) {
                    fail("expected 'max_dt = expression'");
                    continue;
                }
                Parser p(law, t, 2, nullptr);
                const int e = p.expression();
                if (!p.ok() || !p.at_end()) {
                    fail(p.ok() ? "trailing tokens after the expression" : p.error());
                    continue;
                }
                if (!always_scalar(law, e)) {
                    fail("max_dt must be a number: use maxof/minof/sumof to reduce a field");
                    continue;
                }
                if (reads_dt(law, e)) {
                    fail("max_dt sets the step: it cannot read dt");
                    continue;
                }
                term.max_dt = e;
            }
            continue;
        }
        fail("unknown keyword '" + k + "'");
    }

    // Whole-law validation (Law.cpp:2318-2370).
    for (Term& term : law.terms) {
        std::set<int> reads, writes;
        for (const Equation& eq : term.equations) {
            collect_reads(law, eq.rhs, reads);
            writes.insert(eq.target);
            const FieldDecl& d = law.fields[static_cast<std::size_t>(eq.target)];
            if (d.is_static) errors.push_back(term.where + ": term '" + term.name + "' writes static field '" + d.name + "'");
            if (d.derived) errors.push_back(term.where + ": term '" + term.name + "' writes derived field '" + d.name + "'");
        }
        if (term.equations.empty()) errors.push_back(term.where + ": term '" + term.name + "' has no equations");
        for (const Equation& eq : term.learned) {
            collect_reads(law, eq.rhs, reads);
            if (!writes.count(eq.target)) {
                errors.push_back(term.where + ": term '" + term.name + "' has a learned equation for '" +
                    law.fields[static_cast<std::size_t>(eq.target)].name + "', which its own equations do not write");
            }
        }
        for (const std::vector<int>& group : term.conserves) {
            bool touched = false;
            std::string names;
            for (const int f : group) {
                touched = touched || writes.count(f);
                names += (names.empty() ? "" : " + ") + law.fields[static_cast<std::size_t>(f)].name;
            }
            if (!touched) {
                errors.push_back(term.where + ": term '" + term.name + "' conserves '" + names + "' but never writes it");
            }
        }
        term.reads.assign(reads.begin(), reads.end());
        term.writes.assign(writes.begin(), writes.end());
    }
    // Derives grouped per field in order of first appearance, '=' before '+=' (Law.cpp:2372-2392).
    {
        std::vector<int> order;
        for (const Derive& d : law.derives) {
            if (std::find(order.begin(), order.end(), d.target) == order.end()) order.push_back(d.target);
        }
        std::vector<Derive> grouped;
        for (const int target : order) {
            for (int pass = 0; pass < 2; ++pass) {
                for (const Derive& d : law.derives) {
                    if (d.target == target && d.accumulate == (pass == 1)) grouped.push_back(d);
                }
            }
        }
        law.derives = grouped;
    }
    return law;
}

} // namespace fe::law
