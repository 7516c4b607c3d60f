// The law language's front end: lines to tokens, tokens to expression nodes, statements to the Law.
//
// Design. A line is scanned once into tokens by a small character-class scanner. Expressions are read by a Pratt
// parser: one loop over infix operators ordered by binding power (+ - below * / below prefix signs below ^, which is
// right-associative and takes a signed exponent), with prefix handling for numbers, parentheses, names and calls.
// Calls are checked against a table of callees that carries each function's op, argument counts and special form
// (a net's name first, a solve's axis, poisson's iteration count, shift's whole-cell offsets). Statements are handled
// by keyword: a declaration table for the first pass (nets, fields, fields a derive names) and a statement table for
// the second (params in order, terms with their lets, equations, contracts and learned equations, derives), each
// handler reading its line through a small pattern view (Words). Two passes because a term may name any field or net
// of the law, wherever it is declared.
//
// The language is the reference's, unchanged: its lexical rules (src/field/Law.cpp:55-115), its grammar and
// precedence (Law.cpp:148-410), its function table (Law.cpp:126-144), its statements and their checks
// (Law.cpp:1662-2392) and its error messages, which tools and users match on. What the GPU backend does not run
// (creatures, `show` lines) is read past, not built.
#include "law.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <functional>
#include <map>
#include <set>
#include <sstream>
#include <string_view>
#include <unordered_map>

namespace fe::law {

const char* op_name(Op op)
{
    static constexpr const char* kNames[] = {"const", "param", "h", "rim", "field", "neg", "add", "sub", "mul", "div", "pow", "min",
        "max", "abs", "sqrt", "exp", "log", "step", "pos", "clamp", "lap", "gx", "gy", "gz", "diffuse", "adv", "distance",
        "poisson", "maxof", "minof", "sumof", "fall", "spread", "topple", "shift", "local", "mlp", "flux", "ldiffuse", "dt",
        "tridiag", "shift_t", "gx_t", "gy_t", "gz_t"};
    const auto i = static_cast<std::size_t>(op);
    return i < std::size(kNames) ? kNames[i] : "?";
}

namespace {

template <class T, class Name>
int index_named(const std::vector<T>& items, const std::string& name, Name name_of)
{
    const auto it = std::find_if(items.begin(), items.end(), [&](const T& x) { return name_of(x) == name; });
    return it == items.end() ? -1 : static_cast<int>(it - items.begin());
}

} // namespace

int Law::field_id(const std::string& name) const
{
    return index_named(fields, name, [](const FieldDecl& f) -> const std::string& { return f.name; });
}

int Law::param_id(const std::string& name) const
{
    return index_named(param_names, name, [](const std::string& s) -> const std::string& { return s; });
}

int Law::net_id(const std::string& name) const
{
    return index_named(nets, name, [](const NetDecl& n) -> const std::string& { return n.name; });
}

namespace {

// ---- scanning ------------------------------------------------------------------------------------------------------------

struct Token {
    enum Kind { Number, Name, Symbol, End } kind = End;
    std::string text;
    double number = 0.0;
};

bool digit(char c) { return std::isdigit(static_cast<unsigned char>(c)) != 0; }
bool name_start(char c) { return std::isalpha(static_cast<unsigned char>(c)) != 0 || c == '_'; }
bool name_char(char c) { return std::isalnum(static_cast<unsigned char>(c)) != 0 || c == '_'; }
bool symbol_char(char c) { return std::string_view("+-*/^(),=").find(c) != std::string_view::npos; }

class Scanner {
public:
    explicit Scanner(std::string_view s) : s_(s) {}

    // Every token of the line, ended by an End token; empty with `error` set when a character or number is bad.
    std::vector<Token> all(std::string& error)
    {
        std::vector<Token> out;
        for (;;) {
            skip_blanks();
            if (done()) break;
            const char c = s_[i_];
            if (digit(c) || (c == '.' && digit(at(i_ + 1)))) {
                Token t{Token::Number, std::string(take_number()), 0.0};
                try {
                    t.number = std::stod(t.text);
                } catch (...) {
                    error = "bad number '" + t.text + "'";
                    return {};
                }
                out.push_back(std::move(t));
            } else if (name_start(c)) {
                out.push_back(Token{Token::Name, std::string(take_while(name_char)), 0.0});
            } else if (symbol_char(c)) {
                out.push_back(Token{Token::Symbol, std::string(1, c), 0.0});
                ++i_;
            } else {
                error = std::string("unexpected character '") + c + "'";
                return {};
            }
        }
        out.push_back(Token{});
        return out;
    }

private:
    [[nodiscard]] char at(std::size_t i) const { return i < s_.size() ? s_[i] : '\0'; }
    // The line ends at its end or at a comment.
    [[nodiscard]] bool done() const { return i_ >= s_.size() || s_[i_] == '#'; }
    void skip_blanks()
    {
        while (i_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[i_]))) ++i_;
    }
    std::string_view take_while(bool (*pred)(char))
    {
        const std::size_t from = i_;
        while (i_ < s_.size() && pred(s_[i_])) ++i_;
        return s_.substr(from, i_ - from);
    }
    // Digits and dots, then an exponent only when digits follow its optional sign.
    std::string_view take_number()
    {
        const std::size_t from = i_;
        take_while([](char c) { return digit(c) || c == '.'; });
        if (at(i_) == 'e' || at(i_) == 'E') {
            std::size_t k = i_ + 1;
            if (at(k) == '+' || at(k) == '-') ++k;
            if (digit(at(k))) {
                i_ = k;
                take_while(digit);
            }
        }
        return s_.substr(from, i_ - from);
    }

    std::string_view s_;
    std::size_t i_ = 0;
};

// A line's tokens, read by position: what a statement expects at each place.
class Words {
public:
    explicit Words(const std::vector<Token>& t) : t_(t) {}
    [[nodiscard]] const Token& operator[](std::size_t i) const { return i < t_.size() ? t_[i] : t_.back(); }
    [[nodiscard]] bool name(std::size_t i) const { return (*this)[i].kind == Token::Name; }
    [[nodiscard]] bool name(std::size_t i, std::string_view s) const { return name(i) && (*this)[i].text == s; }
    [[nodiscard]] bool sym(std::size_t i, std::string_view s) const { return (*this)[i].kind == Token::Symbol && (*this)[i].text == s; }
    [[nodiscard]] bool end(std::size_t i) const { return (*this)[i].kind == Token::End; }
    [[nodiscard]] const std::string& text(std::size_t i) const { return (*this)[i].text; }
    [[nodiscard]] const std::vector<Token>& tokens() const { return t_; }

private:
    const std::vector<Token>& t_;
};

// ---- callees ---------------------------------------------------------------------------------------------------------------

enum class Form : unsigned char { Plain, Net, Solve, Poisson, Shift };

struct Callee {
    Op op;
    int min_args, max_args; // a net op counts the net's place among its arguments
    Form form = Form::Plain;
    int axis = 0;           // Solve: 0..2 along x/y/z, 3..5 the transposed solves (adjoint laws; not in the reference)
};

const std::unordered_map<std::string, Callee>& callees()
{
    static const std::unordered_map<std::string, Callee> table = [] {
        std::unordered_map<std::string, Callee> t;
        auto plain = [&t](const char* n, Op op, int lo, int hi) { t.emplace(n, Callee{op, lo, hi}); };
        for (auto [n, op] : {std::pair{"abs", Op::Abs}, {"sqrt", Op::Sqrt}, {"exp", Op::Exp}, {"log", Op::Log}, {"step", Op::Step},
                             {"pos", Op::Pos}, {"lap", Op::Lap}, {"gx", Op::Gx}, {"gy", Op::Gy}, {"gz", Op::Gz},
                             {"distance", Op::Distance}, {"maxof", Op::MaxOf}, {"minof", Op::MinOf}, {"sumof", Op::SumOf},
                             {"gx_t", Op::GxT}, {"gy_t", Op::GyT}, {"gz_t", Op::GzT}}) {
            plain(n, op, 1, 1);
        }
        plain("min", Op::Min, 2, 2);
        plain("max", Op::Max, 2, 2);
        plain("diffuse", Op::Diffuse, 2, 2);
        for (auto [n, op] : {std::pair{"clamp", Op::Clamp}, {"fall", Op::Fall}, {"spread", Op::Spread}, {"topple", Op::Topple}}) plain(n, op, 3, 3);
        plain("adv", Op::Adv, 4, 4);
        t.emplace("poisson", Callee{Op::Poisson, 1, 2, Form::Poisson});
        t.emplace("shift", Callee{Op::Shift, 4, 4, Form::Shift});
        t.emplace("shift_t", Callee{Op::ShiftT, 4, 4, Form::Shift});
        const char* solves[] = {"tridiag_x", "tridiag_y", "tridiag_z", "tridiag_x_t", "tridiag_y_t", "tridiag_z_t"};
        for (int a = 0; a < 6; ++a) t.emplace(solves[a], Callee{Op::Tridiag, 4, 4, Form::Solve, a});
        t.emplace("mlp", Callee{Op::Mlp, 2, 33, Form::Net});
        t.emplace("flux", Callee{Op::Flux, 2, 9, Form::Net});
        t.emplace("ldiffuse", Callee{Op::LDiffuse, 3, 3, Form::Net});
        return t;
    }();
    return table;
}

bool keyword(const std::string& s)
{
    static const std::set<std::string> words = {"field", "param", "term", "derive", "creature", "show", "d", "conserves",
        "max_dt", "h", "dt", "pi", "inf", "init", "range", "unit", "static", "clamp", "net", "learned", "plan", "observe", "let"};
    return words.count(s) != 0 || callees().count(s) != 0;
}

// ---- expressions ---------------------------------------------------------------------------------------------------------

using Lets = std::map<std::string, int>;

struct Infix {
    const char* symbol;
    Op op;
    int left;   // binding power against the operator before it
    int right;  // the least binding power its right operand may hold
};

// Sums bind loosest, then products, then a prefix sign, then powers; + - * / are left-associative, ^ right-associative
// with a signed exponent (2^-x).
constexpr int kPrefix = 30;
constexpr Infix kInfix[] = {
    {"+", Op::Add, 10, 11}, {"-", Op::Sub, 10, 11}, {"*", Op::Mul, 20, 21}, {"/", Op::Div, 20, 21}, {"^", Op::Pow, 40, kPrefix},
};

class Expr {
public:
    Expr(Law& law, const std::vector<Token>& tokens, std::size_t from, const Lets* lets) : law_(law), w_(tokens), pos_(from), lets_(lets) {}

    int parse() { return climb(0); }
    [[nodiscard]] bool ok() const { return error_.empty(); }
    [[nodiscard]] bool finished() const { return w_.end(pos_); }
    [[nodiscard]] const std::string& error() const { return error_; }

private:
    int climb(int min_power)
    {
        int left = operand();
        while (ok()) {
            const Infix* op = infix_here();
            if (op == nullptr || op->left < min_power) break;
            ++pos_;
            const int right = climb(op->right);
            left = node(op->op, {left, right});
        }
        return left;
    }

    const Infix* infix_here() const
    {
        for (const Infix& op : kInfix) {
            if (w_.sym(pos_, op.symbol)) return &op;
        }
        return nullptr;
    }

    int operand()
    {
        const Token& tok = w_[pos_];
        if (w_.sym(pos_, "-") || w_.sym(pos_, "+")) {
            ++pos_;
            const int inner = climb(kPrefix);
            return tok.text == "-" ? node(Op::Neg, {inner}) : inner;
        }
        if (tok.kind == Token::Number) {
            ++pos_;
            return number(tok.number);
        }
        if (w_.sym(pos_, "(")) {
            ++pos_;
            const int inner = climb(0);
            need(")");
            return inner;
        }
        if (tok.kind == Token::Name) {
            ++pos_;
            return w_.sym(pos_, "(") ? call(tok.text) : named(tok.text);
        }
        return bad(tok.kind == Token::End ? "expression ends too early" : "unexpected '" + tok.text + "'");
    }

    int call(const std::string& fn)
    {
        ++pos_; // (
        const auto entry = callees().find(fn);
        const bool takes_net = fn == "mlp" || fn == "flux" || fn == "ldiffuse";
        int net = -1;
        if (takes_net) {
            net = w_.name(pos_) ? law_.net_id(w_.text(pos_)) : -1;
            if (net < 0) return bad("'" + fn + "' takes the name of a declared net first");
            ++pos_;
            if (!w_.sym(pos_, ",")) return bad("expected ',' after the net's name");
            ++pos_;
        }
        std::vector<int> args;
        if (!w_.sym(pos_, ")")) {
            do {
                if (!args.empty()) ++pos_; // the comma
                args.push_back(climb(0));
            } while (ok() && w_.sym(pos_, ","));
        }
        need(")");
        if (entry == callees().end()) return bad("unknown function '" + fn + "'");
        const Callee& c = entry->second;
        const int count = static_cast<int>(args.size()) + (takes_net ? 1 : 0);
        if (count < c.min_args || count > c.max_args) {
            const std::string range = std::to_string(c.min_args) + (c.max_args != c.min_args ? "-" + std::to_string(c.max_args) : "");
            return bad("'" + fn + "' takes " + range + " argument(s), got " + std::to_string(count));
        }
        switch (c.form) {
        case Form::Net: return net_call(fn, c.op, net, std::move(args));
        case Form::Solve: {
            const int id = node(c.op, std::move(args));
            law_.nodes[static_cast<std::size_t>(id)].index = c.axis;
            return id;
        }
        case Form::Poisson: {
            int iterations = 24;
            if (args.size() == 2) {
                const Node& k = law_.nodes[static_cast<std::size_t>(args[1])];
                if (k.op == Op::Const && k.number >= 1.0) iterations = static_cast<int>(k.number);
                else bad("poisson's iteration count must be a positive number");
            }
            const int id = node(c.op, {args[0]});
            law_.nodes[static_cast<std::size_t>(id)].iterations = iterations;
            return id;
        }
        case Form::Shift:
            // Offsets are whole cells fixed when the law is written (a signed literal), at most 8 either way.
            for (std::size_t a = 1; a < 4; ++a) {
                double v = 0.0;
                if (!signed_literal(args[a], v) || v != std::floor(v) || std::abs(v) > 8.0) {
                    return bad("shift's offsets must be whole numbers of cells (at most 8)");
                }
                args[a] = number(v);
            }
            return node(c.op, std::move(args));
        case Form::Plain:
            break;
        }
        return node(c.op, std::move(args));
    }

    bool signed_literal(int id, double& v) const
    {
        const Node* n = &law_.nodes[static_cast<std::size_t>(id)];
        double sign = 1.0;
        if (n->op == Op::Neg) {
            sign = -1.0;
            n = &law_.nodes[static_cast<std::size_t>(n->args[0])];
        }
        if (n->op != Op::Const) return false;
        v = sign * n->number;
        return true;
    }

    int net_call(const std::string& fn, Op op, int net, std::vector<int> args)
    {
        const NetDecl& decl = law_.nets[static_cast<std::size_t>(net)];
        const int ins = decl.sizes.empty() ? 0 : decl.sizes.front();
        const int outs = decl.sizes.empty() ? 0 : decl.sizes.back();
        const int given = static_cast<int>(args.size());
        // mlp feeds its arguments; flux each argument on both sides of a face; ldiffuse a face's window of 4 cells
        // and the conductivity.
        const int feeds = op == Op::Mlp ? given : (op == Op::Flux ? 2 * given : 5);
        if (ins != feeds) {
            return bad("net '" + decl.name + "' takes " + std::to_string(ins) + " inputs; " + fn + " here gives it " + std::to_string(feeds));
        }
        if (op == Op::LDiffuse && outs != 4) {
            return bad("ldiffuse's net gives 4 weights (one per cell of the face's window), '" + decl.name + "' gives " + std::to_string(outs));
        }
        if (op != Op::Mlp) {
            const std::size_t moved = op == Op::LDiffuse ? 1 : 0;
            if (law_.nodes[static_cast<std::size_t>(args[moved])].op != Op::Field) {
                return bad(fn + " moves a field: its " + (moved == 0 ? "first" : "second") + " argument after the net is a field's name");
            }
        }
        if (op == Op::Flux) {
            // The moved field's declared range bounds the flux (its limiter).
            const FieldDecl& f = law_.fields[static_cast<std::size_t>(law_.nodes[static_cast<std::size_t>(args[0])].index)];
            args.push_back(number(f.lo));
            args.push_back(number(f.hi));
        }
        const int id = node(op, std::move(args));
        law_.nodes[static_cast<std::size_t>(id)].index = net;
        return id;
    }

    int named(const std::string& s)
    {
        if (s == "h") return node(Op::Cell);
        if (s == "dt") return node(Op::Dt);
        if (s == "rim") return node(Op::Rim);
        if (s == "pi") return number(3.14159265358979323846);
        if (lets_ != nullptr) {
            if (const auto it = lets_->find(s); it != lets_->end()) return it->second; // one node: every use is one value
        }
        for (const auto& [op, id] : {std::pair{Op::Param, law_.param_id(s)}, std::pair{Op::Field, law_.field_id(s)}}) {
            if (id < 0) continue;
            const int n = node(op);
            law_.nodes[static_cast<std::size_t>(n)].index = id;
            return n;
        }
        return bad("unknown name '" + s + "' (not a field, param, h or pi)");
    }

    int node(Op op, std::vector<int> args = {})
    {
        law_.nodes.push_back(Node{op, 0.0, -1, 0, std::move(args)});
        return static_cast<int>(law_.nodes.size()) - 1;
    }

    int number(double v)
    {
        const int id = node(Op::Const);
        law_.nodes[static_cast<std::size_t>(id)].number = v;
        return id;
    }

    void need(const char* s)
    {
        if (w_.sym(pos_, s)) ++pos_;
        else bad(std::string("expected '") + s + "'");
    }

    // The first error is the one reported; a stand-in node keeps the parse going.
    int bad(const std::string& message)
    {
        if (error_.empty()) error_ = message;
        return number(0.0);
    }

    Law& law_;
    Words w_;
    std::size_t pos_;
    const Lets* lets_;
    std::string error_;
};

// ---- graph queries -------------------------------------------------------------------------------------------------------

// Visits every node reachable from `root` (shared nodes once).
void visit(const Law& law, int root, const std::function<void(const Node&)>& f)
{
    std::vector<char> seen(law.nodes.size(), 0);
    std::vector<int> todo{root};
    while (!todo.empty()) {
        const int id = todo.back();
        todo.pop_back();
        if (seen[static_cast<std::size_t>(id)]) continue;
        seen[static_cast<std::size_t>(id)] = 1;
        const Node& n = law.nodes[static_cast<std::size_t>(id)];
        f(n);
        todo.insert(todo.end(), n.args.begin(), n.args.end());
    }
}

bool reads_dt(const Law& law, int id)
{
    bool dt = false;
    visit(law, id, [&](const Node& n) { dt = dt || n.op == Op::Dt; });
    return dt;
}

// Whether a node is one number whatever the fields hold (the reference's is_scalar, src/field/LawNode.hpp:87-123):
// numbers, params, h and the lattice reductions are; fields and whatever reads cells around a cell are not; the rest
// are when all their arguments are.
bool scalar(const Law& law, int id)
{
    const Node& n = law.nodes[static_cast<std::size_t>(id)];
    switch (n.op) {
    case Op::Const: case Op::Param: case Op::Cell: case Op::MaxOf: case Op::MinOf: case Op::SumOf:
        return true;
    case Op::Flux: case Op::LDiffuse: case Op::Field: case Op::Distance: case Op::Poisson: case Op::Fall: case Op::Spread:
    case Op::Topple: case Op::Tridiag: case Op::ShiftT: case Op::GxT: case Op::GyT: case Op::GzT:
        return false;
    default:
        return std::all_of(n.args.begin(), n.args.end(), [&](int a) { return scalar(law, a); });
    }
}

// ---- statements ----------------------------------------------------------------------------------------------------------

struct Line {
    std::string where;
    std::vector<Token> tokens;
};

// A field bound: an optionally negated number, or inf (1e30).
bool bound(const Words& w, std::size_t& i, double& out)
{
    const double sign = w.sym(i, "-") ? -1.0 : 1.0;
    if (sign < 0) ++i;
    if (w[i].kind == Token::Number) out = sign * w[i].number;
    else if (w.name(i, "inf")) out = sign * 1e30;
    else return false;
    ++i;
    return true;
}

// Statements that open a top-level block (and so end a creature's block).
bool opens_block(const std::string& k)
{
    return k == "field" || k == "param" || k == "term" || k == "derive" || k == "show" || k == "net";
}

class Compiler {
public:
    Compiler(Law& law, std::vector<std::string>& errors) : law_(law), errors_(errors) {}

    void run(const std::vector<Line>& lines)
    {
        using Handler = void (Compiler::*)(const Words&);
        static const std::unordered_map<std::string, Handler> declarations = {
            {"net", &Compiler::declare_net}, {"field", &Compiler::declare_field}, {"derive", &Compiler::declare_derived}};
        static const std::unordered_map<std::string, Handler> statements = {
            {"field", &Compiler::leave_term}, {"param", &Compiler::param}, {"term", &Compiler::term}, {"let", &Compiler::let},
            {"derive", &Compiler::derive}, {"learned", &Compiler::learned}, {"d", &Compiler::equation},
            {"conserves", &Compiler::conserves}, {"max_dt", &Compiler::max_dt}};
        // Pass 1: what every term may name.
        in_creature_ = false;
        for (const Line& line : lines) {
            where_ = &line.where;
            const Words w(line.tokens);
            if (!w.name(0) || skipped(w)) continue;
            if (const auto h = declarations.find(w.text(0)); h != declarations.end()) (this->*h->second)(w);
        }
        // Pass 2: everything else, in order.
        in_creature_ = false;
        for (const Line& line : lines) {
            where_ = &line.where;
            const Words w(line.tokens);
            if (!w.name(0)) {
                fail("a line starts with a keyword (field, param, term, let, derive, creature, d, conserves, max_dt)");
                continue;
            }
            if (skipped(w) || w.name(0, "net") || w.name(0, "show")) continue; // creatures and looks are not the law step's
            if (const auto h = statements.find(w.text(0)); h != statements.end()) (this->*h->second)(w);
            else fail("unknown keyword '" + w.text(0) + "'");
        }
        validate();
        order_derives();
    }

private:
    void fail(const std::string& m) { errors_.push_back(*where_ + ": " + m); }

    // Tracks creature blocks (from `creature` to the next top-level statement); true for lines inside one.
    bool skipped(const Words& w)
    {
        const std::string& k = w.text(0);
        if (opens_block(k)) in_creature_ = false;
        if (k == "creature") {
            in_creature_ = true;
            current_ = -1;
            return true;
        }
        return in_creature_;
    }

    // Parses the expression from token `from`; -1 after reporting a parse error or trailing tokens (with `trailing`
    // as the message for the latter, when given).
    int expression(const Words& w, std::size_t from, const Lets* lets, const char* trailing = "trailing tokens after the expression")
    {
        Expr e(law_, w.tokens(), from, lets);
        const int id = e.parse();
        if (!e.ok()) {
            fail(e.error());
            return -1;
        }
        if (!e.finished()) {
            fail(trailing);
            return -1;
        }
        return id;
    }

    Term* term_or_fail(const std::string& what)
    {
        if (current_ >= 0) return &law_.terms[static_cast<std::size_t>(current_)];
        fail("'" + what + "' outside a term");
        return nullptr;
    }

    // -- pass 1 --

    void declare_net(const Words& w)
    {
        if (!w.name(1) || keyword(w.text(1)) || law_.net_id(w.text(1)) >= 0) {
            fail("expected 'net NAME in N hidden H... out M act tanh|relu|silu [half] [file PATH]'");
            return;
        }
        NetDecl net;
        net.name = w.text(1);
        net.file = "assets/nets/" + net.name + ".net";
        // Sections: `in N`, `hidden H...`, `out M` take numbers; `act A`; `half`; `file` takes the rest of the line up
        // to `half` or `act`, its tokens joined as written (numbers as integers).
        std::map<std::string, std::vector<int>> sizes;
        std::string section;
        bool bad = false;
        for (std::size_t i = 2; !w.end(i) && !bad;) {
            if (w[i].kind == Token::Number) {
                bad = !(section == "in" || section == "hidden" || section == "out");
                sizes[section].push_back(static_cast<int>(w[i].number));
                ++i;
                continue;
            }
            section = w.text(i++);
            if (section == "act") {
                bad = !(w.name(i, "tanh") || w.name(i, "relu") || w.name(i, "silu") || w.name(i, "linear"));
                net.act = w.text(i++);
            } else if (section == "half") {
                net.half = true;
            } else if (section == "file") {
                std::string path;
                for (; !w.end(i) && !w.name(i, "half") && !w.name(i, "act"); ++i) {
                    path += w[i].kind == Token::Number ? std::to_string(static_cast<long long>(w[i].number)) : w.text(i);
                }
                bad = path.empty();
                net.file = path;
            } else {
                bad = !(section == "in" || section == "hidden" || section == "out");
            }
        }
        // The last number given for `in` and `out` counts; every `hidden` number is a layer.
        const int in = sizes["in"].empty() ? 0 : sizes["in"].back();
        const int out = sizes["out"].empty() ? 0 : sizes["out"].back();
        const std::vector<int>& hidden = sizes["hidden"];
        const bool hidden_ok = hidden.size() <= 6 && std::all_of(hidden.begin(), hidden.end(), [](int x) { return x >= 1 && x <= 128; });
        if (bad || in < 1 || in > 64 || out < 1 || out > 64 || !hidden_ok) {
            fail("malformed net (in 1..64, hidden up to 6 layers of 1..128, out 1..64)");
            return;
        }
        net.sizes = {in};
        net.sizes.insert(net.sizes.end(), hidden.begin(), hidden.end());
        net.sizes.push_back(out);
        init_net(net); // untrained unless its file is there (a missing file is not an error: the net outputs 0)
        std::string why;
        if (!load_net(net, why) && why.rfind("no weights at", 0) != 0) {
            fail(why);
            return;
        }
        law_.nets.push_back(std::move(net));
    }

    void declare_field(const Words& w)
    {
        if (!w.name(1) || keyword(w.text(1))) {
            fail("'field' needs a name that is not a keyword");
            return;
        }
        if (law_.field_id(w.text(1)) >= 0) {
            fail("field '" + w.text(1) + "' declared twice");
            return;
        }
        FieldDecl decl;
        decl.name = w.text(1);
        bool good = true;
        for (std::size_t i = 2; good && !w.end(i);) {
            const std::string& option = w.text(i++);
            if (option == "init") good = bound(w, i, decl.init);
            else if (option == "range") good = bound(w, i, decl.lo) && bound(w, i, decl.hi) && decl.lo <= decl.hi;
            else if (option == "unit") {
                good = w.name(i);
                decl.unit = w.text(i++);
            } else if (option == "static") decl.is_static = true;
            else if (option == "clamp") decl.clamp = true;
            else good = false;
        }
        if (!good) {
            fail("malformed field declaration (expected init N, range LO HI, unit U, static, clamp)");
            return;
        }
        law_.fields.push_back(std::move(decl));
    }

    // `derive NAME ...` with NAME not yet a field declares a derived field.
    void declare_derived(const Words& w)
    {
        if (!w.name(1) || law_.field_id(w.text(1)) >= 0 || keyword(w.text(1))) return;
        FieldDecl decl;
        decl.name = w.text(1);
        decl.derived = true;
        law_.fields.push_back(std::move(decl));
    }

    // -- pass 2 --

    void leave_term(const Words&) { current_ = -1; }

    void param(const Words& w)
    {
        current_ = -1;
        if (!w.name(1) || keyword(w.text(1)) || !w.sym(2, "=")) {
            fail("expected 'param NAME = expression'");
            return;
        }
        if (law_.param_id(w.text(1)) >= 0 || law_.field_id(w.text(1)) >= 0) {
            fail("'" + w.text(1) + "' is already a param or a field");
            return;
        }
        const int e = expression(w, 3, nullptr);
        if (e < 0) return;
        if (!scalar(law_, e)) {
            fail("a param cannot read a field");
            return;
        }
        // Evaluated once, on a one-cell lattice at h = 1 (what a param cannot know yet is 0).
        double v = 0.0;
        if (!evaluate_scalar(law_, e, 1.0, 0.0, v)) v = 0.0;
        law_.param_names.push_back(w.text(1));
        law_.param_values.push_back(v);
    }

    void term(const Words& w)
    {
        if (!w.name(1) || !w.end(2)) {
            fail("expected 'term NAME'");
            current_ = -1;
            return;
        }
        if (index_named(law_.terms, w.text(1), [](const Term& t) -> const std::string& { return t.name; }) >= 0) {
            fail("term '" + w.text(1) + "' declared twice");
        }
        Term t;
        t.name = w.text(1);
        t.where = *where_;
        law_.terms.push_back(std::move(t));
        current_ = static_cast<int>(law_.terms.size()) - 1;
        lets_.clear();
    }

    void let(const Words& w)
    {
        if (term_or_fail("let") == nullptr) return;
        if (!w.name(1) || !w.sym(2, "=")) {
            fail("expected 'let NAME = expression'");
            return;
        }
        const std::string& nm = w.text(1);
        if (keyword(nm) || law_.field_id(nm) >= 0 || law_.param_id(nm) >= 0 || lets_.count(nm) != 0) {
            fail("'" + nm + "' is already a keyword, field, param or let");
            return;
        }
        const int e = expression(w, 3, &lets_);
        if (e >= 0) lets_.emplace(nm, e);
    }

    void derive(const Words& w)
    {
        current_ = -1;
        const int target = w.name(1) ? law_.field_id(w.text(1)) : -1;
        const bool adds = w.sym(2, "+") && w.sym(3, "=");
        if (target < 0 || !(adds || w.sym(2, "="))) {
            fail("expected 'derive FIELD = expression' or 'derive FIELD += expression'");
            return;
        }
        if (!adds && set_by_derive_.count(target) != 0) {
            fail("field '" + w.text(1) + "' is derived twice with '=' (use '+=' to add to it)");
            return;
        }
        const int e = expression(w, adds ? 4 : 3, nullptr);
        if (e < 0) return;
        law_.fields[static_cast<std::size_t>(target)].derived = true;
        if (!adds) set_by_derive_.insert(target);
        law_.derives.push_back(Derive{target, adds, *where_, e});
    }

    void learned(const Words& w)
    {
        Term* t = term_or_fail("learned");
        if (t == nullptr) return;
        if (w.name(1, "d")) {
            const int target = w.name(2) ? law_.field_id(w.text(2)) : -1;
            if (target < 0 || !w.sym(3, "=")) {
                fail("expected 'learned d FIELD = expression'");
                return;
            }
            const int e = expression(w, 4, &lets_);
            if (e >= 0) t->learned.push_back(Equation{target, e});
        } else if (w.name(1, "max_dt") && w.sym(2, "=")) {
            static const char* kMessage = "learned max_dt must be a number that does not read dt";
            const int e = expression(w, 3, nullptr, kMessage);
            if (e < 0) return;
            if (!scalar(law_, e) || reads_dt(law_, e)) {
                fail(kMessage);
                return;
            }
            t->learned_max_dt = e;
        } else {
            fail("expected 'learned d FIELD = expression' or 'learned max_dt = expression'");
        }
    }

    void equation(const Words& w)
    {
        Term* t = term_or_fail("d");
        if (t == nullptr) return;
        const int target = w.name(1) ? law_.field_id(w.text(1)) : -1;
        if (target < 0 || !w.sym(2, "=")) {
            fail("expected 'd FIELD = expression' with a declared field");
            return;
        }
        const int e = expression(w, 3, &lets_);
        if (e >= 0) t->equations.push_back(Equation{target, e});
    }

    // `conserves A + B C`: A and B conserved together, C alone.
    void conserves(const Words& w)
    {
        Term* t = term_or_fail("conserves");
        if (t == nullptr) return;
        bool joined = false;
        for (std::size_t i = 1; !w.end(i); ++i) {
            if (w.sym(i, "+")) {
                joined = true;
                continue;
            }
            const int f = w.name(i) ? law_.field_id(w.text(i)) : -1;
            if (f < 0) {
                fail("conserves: '" + w.text(i) + "' is not a field");
                continue;
            }
            if (joined && !t->conserves.empty()) t->conserves.back().push_back(f);
            else t->conserves.push_back({f});
            joined = false;
        }
    }

    void max_dt(const Words& w)
    {
        Term* t = term_or_fail("max_dt");
        if (t == nullptr) return;
        if (!w.sym(1, "=")) {
            fail("expected 'max_dt = expression'");
            return;
        }
        const int e = expression(w, 2, nullptr);
        if (e < 0) return;
        if (!scalar(law_, e)) fail("max_dt must be a number: use maxof/minof/sumof to reduce a field");
        else if (reads_dt(law_, e)) fail("max_dt sets the step: it cannot read dt");
        else t->max_dt = e;
    }

    // -- the whole law --

    void validate()
    {
        for (Term& term : law_.terms) {
            const std::string at = term.where + ": term '" + term.name + "' ";
            std::set<int> reads, writes;
            auto read = [&](int rhs) {
                visit(law_, rhs, [&](const Node& n) {
                    if (n.op == Op::Field) reads.insert(n.index);
                });
            };
            for (const Equation& eq : term.equations) {
                read(eq.rhs);
                writes.insert(eq.target);
                const FieldDecl& d = law_.fields[static_cast<std::size_t>(eq.target)];
                if (d.is_static) errors_.push_back(at + "writes static field '" + d.name + "'");
                if (d.derived) errors_.push_back(at + "writes derived field '" + d.name + "'");
            }
            if (term.equations.empty()) errors_.push_back(at + "has no equations");
            for (const Equation& eq : term.learned) {
                read(eq.rhs);
                if (writes.count(eq.target) == 0) {
                    errors_.push_back(at + "has a learned equation for '" + law_.fields[static_cast<std::size_t>(eq.target)].name +
                        "', which its own equations do not write");
                }
            }
            for (const std::vector<int>& group : term.conserves) {
                std::string names;
                bool written = false;
                for (const int f : group) {
                    written = written || writes.count(f) != 0;
                    names += (names.empty() ? "" : " + ") + law_.fields[static_cast<std::size_t>(f)].name;
                }
                if (!written) errors_.push_back(at + "conserves '" + names + "' but never writes it");
            }
            term.reads.assign(reads.begin(), reads.end());
            term.writes.assign(writes.begin(), writes.end());
        }
    }

    // Derives run per field in the order fields are first derived, each field's '=' before its '+='.
    void order_derives()
    {
        std::vector<int> first_seen;
        for (const Derive& d : law_.derives) {
            if (std::find(first_seen.begin(), first_seen.end(), d.target) == first_seen.end()) first_seen.push_back(d.target);
        }
        std::vector<Derive> ordered;
        for (const int f : first_seen) {
            for (const bool adds : {false, true}) {
                std::copy_if(law_.derives.begin(), law_.derives.end(), std::back_inserter(ordered),
                    [&](const Derive& d) { return d.target == f && d.accumulate == adds; });
            }
        }
        law_.derives = std::move(ordered);
    }

    Law& law_;
    std::vector<std::string>& errors_;
    const std::string* where_ = nullptr;
    bool in_creature_ = false;
    int current_ = -1;
    Lets lets_;
    std::set<int> set_by_derive_;
};

} // namespace

// Scalar semantics of the CPU (src/field/Law.cpp:757-860): double arithmetic, guarded division, clamped exp/log/sqrt,
// and zero times anything is zero without looking at the anything.
bool evaluate_scalar(const Law& law, int id, double h, double dt, double& out)
{
    const Node& n = law.nodes[static_cast<std::size_t>(id)];
    double v[3] = {0.0, 0.0, 0.0};
    auto args = [&](std::size_t count) {
        for (std::size_t k = 0; k < count; ++k) {
            if (!evaluate_scalar(law, n.args[k], h, dt, v[k])) return false;
        }
        return true;
    };
    switch (n.op) {
    case Op::Const: out = n.number; return true;
    case Op::Param: out = law.param_values[static_cast<std::size_t>(n.index)]; return true;
    case Op::Cell: out = h; return true;
    case Op::Dt: out = dt; return true;
    case Op::Shift: case Op::MaxOf: case Op::MinOf: return args(1) && (out = v[0], true); // of one number: that number
    case Op::Lap: case Op::Gx: case Op::Gy: case Op::Gz: return args(1) && (out = 0.0, true); // nothing varies
    case Op::Mul:
        if (!args(1)) return false;
        if (v[0] == 0.0) {
            out = 0.0;
            return true;
        }
        if (!evaluate_scalar(law, n.args[1], h, dt, v[1])) return false;
        out = v[1] == 0.0 ? 0.0 : v[0] * v[1];
        return true;
    default:
        break;
    }
    using Unary = double (*)(double);
    using Binary = double (*)(double, double);
    static const std::map<Op, Unary> unary = {
        {Op::Neg, [](double a) { return -a; }},
        {Op::Abs, [](double a) { return std::fabs(a); }},
        {Op::Sqrt, [](double a) { return std::sqrt(std::max(0.0, a)); }},
        {Op::Exp, [](double a) { return std::exp(std::min(a, 80.0)); }},
        {Op::Log, [](double a) { return std::log(std::max(a, 1e-30)); }},
        {Op::Step, [](double a) { return a > 0.0 ? 1.0 : 0.0; }},
        {Op::Pos, [](double a) { return std::max(a, 0.0); }},
    };
    static const std::map<Op, Binary> binary = {
        {Op::Add, [](double a, double b) { return a + b; }},
        {Op::Sub, [](double a, double b) { return a - b; }},
        {Op::Div, [](double a, double b) { return b == 0.0 ? 0.0 : a / b; }},
        {Op::Pow, [](double a, double b) { return std::pow(a, b); }},
        {Op::Min, [](double a, double b) { return std::min(a, b); }},
        {Op::Max, [](double a, double b) { return std::max(a, b); }},
    };
    if (const auto u = unary.find(n.op); u != unary.end()) return args(1) && (out = u->second(v[0]), true);
    if (const auto b = binary.find(n.op); b != binary.end()) return args(2) && (out = b->second(v[0], v[1]), true);
    if (n.op == Op::Clamp) return args(3) && (out = std::clamp(v[0], v[1], std::max(v[1], v[2])), true);
    return false;
}

Law compile(const std::vector<Source>& sources, std::vector<std::string>& errors)
{
    Law law;
    std::vector<Line> lines;
    for (const Source& src : sources) {
        std::istringstream stream(src.text);
        std::string raw;
        for (int number = 1; std::getline(stream, raw); ++number) {
            if (!raw.empty() && raw.back() == '\r') raw.pop_back();
            std::string where = src.name + ":" + std::to_string(number);
            std::string error;
            std::vector<Token> tokens = Scanner(raw).all(error);
            if (!error.empty()) errors.push_back(where + ": " + error);
            else if (tokens.size() > 1) lines.push_back(Line{std::move(where), std::move(tokens)});
        }
    }
    Compiler(law, errors).run(lines);
    return law;
}

} // namespace fe::law
