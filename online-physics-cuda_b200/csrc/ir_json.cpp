// A law given as its IR JSON (the format src/field/ir/LawIR.cpp:528-593 writes: fields, params, nets, instructions and
// the programs), turned back into a Law whose expression graph is the instructions themselves. The reference's own
// CUDA backend starts from the in-memory Law (CudaSolver::create lowers it, CudaSolver.cpp:122); a backend loaded
// beside it gets the same graph through this text, which the reference can always write (ir::to_json).
//
// The rebuilt law is lowered again by this backend's lowering and written back: it must give the JSON it came from
// (same instructions, same programs), or the law is refused, so what runs is exactly what the caller's IR says.
#include "ir_json.hpp"

#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <tuple>

namespace fe {

namespace {

// ---- a small JSON reader -----------------------------------------------------------------------------------------------

struct Json;
using JsonPtr = std::shared_ptr<Json>;

struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<JsonPtr> items;                       // Array
    std::vector<std::pair<std::string, JsonPtr>> members; // Object, in order

    [[nodiscard]] const Json* get(const std::string& key) const
    {
        for (const auto& [k, v] : members) {
            if (k == key) return v.get();
        }
        return nullptr;
    }
};

class Reader {
public:
    explicit Reader(const std::string& s) : s_(s) {}

    JsonPtr document(std::string& why)
    {
        JsonPtr v = value();
        blanks();
        if (v && i_ != s_.size()) {
            error_ = "text after the JSON value";
            v = nullptr;
        }
        if (!v) why = "IR JSON: " + error_ + " at offset " + std::to_string(i_);
        return v;
    }

private:
    void blanks()
    {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\n' || s_[i_] == '\r' || s_[i_] == '\t')) ++i_;
    }
    bool eat(char c)
    {
        blanks();
        if (i_ < s_.size() && s_[i_] == c) {
            ++i_;
            return true;
        }
        return false;
    }
    JsonPtr fail(const char* what)
    {
        if (error_.empty()) error_ = what;
        return nullptr;
    }

    JsonPtr value()
    {
        blanks();
        if (i_ >= s_.size()) return fail("unexpected end");
        auto v = std::make_shared<Json>();
        const char c = s_[i_];
        if (c == '{') {
            ++i_;
            v->kind = Json::Object;
            if (eat('}')) return v;
            do {
                blanks();
                std::string key;
                if (!string(key)) return fail("expected a key");
                if (!eat(':')) return fail("expected ':'");
                JsonPtr m = value();
                if (!m) return nullptr;
                v->members.emplace_back(std::move(key), std::move(m));
            } while (eat(','));
            if (!eat('}')) return fail("expected '}'");
            return v;
        }
        if (c == '[') {
            ++i_;
            v->kind = Json::Array;
            if (eat(']')) return v;
            do {
                JsonPtr item = value();
                if (!item) return nullptr;
                v->items.push_back(std::move(item));
            } while (eat(','));
            if (!eat(']')) return fail("expected ']'");
            return v;
        }
        if (c == '"') {
            v->kind = Json::String;
            if (!string(v->str)) return fail("bad string");
            return v;
        }
        for (const auto& [word, kind, truth] : {std::tuple{"true", Json::Bool, true}, {"false", Json::Bool, false}, {"null", Json::Null, false}}) {
            const std::size_t n = std::char_traits<char>::length(word);
            if (s_.compare(i_, n, word) == 0) {
                i_ += n;
                v->kind = kind;
                v->b = truth;
                return v;
            }
        }
        const char* start = s_.c_str() + i_;
        char* end = nullptr;
        v->num = std::strtod(start, &end);
        if (end == start) return fail("unexpected character");
        i_ += static_cast<std::size_t>(end - start);
        v->kind = Json::Number;
        return v;
    }

    bool string(std::string& out)
    {
        if (i_ >= s_.size() || s_[i_] != '"') return false;
        ++i_;
        while (i_ < s_.size() && s_[i_] != '"') {
            char c = s_[i_++];
            if (c == '\\') {
                if (i_ >= s_.size()) return false;
                const char e = s_[i_++];
                c = e == 'n' ? '\n' : e == 't' ? '\t' : e == 'r' ? '\r' : e; // \" \\ \/ as themselves
            }
            out.push_back(c);
        }
        if (i_ >= s_.size()) return false;
        ++i_;
        return true;
    }

    const std::string& s_;
    std::size_t i_ = 0;
    std::string error_;
};

bool same(const Json& a, const Json& b)
{
    if (a.kind != b.kind) return false;
    switch (a.kind) {
    case Json::Null: return true;
    case Json::Bool: return a.b == b.b;
    case Json::Number: return a.num == b.num || (std::isnan(a.num) && std::isnan(b.num));
    case Json::String: return a.str == b.str;
    case Json::Array:
        if (a.items.size() != b.items.size()) return false;
        for (std::size_t i = 0; i < a.items.size(); ++i) {
            if (!same(*a.items[i], *b.items[i])) return false;
        }
        return true;
    case Json::Object:
        if (a.members.size() != b.members.size()) return false;
        for (const auto& [k, v] : a.members) {
            const Json* w = b.get(k);
            if (w == nullptr || !same(*v, *w)) return false;
        }
        return true;
    }
    return false;
}

// ---- the law ---------------------------------------------------------------------------------------------------------

class Builder {
public:
    Builder(const Json& doc, law::Law& law, std::string& why) : doc_(doc), law_(law), why_(why) {}

    bool run()
    {
        return fields() && params() && nets() && insts() && programs();
    }

private:
    const Json* array(const Json& obj, const char* key)
    {
        const Json* v = obj.get(key);
        if (v == nullptr || v->kind != Json::Array) {
            why_ = std::string("IR JSON: no array '") + key + "'";
            return nullptr;
        }
        return v;
    }
    static double num(const Json& obj, const char* key, double fallback = 0.0)
    {
        const Json* v = obj.get(key);
        return v != nullptr && v->kind == Json::Number ? v->num : fallback;
    }
    static bool flag(const Json& obj, const char* key)
    {
        const Json* v = obj.get(key);
        return v != nullptr && v->kind == Json::Bool && v->b;
    }
    static std::string text(const Json& obj, const char* key)
    {
        const Json* v = obj.get(key);
        return v != nullptr && v->kind == Json::String ? v->str : std::string();
    }
    static std::vector<int> ints(const Json* v)
    {
        std::vector<int> out;
        if (v == nullptr || v->kind != Json::Array) return out;
        for (const JsonPtr& x : v->items) out.push_back(static_cast<int>(x->num));
        return out;
    }

    bool fields()
    {
        const Json* a = array(doc_, "fields");
        if (a == nullptr) return false;
        for (const JsonPtr& f : a->items) {
            law::FieldDecl d;
            d.name = text(*f, "name");
            d.init = num(*f, "init");
            d.lo = num(*f, "lo");
            d.hi = num(*f, "hi");
            d.clamp = flag(*f, "clamp");
            d.is_static = flag(*f, "static");
            d.derived = flag(*f, "derived");
            law_.fields.push_back(std::move(d));
        }
        return true;
    }

    bool params()
    {
        const Json* a = array(doc_, "params");
        if (a == nullptr) return false;
        for (const JsonPtr& p : a->items) {
            law_.param_names.push_back(text(*p, "name"));
            law_.param_values.push_back(num(*p, "value"));
        }
        return true;
    }

    // A net's weights come from its file (the untrained start when it has none), as when the law text is compiled.
    bool nets()
    {
        const Json* a = array(doc_, "nets");
        if (a == nullptr) return false;
        for (const JsonPtr& n : a->items) {
            law::NetDecl net;
            net.name = text(*n, "name");
            net.file = text(*n, "file");
            net.sizes = ints(n->get("sizes"));
            net.act = text(*n, "act");
            net.half = flag(*n, "half");
            if (net.sizes.size() < 2) {
                why_ = "IR JSON: net '" + net.name + "' has no sizes";
                return false;
            }
            law::init_net(net);
            std::string why;
            if (!law::load_net(net, why) && why.rfind("no weights at", 0) != 0) {
                why_ = why;
                return false;
            }
            if (flag(*n, "loaded") && !net.loaded) {
                why_ = "IR JSON: net '" + net.name + "' was loaded from " + net.file + ", which is not readable here";
                return false;
            }
            law_.nets.push_back(std::move(net));
        }
        return true;
    }

    // Each instruction becomes one node with the same id; a shift's offsets become number nodes after them.
    bool insts()
    {
        const Json* a = array(doc_, "insts");
        if (a == nullptr) return false;
        std::map<std::string, law::Op> ops;
        for (int o = 0; o <= static_cast<int>(law::Op::GzT); ++o) ops.emplace(law::op_name(static_cast<law::Op>(o)), static_cast<law::Op>(o));
        const std::size_t n = a->items.size();
        law_.nodes.resize(n);
        for (std::size_t i = 0; i < n; ++i) {
            const Json& in = *a->items[i];
            const auto op = ops.find(text(in, "op"));
            if (op == ops.end()) {
                why_ = "IR JSON: instruction " + std::to_string(i) + " has an unknown op '" + text(in, "op") + "'";
                return false;
            }
            law::Node node;
            node.op = op->second;
            node.number = num(in, "number");
            node.index = static_cast<int>(num(in, "index", -1));
            node.iterations = static_cast<int>(num(in, "iterations"));
            node.args = ints(in.get("args"));
            for (const int arg : node.args) {
                if (arg < 0 || static_cast<std::size_t>(arg) >= i) {
                    why_ = "IR JSON: instruction " + std::to_string(i) + " reads a later or missing instruction";
                    return false;
                }
            }
            if (node.op == law::Op::Shift || node.op == law::Op::ShiftT) {
                const std::vector<int> off = ints(in.get("offset"));
                for (int k = 0; k < 3; ++k) {
                    law::Node c;
                    c.number = k < static_cast<int>(off.size()) ? off[static_cast<std::size_t>(k)] : 0;
                    law_.nodes.push_back(c);
                    node.args.push_back(static_cast<int>(law_.nodes.size()) - 1);
                }
            }
            law_.nodes[i] = std::move(node);
        }
        return true;
    }

    bool program_list(const char* key, std::vector<const Json*>& out)
    {
        const Json* a = array(doc_, key);
        if (a == nullptr) return false;
        for (const JsonPtr& p : a->items) out.push_back(p.get());
        return true;
    }

    std::vector<law::Equation> equations(const Json& p) const
    {
        std::vector<law::Equation> out;
        const Json* eqs = p.get("equations");
        if (eqs == nullptr) return out;
        for (const JsonPtr& e : eqs->items) {
            const std::vector<int> pair = ints(e.get());
            if (pair.size() == 2) out.push_back(law::Equation{pair[0], pair[1]});
        }
        return out;
    }

    bool programs()
    {
        std::vector<const Json*> terms, learned, derives;
        if (!program_list("terms", terms) || !program_list("learned", learned) || !program_list("derives", derives)) return false;
        if (learned.size() != terms.size()) {
            why_ = "IR JSON: one learned program a term is expected";
            return false;
        }
        for (std::size_t t = 0; t < terms.size(); ++t) {
            law::Term term;
            term.name = text(*terms[t], "name");
            term.where = "ir:term " + term.name;
            term.equations = equations(*terms[t]);
            term.max_dt = static_cast<int>(num(*terms[t], "max_dt", -1));
            const Json* groups = terms[t]->get("conserves");
            if (groups != nullptr) {
                for (const JsonPtr& g : groups->items) term.conserves.push_back(ints(g.get()));
            }
            term.learned = equations(*learned[t]);
            term.learned_max_dt = static_cast<int>(num(*learned[t], "max_dt", -1));
            term.reads = ints(terms[t]->get("reads"));
            term.writes = ints(terms[t]->get("writes"));
            law_.terms.push_back(std::move(term));
        }
        for (const Json* p : derives) {
            const std::vector<law::Equation> eqs = equations(*p);
            if (eqs.size() != 1) {
                why_ = "IR JSON: a derive program has one equation";
                return false;
            }
            law_.derives.push_back(law::Derive{eqs[0].target, flag(*p, "accumulate"), "ir:" + text(*p, "name"), eqs[0].rhs});
        }
        const auto field_ok = [&](int f) { return f >= 0 && static_cast<std::size_t>(f) < law_.fields.size(); };
        const auto node_ok = [&](int id) { return id >= -1 && id < static_cast<int>(law_.nodes.size()); };
        for (const law::Term& t : law_.terms) {
            for (const auto* eqs : {&t.equations, &t.learned}) {
                for (const law::Equation& e : *eqs) {
                    if (!field_ok(e.target) || !node_ok(e.rhs) || e.rhs < 0) {
                        why_ = "IR JSON: term '" + t.name + "' has an equation outside the law";
                        return false;
                    }
                }
            }
            if (!node_ok(t.max_dt) || !node_ok(t.learned_max_dt)) {
                why_ = "IR JSON: term '" + t.name + "' has a max_dt outside the law";
                return false;
            }
        }
        for (const law::Derive& d : law_.derives) {
            if (!field_ok(d.target) || !node_ok(d.rhs) || d.rhs < 0) {
                why_ = "IR JSON: a derive outside the law";
                return false;
            }
        }
        return true;
    }

    const Json& doc_;
    law::Law& law_;
    std::string& why_;
};

} // namespace

bool law_from_ir_json(const std::string& json, law::Law& out, ir::Module& module, std::string& why)
{
    const JsonPtr doc = Reader(json).document(why);
    if (!doc) return false;
    const Json* version = doc->kind == Json::Object ? doc->get("version") : nullptr;
    if (version == nullptr || version->kind != Json::Number || version->num != 1.0) {
        why = "IR JSON: not a version 1 law IR";
        return false;
    }
    law::Law law;
    if (!Builder(*doc, law, why).run()) return false;
    // Every instruction lowered in id order first, the ones no program reads too (numbers the lowering folded away
    // stay in the reference's list), so each keeps its id; the programs then find them.
    module = ir::lower(law, static_cast<int>(doc->get("insts")->items.size()));
    // What this backend will run must be what the caller's IR says.
    const std::string again = ir::to_json(module, law);
    std::string why_again;
    const JsonPtr back = Reader(again).document(why_again);
    if (!back || !same(*doc, *back)) {
        why = "IR JSON: the law does not lower back to the IR it came in (a newer or edited IR?)";
        return false;
    }
    out = std::move(law);
    return true;
}

} // namespace fe
