// The law language: text to fields, params, terms and their expression graphs.
//
// The language is the reference's, unchanged, so a .law file is a drop-in (grammar and keywords:
// src/field/Law.hpp:16-37, Law.cpp:47-410 tokenizer/parser, Law.cpp:1662-2420 compile_law). This is a fresh
// implementation: expressions live in an arena of nodes addressed by index, and what the GPU backend does not run
// (creatures, `show` lines) is read past, not built.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fe::law {

// Operations, in the reference's enumeration (src/field/LawNode.hpp:15-67).
enum class Op : std::uint8_t {
    Const, Param, Cell, Rim, Field, Neg, Add, Sub, Mul, Div, Pow, Min, Max, Abs, Sqrt, Exp, Log, Step, Pos, Clamp,
    Lap, Gx, Gy, Gz, Diffuse, Adv, Distance, Poisson, MaxOf, MinOf, SumOf, Fall, Spread, Topple, Shift, Local,
    Mlp, Flux, LDiffuse, Dt, Tridiag, ShiftT, GxT, GyT, GzT,
};

const char* op_name(Op op);

struct Node {
    Op op = Op::Const;
    double number = 0.0;
    int index = -1;      // field, param, net, or the axis of a tridiag
    int iterations = 0;  // poisson
    std::vector<int> args;
};

struct FieldDecl {
    std::string name;
    double init = 0.0;
    double lo = -1e30;
    double hi = 1e30;
    bool clamp = false;
    bool is_static = false;
    bool derived = false;
    std::string unit;
};

struct Equation {
    int target = -1;
    int rhs = -1; // node id
};

struct Term {
    std::string name;
    std::string where;
    std::vector<Equation> equations;
    std::vector<std::vector<int>> conserves;
    int max_dt = -1;
    std::vector<Equation> learned;
    int learned_max_dt = -1;
    std::vector<int> reads;
    std::vector<int> writes;
};

struct Derive {
    int target = -1;
    bool accumulate = false;
    std::string where;
    int rhs = -1;
};

struct NetDecl {
    std::string name;
    std::vector<int> sizes;
    std::string act;
    bool half = false;
    std::string file;
    // Its parameters (Net.hpp's layout): per layer the out x in weights row by row, then the out biases; the inputs'
    // shift and scale; the output scale. Untrained (no file) it starts from init_net; `loaded` once a file was read.
    std::vector<float> weights, in_shift, in_scale;
    float out_scale = 1.0f;
    bool loaded = false;
    [[nodiscard]] int layers() const { return static_cast<int>(sizes.size()) - 1; }
    [[nodiscard]] std::size_t weight_offset(int layer) const;
    [[nodiscard]] std::size_t parameter_count() const { return weight_offset(layers()); }
};

// The starting weights of a net (Net.cpp:241-262): hidden layers uniform in +-sqrt(6 / (in + out)) from a hash of the
// net's name, layer and index; the last layer and every bias zero, so an untrained net outputs 0.
void init_net(NetDecl& net, std::uint64_t seed = 0);
// Reads the net's weight file (Net.cpp:264-333's text format). False with "no weights at ..." when there is no file.
bool load_net(NetDecl& net, std::string& error);

struct Law {
    std::vector<Node> nodes;
    std::vector<FieldDecl> fields;
    std::vector<std::string> param_names;
    std::vector<double> param_values;
    std::vector<Term> terms;
    std::vector<Derive> derives;
    std::vector<NetDecl> nets;

    [[nodiscard]] int field_id(const std::string& name) const;
    [[nodiscard]] int param_id(const std::string& name) const;
    [[nodiscard]] int net_id(const std::string& name) const;
};

struct Source {
    std::string name;
    std::string text;
};

// Compiles the sources together (several files may make one law). On failure `errors` holds "source:line: message"
// lines, in source order, and the returned law is not to be used.
Law compile(const std::vector<Source>& sources, std::vector<std::string>& errors);

// Evaluates a scalar expression the way the reference's CPU does (in double; Law.cpp:757-860 for the scalar paths).
// Field reads and whole-lattice ops make it non-scalar: returns false then.
bool evaluate_scalar(const Law& law, int node, double h, double dt, double& out);

} // namespace fe::law
