// The law as an SSA program: one graph for the whole law, every value computed once (structural hashing across all terms
// and derives), constants folded with the CPU's double semantics, each instruction knowing its shape (one number or one
// per cell) and how far from its cell it reads; per term a Program of stages (stored before the term's kernel), the
// fused gather, and whether it stores in place or ping-pongs.
//
// The lowering rules are the reference's, so a law lowers to the same program (src/field/ir/LawIR.hpp:12-26,
// LawIR.cpp:140-526: folding 162-250, shapes/radii 254-288, the cost model with kInlineBudget = 48 314-338,
// reach and in-place 357-433), and to_json writes the reference's IR JSON format (LawIR.cpp:528-593), so tools that
// read it (tools/lawjax) read ours.
#pragma once

#include "law.hpp"

#include <string>
#include <vector>

namespace fe::ir {

using law::Op;

enum class Shape : unsigned char { Scalar, Cell };

struct Inst {
    Op op = Op::Const;
    Shape shape = Shape::Scalar;
    double number = 0.0;
    int index = -1;
    int iterations = 0;
    int offset[3] = {0, 0, 0};
    std::vector<int> args;
    int radius = 0;
    bool global = false;
    bool net = false;
    int uses = 0;
    int cost = 1;
};

struct Equation {
    int target = -1;
    int value = -1;
};

struct Program {
    std::string name;
    std::vector<Equation> equations;
    std::vector<int> stages;
    std::vector<int> limit_stages;
    bool in_place = false;
    int max_dt = -1;
    std::vector<int> reads;
    std::vector<int> writes;
    std::vector<std::vector<int>> conserves;
    bool accumulate = false;
};

struct Module {
    std::vector<Inst> insts;
    std::vector<Program> terms;
    std::vector<Program> learned;
    std::vector<Program> derives;
    std::vector<char> materialized;
    int folded = 0;
    int shared = 0;

    [[nodiscard]] bool is_stage(int id) const
    {
        const Inst& in = insts[static_cast<std::size_t>(id)];
        return in.global || in.net || materialized[static_cast<std::size_t>(id)] != 0;
    }
};

constexpr int kInlineBudget = 48;

// `prelower`: nodes [0, prelower) are lowered first, in order (a law rebuilt from IR instructions keeps their ids).
Module lower(const law::Law& law, int prelower = 0);
// The code generator's own staging on top of the IR's (the IR, and its JSON, stay the reference's): a value that
// stencil ops read at several offsets, each read inlining its whole expression, is stored once when its inlined cost
// times the points read passes the inline budget (the IR's rule counts one reader at a time). Stored or inlined it is
// the same fp32 number, so results do not change. The programs' stage lists are redone; in_place is kept.
void widen_stages(Module& m);
std::string to_json(const Module& m, const law::Law& law);
std::string describe(const Module& m, const law::Law& law);

} // namespace fe::ir
