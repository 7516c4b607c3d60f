// A law given as its IR JSON (src/field/ir/LawIR.cpp:528-593's format) instead of its text.
#pragma once

#include "ir.hpp"
#include "law.hpp"

#include <string>

namespace fe {

// Rebuilds the Law from the IR JSON (the instructions become its expression nodes; nets' weights from their files) and
// lowers it; false with `why` when the JSON is malformed, names what this backend does not know, or does not lower
// back to itself.
bool law_from_ir_json(const std::string& json, law::Law& out, ir::Module& module, std::string& why);

} // namespace fe
