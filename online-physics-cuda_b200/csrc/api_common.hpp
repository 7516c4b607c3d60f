// Status and error-message helpers shared by the C-ABI translation units.
#pragma once

#include <string>

namespace fe {

// Records `message` for fe_last_error() on this thread and returns `code`.
int fail(int code, const std::string& message);
// Clears the message and returns FE_OK.
int ok();
const char* last_error();

} // namespace fe
