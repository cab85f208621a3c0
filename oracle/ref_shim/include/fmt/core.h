// Oracle test infrastructure, not product code.
// Stand-in for fmt's header: the hydro hot-path sources include it
// (source/Boundaries.hpp) but call nothing from it; the configuration reader
// (source/MosscapConfig.hpp) formats error messages with fmt::format, which
// here returns its format string unformatted.
#pragma once

#include <string>

namespace fmt {

template <class... Args>
std::string format(const char* f, Args&&...) {
    return std::string(f);
}

} // namespace fmt
