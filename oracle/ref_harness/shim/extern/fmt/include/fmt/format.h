// Host-only stand-in for the `fmt` formatting library, which the reference
// includes through a relative path into its (empty) extern/ submodule. The
// oracle harness never relies on formatted log text, so format() returns the
// format string unchanged.
#pragma once
#include <stdexcept>
#include <string>
#include <string_view>

namespace fmt {
struct format_error : std::runtime_error {
	using std::runtime_error::runtime_error;
};
inline std::string runtime(std::string s) { return s; }
template <typename... Args>
std::string format(std::string_view f, Args&&...) { return std::string(f); }
template <typename T, typename Char = char, typename Enable = void>
struct formatter {};
} // namespace fmt
