/* Stand-in for the one tlx header missing from the reference's vendored tlx snapshot. */
#pragma once
#include <type_traits>
namespace tlx {
template <bool B, typename T = void>
using enable_if = std::enable_if<B, T>;
} // namespace tlx
