// Stand-in for tl::optional (empty submodule in the reference tree), on std::optional.
#pragma once
#include <optional>
namespace tl {
using std::optional;
using std::nullopt;
}  // namespace tl
