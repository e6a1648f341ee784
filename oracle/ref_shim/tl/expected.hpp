// Stand-in for tl::expected (empty submodule); the kernel libraries only need the header.
#pragma once
#include <string>
#include <utility>
namespace tl {
template <typename E> struct unexpected { E e; };
template <typename E> unexpected<E> make_unexpected(E e) { return unexpected<E>{std::move(e)}; }
}  // namespace tl
