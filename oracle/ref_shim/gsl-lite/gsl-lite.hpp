// Minimal stand-in for the gsl-lite library (absent from this machine) covering only what the
// reference headers compiled by oracle/build_ref.py use: span, narrow, narrow_cast, make_span.
// Test infrastructure of the reference-code harness; not part of the product.
#pragma once
#include <cstddef>
#include <span>
#include <utility>

namespace gsl {
template <class T, std::size_t E = std::dynamic_extent>
using span = std::span<T, E>;
template <class T, class U>
constexpr T narrow_cast(U&& u) noexcept { return static_cast<T>(std::forward<U>(u)); }
template <class T, class U>
constexpr T narrow(U u) { return static_cast<T>(u); }
template <class T>
constexpr span<T> make_span(T* p, std::size_t n) { return span<T>(p, n); }
template <class C>
constexpr auto make_span(C& c) { return span<typename C::value_type>(c.data(), c.size()); }
} // namespace gsl
namespace gsl_lite = gsl;
