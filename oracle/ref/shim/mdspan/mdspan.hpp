// Minimal column-major multidimensional view used only to compile the
// reference MACIS headers for the CPU oracle (test infrastructure).
//
// The reference names Kokkos::mdspan<T, Kokkos::dextents<size_t,R>,
// Kokkos::layout_left> (include/macis/types.hpp:19-24) and the namespace
// alias MDSPAN_IMPL_STANDARD_NAMESPACE::MDSPAN_IMPL_PROPOSED_NAMESPACE.
// Only dynamic extents with layout_left are provided: data_handle(),
// extent(i), size() and operator()(i, j, ...), which is all the hot-path
// headers use, and a contiguous-only submdspan for the FCIDUMP reader.
#pragma once
#include <array>
#include <cstddef>
#include <stdexcept>
#include <type_traits>
#include <utility>

#define MDSPAN_IMPL_STANDARD_NAMESPACE Kokkos
#define MDSPAN_IMPL_PROPOSED_NAMESPACE Experimental

namespace Kokkos {
namespace Experimental {}

struct layout_left {};
struct full_extent_t {};
inline constexpr full_extent_t full_extent{};

template <typename IndexType, size_t Rank>
struct dextents {
  using index_type = IndexType;
  static constexpr size_t rank() { return Rank; }
};

template <typename T, typename Extents, typename Layout = layout_left>
class mdspan {
  static constexpr size_t R = Extents::rank();
  T* p_ = nullptr;
  std::array<size_t, R> ext_{};

 public:
  using element_type = T;
  using index_type = typename Extents::index_type;

  mdspan() = default;
  template <typename... I,
            typename = std::enable_if_t<sizeof...(I) == R>>
  mdspan(T* p, I... e) : p_(p), ext_{static_cast<size_t>(e)...} {}

  T* data_handle() const { return p_; }
  size_t extent(size_t i) const { return ext_[i]; }
  static constexpr size_t rank() { return R; }
  size_t size() const {
    size_t s = 1;
    for(size_t i = 0; i < R; ++i) s *= ext_[i];
    return s;
  }

  template <typename... I>
  T& operator()(I... idx) const {
    static_assert(sizeof...(I) == R, "wrong number of indices");
    const size_t ii[R] = {static_cast<size_t>(idx)...};
    size_t off = 0, stride = 1;
    for(size_t d = 0; d < R; ++d) {
      off += ii[d] * stride;
      stride *= ext_[d];
    }
    return p_[off];
  }
};

namespace detail {
template <typename S>
size_t slice_first(const S& s) {
  if constexpr(std::is_same_v<S, full_extent_t>)
    return 0;
  else
    return static_cast<size_t>(s.first);
}
template <typename S>
size_t slice_extent(const S& s, size_t full) {
  if constexpr(std::is_same_v<S, full_extent_t>)
    return full;
  else
    return static_cast<size_t>(s.second) - static_cast<size_t>(s.first);
}
template <typename T, size_t R, size_t... I>
mdspan<T, dextents<size_t, R>, layout_left> make_view(
    T* p, const std::array<size_t, R>& e, std::index_sequence<I...>) {
  return mdspan<T, dextents<size_t, R>, layout_left>(p, e[I]...);
}
}  // namespace detail

// submdspan with pair / full_extent slices, for the views that stay
// contiguous in column-major order (every dimension before the last one
// sliced to less than its extent keeps its full extent), which is how
// src/macis/fcidump.cxx uses it when the leading dimensions equal norb.
template <typename T, typename E, typename L, typename... S>
auto submdspan(const mdspan<T, E, L>& m, S... slices) {
  constexpr size_t R = sizeof...(S);
  static_assert(R == E::rank(), "one slice per dimension");
  const size_t first[R] = {detail::slice_first(slices)...};
  std::array<size_t, R> ext{};
  size_t d = 0;
  ((ext[d] = detail::slice_extent(slices, m.extent(d)), ++d), ...);
  size_t off = 0, stride = 1;
  bool cut = false;
  for(size_t i = 0; i < R; ++i) {
    if(cut && ext[i] > 1)
      throw std::runtime_error("submdspan: strided views are not supported");
    off += first[i] * stride;
    stride *= m.extent(i);
    if(ext[i] != m.extent(i)) cut = true;
  }
  return detail::make_view<T, R>(m.data_handle() + off, ext,
                                 std::make_index_sequence<R>{});
}

}  // namespace Kokkos
