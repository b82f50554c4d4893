// Minimal column-major multidimensional view used only to compile the
// reference MACIS headers for the CPU oracle (test infrastructure).
//
// The reference names Kokkos::mdspan<T, Kokkos::dextents<size_t,R>,
// Kokkos::layout_left> (include/macis/types.hpp:19-24) and the namespace
// alias MDSPAN_IMPL_STANDARD_NAMESPACE::MDSPAN_IMPL_PROPOSED_NAMESPACE.
// Only dynamic extents with layout_left are provided: data_handle(),
// extent(i), size() and operator()(i, j, ...), which is all the hot-path
// headers use.
#pragma once
#include <array>
#include <cstddef>
#include <type_traits>

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

}  // namespace Kokkos
