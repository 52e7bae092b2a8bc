// Stand-in for the reference's dr/views/csr_matrix_view.hpp, used ONLY to
// compile the reference's own include/dr/detail/generate_csr.hpp into the
// oracle/_ref/ref_gen golden-vector generator.  The real header needs range-v3
// (rng::view_interface, rng::views) which is not available offline; the
// generators only need the constructor, size(), shape() and the three data
// pointers, which this minimal class provides.
#pragma once
#include <algorithm>
#include <cassert>
#include <vector>
#include <cstddef>
#include <iterator>

#include <dr/detail/index.hpp>

namespace dr::views {

template <typename T, typename I, typename TIter = T *, typename IIter = I *>
class csr_matrix_view {
public:
  using key_type = dr::index<I>;
  csr_matrix_view() = default;
  csr_matrix_view(TIter values, IIter rowptr, IIter colind, key_type shape,
                  std::size_t nnz, std::size_t rank)
      : values_(values), rowptr_(rowptr), colind_(colind), shape_(shape),
        nnz_(nnz), rank_(rank) {}
  key_type shape() const noexcept { return shape_; }
  std::size_t size() const noexcept { return nnz_; }
  std::size_t rank() const { return rank_; }
  TIter values_data() const { return values_; }
  IIter rowptr_data() const { return rowptr_; }
  IIter colind_data() const { return colind_; }

private:
  TIter values_{};
  IIter rowptr_{};
  IIter colind_{};
  key_type shape_{};
  std::size_t nnz_ = 0;
  std::size_t rank_ = 0;
};

template <typename TIter, typename IIter, typename... Args>
csr_matrix_view(TIter, IIter, IIter, Args &&...)
    -> csr_matrix_view<std::iter_value_t<TIter>, std::iter_value_t<IIter>,
                       TIter, IIter>;

} // namespace dr::views
